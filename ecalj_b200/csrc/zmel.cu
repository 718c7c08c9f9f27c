// Product-basis matrix elements <psi_q(itp) | psi_{q-k}(it) M_i>: the
// muffin-tin part of get_zmel_init_gemm (m_zmel.f90:323-390) and its M->E
// change + conjugation (:546-563, :590-594).
//
// For every atom the reference runs two batched ZGEMMs with tiny K (the
// atom's valence channels, nv ~ 10-30): ppbvphiq = ppb_v^T cphiq and
// zmelt = phase cphim^H ppbvphiq, each a separate library call per atom.
// Here one launch covers all atoms: a CTA owns (atom, 16 target columns itp,
// 16 middle states it) and loops over the atom's product functions i, with
// ppb(:,:,i), the cphiq block and T = ppb^T cphiq staged in shared memory;
// consecutive threads write consecutive product-basis rows of zmelt.
#include <vector>
#include "zgemm_f64.cuh"
#include "ozaki_i8.cuh"

namespace qsgw {

struct ZmelAtomDev {
  const double* ppb;      // (nlnm, nlnm, mdim) real, column-major
  int nlnm, nc, nv, ias, ics, ims, mdim, ncore;
  double ph_re, ph_im;    // exp(-i 2 pi k . tau)
};

constexpr int ZM_T = 16;          // itp and it block
constexpr int ZM_NVMAX = 96;      // valence channels per atom handled in shared memory

__global__ void zmel_mt_kernel(double2* __restrict__ zt, int nbloch, int nm1, int nmtot, int nctot, int ntp0,
                               int nm1v, int nm2v, int nm1c, int nm2c, const double2* __restrict__ cphim,
                               int ldm, const double2* __restrict__ cphiq, int ldq,
                               const ZmelAtomDev* __restrict__ atoms, int nvmax) {
  // dynamic shared memory, sized for the largest atom:
  //   sq, sT, sm_ : (nvmax x 16) complex   cphiq block, T = ppb^T cphiq, conj(cphim) block
  //   sp          : nvmax^2 doubles        ppb valence block of one product function
  extern __shared__ double2 zm_smem[];
  double2 (*sq)[ZM_T] = reinterpret_cast<double2 (*)[ZM_T]>(zm_smem);
  double2 (*sT)[ZM_T] = reinterpret_cast<double2 (*)[ZM_T]>(zm_smem + nvmax * ZM_T);
  double2 (*sm_)[ZM_T] = reinterpret_cast<double2 (*)[ZM_T]>(zm_smem + 2 * nvmax * ZM_T);
  double* sp = reinterpret_cast<double*>(zm_smem + 3 * nvmax * ZM_T);
  const ZmelAtomDev at = atoms[blockIdx.x];
  const int itp0 = blockIdx.y * ZM_T;
  const int it0 = blockIdx.z * ZM_T;                  // index into [nm1, nm2] (0-based)
  const int tid = threadIdx.x;
  const int nv = at.nv, nc = at.nc;
  const double2 ph = make_double2(at.ph_re, at.ph_im);
  // stage cphiq(ias:ias+nv-1, itp0:itp0+15)
  for (int e = tid; e < nv * ZM_T; e += blockDim.x) {
    const int b = e % nv, j = e / nv;
    const int itp = itp0 + j;
    sq[b][j] = (itp < ntp0) ? cphiq[(at.ias - 1 + b) + static_cast<long long>(itp) * ldq] : make_double2(0.0, 0.0);
  }
  // stage conj(cphim) for valence middle states of this block
  for (int e = tid; e < nv * ZM_T; e += blockDim.x) {
    const int a = e % nv, j = e / nv;
    const int it = nm1 + it0 + j;
    double2 v = make_double2(0.0, 0.0);
    if (it0 + j < nmtot && it >= nm1v && it <= nm2v) {
      v = cphim[(at.ias - 1 + a) + static_cast<long long>(it - nm1v) * ldm];
      v.y = -v.y;
    }
    sm_[a][j] = v;
  }
  __syncthreads();
  for (int i = 0; i < at.mdim; ++i) {
    // ppb(nc+1:nc+nv, nc+1:nc+nv, i) valence block
    for (int e = tid; e < nv * nv; e += blockDim.x) {
      const int b = e % nv, a = e / nv;
      sp[e] = at.ppb[(nc + b) + static_cast<long long>(nc + a) * at.nlnm + static_cast<long long>(i) * at.nlnm * at.nlnm];
    }
    __syncthreads();
    for (int e = tid; e < nv * ZM_T; e += blockDim.x) {   // T(a, itp) (m_zmel.f90:358)
      const int a = e % nv, j = e / nv;
      double2 acc = make_double2(0.0, 0.0);
      for (int b = 0; b < nv; ++b) {
        const double w = sp[b + a * nv];
        acc.x += w * sq[b][j].x;
        acc.y += w * sq[b][j].y;
      }
      sT[a][j] = acc;
    }
    __syncthreads();
    // zmelt(ims+i-1, it, itp) for this block (valence :365, core :383)
    for (int e = tid; e < ZM_T * ZM_T; e += blockDim.x) {
      const int jt = e % ZM_T, jp = e / ZM_T;
      const int itl = it0 + jt, itp = itp0 + jp;
      if (itl >= nmtot || itp >= ntp0) continue;
      const int it = nm1 + itl;
      double2 acc = make_double2(0.0, 0.0);
      bool write = false;
      if (it >= nm1v && it <= nm2v) {
        for (int a = 0; a < nv; ++a) {
          const double2 m = sm_[a][jt], t = sT[a][jp];
          acc.x += m.x * t.x - m.y * t.y;
          acc.y += m.x * t.y + m.y * t.x;
        }
        write = true;
      } else if (it >= nm1c && it <= nm2c) {
        const int ncorec = nctot > 0 ? at.ncore : 0;
        if (it > at.ics && it <= at.ics + ncorec) {
          // sum_b ppb(nc+b, it-ics, i) cphiq(b, itp)
          const double* pc = at.ppb + static_cast<long long>(it - at.ics - 1) * at.nlnm +
                             static_cast<long long>(i) * at.nlnm * at.nlnm;
          for (int b = 0; b < nv; ++b) {
            const double w = pc[nc + b];
            acc.x += w * sq[b][jp].x;
            acc.y += w * sq[b][jp].y;
          }
          write = true;
        }
      }
      if (write) {
        const double2 o = make_double2(ph.x * acc.x - ph.y * acc.y, ph.x * acc.y + ph.y * acc.x);
        zt[(at.ims - 1 + i) + static_cast<long long>(itl) * nbloch + static_cast<long long>(itp) * nbloch * nmtot] = o;
      }
    }
    __syncthreads();
  }
}

__global__ void conj_kernel(double2* a, long long n) {
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x)
    a[e].y = -a[e].y;
}

static DevBuf g_zm_atoms;

// ---- interstitial plane-wave part (m_zmel.f90:418-535)
// M(c, g) = ggg(sg * vg(g) - vc(c) - nadd) or 0 when that vector is not in the ggg table.
__global__ void ipw_gmat_kernel(double2* __restrict__ M, int ncgp, int ng, const int* __restrict__ vc,
                                const int* __restrict__ vg, int sg, int ax, int ay, int az,
                                const int* __restrict__ box, int x0, int nx, int y0, int ny, int z0, int nz,
                                const double2* __restrict__ ggg) {
  const long long tot = static_cast<long long>(ncgp) * ng;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(e % ncgp), g = static_cast<int>(e / ncgp);
    const int x = sg * vg[3 * g] - vc[3 * c] - ax - x0;
    const int y = sg * vg[3 * g + 1] - vc[3 * c + 1] - ay - y0;
    const int z = sg * vg[3 * g + 2] - vc[3 * c + 2] - az - z0;
    double2 v = make_double2(0.0, 0.0);
    if (x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz) {
      const int k = box[x + nx * (y + ny * z)];
      if (k >= 0) v = ggg[k];
    }
    M[e] = v;
  }
}

// Tg[k + nidx b] = T[cidx[k] + ldt b]
__global__ void gather_rows_kernel(double2* __restrict__ Tg, const double2* __restrict__ T, int ldt,
                                   const int* __restrict__ cidx, long long nidx, int nbatch) {
  const long long tot = nidx * nbatch;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long k = e % nidx, b = e / nidx;
    Tg[e] = T[cidx[k] + static_cast<long long>(ldt) * b];
  }
}

// zmelt(row0 + igc, it0 + it, itp) = phase(igc) * Z(igc, it, itp)
__global__ void ipw_scatter_kernel(double2* __restrict__ zt, int ldz, int row0, int it0, int nmtot,
                                   const double2* __restrict__ Z, int ngc, int nmv, int ntp0,
                                   const double2* __restrict__ phase) {
  const long long tot = static_cast<long long>(ngc) * nmv * ntp0;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int igc = static_cast<int>(e % ngc);
    const long long r = e / ngc;
    const int it = static_cast<int>(r % nmv), itp = static_cast<int>(r / nmv);
    const double2 p = phase[igc], z = Z[e];
    zt[row0 + igc + static_cast<long long>(ldz) * (it0 + it + static_cast<long long>(nmtot) * itp)] =
        make_double2(p.x * z.x - p.y * z.y, p.x * z.y + p.y * z.x);
  }
}

// Inverse table of a list of integer 3-vectors over their bounding box (-1 = absent).
struct Box {
  int x0 = 0, nx = 0, y0 = 0, ny = 0, z0 = 0, nz = 0;
  std::vector<int> map;
  void build(const int* v, int n) {
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], v[3 * i + d]); hi[d] = std::max(hi[d], v[3 * i + d]); }
    x0 = lo[0]; y0 = lo[1]; z0 = lo[2];
    nx = hi[0] - lo[0] + 1; ny = hi[1] - lo[1] + 1; nz = hi[2] - lo[2] + 1;
    map.assign(static_cast<size_t>(nx) * ny * nz, -1);
    for (int i = 0; i < n; ++i) map[(v[3 * i] - x0) + static_cast<size_t>(nx) * ((v[3 * i + 1] - y0) + static_cast<size_t>(ny) * (v[3 * i + 2] - z0))] = i;
  }
  int find(int x, int y, int z) const {
    x -= x0; y -= y0; z -= z0;
    if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz) return -1;
    return map[x + static_cast<size_t>(nx) * (y + static_cast<size_t>(ny) * z)];
  }
};

static DevBuf g_ipw_tab, g_ipw_m, g_ipw_t, g_ipw_tg, g_ipw_z;

static int ipw_grid(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 16LL * ctx().sm_count)));
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_zmel_mt_d(double* zmelt_d, int nbloch, int nm1, int nm2, int nctot, int ntp0,
                              const double* cphim_d, int ldm, const double* cphiq_d, int ldq, int natom,
                              const qsgw_zmel_atom* atoms) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(zmelt_d && cphiq_d && atoms && natom >= 1, "zmel_mt: null pointer / natom=%d", natom);
  QSGW_ARG(nm2 >= nm1 && ntp0 >= 1 && nbloch >= 1, "zmel_mt: nm %d..%d ntp0=%d nbloch=%d", nm1, nm2, ntp0, nbloch);
  int nm1c, nm2c, nm1v, nm2v;                                      // m_zmel.f90:233-248
  if (nm1 > nctot) { nm1c = 0; nm2c = -1; nm1v = nm1; nm2v = nm2; }
  else if (nm2 > nctot) { nm1c = nm1; nm2c = nctot; nm1v = nctot + 1; nm2v = nm2; }
  else { nm1c = nm1; nm2c = nm2; nm1v = 0; nm2v = -1; }
  QSGW_ARG(nm2v < nm1v || cphim_d, "zmel_mt: cphim required for valence middle states");
  std::vector<ZmelAtomDev> h(natom);
  int nvmax = 1;
  for (int ia = 0; ia < natom; ++ia) {
    const qsgw_zmel_atom& a = atoms[ia];
    QSGW_ARG(a.nv >= 1 && a.nv <= ZM_NVMAX && a.nc >= 0 && a.nc + a.nv <= a.nlnm && a.ppb_d,
             "zmel_mt: atom %d nv=%d nc=%d nlnm=%d (nv <= %d)", ia, a.nv, a.nc, a.nlnm, ZM_NVMAX);
    QSGW_ARG(a.ims >= 1 && a.ims - 1 + a.mdim <= nbloch && a.ias >= 1 && a.ias - 1 + a.nv <= ldq,
             "zmel_mt: atom %d offsets outside zmelt/cphi", ia);
    QSGW_ARG(a.ncore <= a.nc, "zmel_mt: atom %d ncore=%d > nc=%d", ia, a.ncore, a.nc);
    h[ia] = ZmelAtomDev{a.ppb_d, a.nlnm, a.nc, a.nv, a.ias, a.ics, a.ims, a.mdim, a.ncore, a.phase_re, a.phase_im};
    nvmax = std::max(nvmax, a.nv);
  }
  const size_t smem = static_cast<size_t>(3 * nvmax * ZM_T) * sizeof(double2) + static_cast<size_t>(nvmax) * nvmax * sizeof(double);
  static uint64_t attr = 0;                       // one bit per device
  rc = smem_limit_once(reinterpret_cast<const void*>(zmel_mt_kernel),
                       static_cast<int>(3 * ZM_NVMAX * ZM_T * sizeof(double2) + ZM_NVMAX * ZM_NVMAX * sizeof(double)),
                       attr);
  if (rc) return rc;
  cudaStream_t s = ctx().stream;
  rc = g_zm_atoms.ensure(natom * sizeof(ZmelAtomDev));
  if (rc) return rc;
  QSGW_CUDA(cudaMemcpyAsync(g_zm_atoms.p, h.data(), natom * sizeof(ZmelAtomDev), cudaMemcpyHostToDevice, s));
  const int nmtot = nm2 - nm1 + 1;
  dim3 grid(natom, (ntp0 + ZM_T - 1) / ZM_T, (nmtot + ZM_T - 1) / ZM_T);
  zmel_mt_kernel<<<grid, 128, smem, s>>>(reinterpret_cast<double2*>(zmelt_d), nbloch, nm1, nmtot, nctot, ntp0, nm1v,
                                         nm2v, nm1c, nm2c, reinterpret_cast<const double2*>(cphim_d), ldm,
                                         reinterpret_cast<const double2*>(cphiq_d), ldq, g_zm_atoms.as<ZmelAtomDev>(),
                                         nvmax);
  count_launch();
  QSGW_LAUNCH_CHECK("zmel_mt_kernel");
  return QSGW_OK;
}

extern "C" int qsgw_zmel_m2e_d(double* zmel_d, const double* zmelt_d, int ngb, int nbb, int nmtot, int nqtot,
                               const double* m2e_d, int is_m_basis, int zmelconjg) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(zmel_d && zmelt_d && (is_m_basis || m2e_d), "zmel_m2e: null pointer");
  QSGW_ARG(ngb >= 1 && nbb >= 1 && nmtot >= 0 && nqtot >= 0, "zmel_m2e: bad sizes");
  cudaStream_t s = ctx().stream;
  const long long ncol = static_cast<long long>(nmtot) * nqtot;
  if (ncol == 0) return QSGW_OK;
  if (is_m_basis) {                                                // copy (m_zmel.f90:549-554)
    QSGW_ARG(nbb == ngb, "zmel_m2e: M basis keeps nbb == ngb");
    QSGW_CUDA(cudaMemcpyAsync(zmel_d, zmelt_d, static_cast<size_t>(ngb) * ncol * 16, cudaMemcpyDeviceToDevice, s));
  } else if (ctx().prec_mode == QSGW_PREC_SPLIT_I8) {              // the same product on the int8 path
    QSGW_ARG(ncol < (1LL << 31), "zmel_m2e: %lld columns", ncol);
    rc = zgemm_ch_i8(reinterpret_cast<double2*>(zmel_d), nbb, nbb, static_cast<int>(ncol), ngb,
                     reinterpret_cast<const double2*>(m2e_d), ngb, reinterpret_cast<const double2*>(zmelt_d), ngb,
                     ctx().nslices > 0 ? ctx().nslices : 4, s);
    if (rc) return rc;
  } else {                                                         // zmel = m2e^H zmelt (:559-560)
    rc = zgemm_f64(2, 0, nbb, static_cast<int>(ncol), ngb, make_double2(1, 0), reinterpret_cast<const double2*>(m2e_d),
                   ngb, 0, reinterpret_cast<const double2*>(zmelt_d), ngb, 0, make_double2(0, 0),
                   reinterpret_cast<double2*>(zmel_d), nbb, 0, 1, s);
    if (rc) return rc;
  }
  if (zmelconjg) {                                                 // :590-594
    const long long n = static_cast<long long>(nbb) * ncol;
    conj_kernel<<<static_cast<int>(std::min<long long>((n + 255) / 256, 4096)), 256, 0, s>>>(
        reinterpret_cast<double2*>(zmel_d), n);
    count_launch();
    QSGW_LAUNCH_CHECK("conj_kernel");
  }
  return QSGW_OK;
}

extern "C" int qsgw_zmel_ipw_d(const qsgw_zmel_ipw_args* a) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(a, "zmel_ipw: null argument block");
  const int ngc = a->ngc, ngp1 = a->ngp1, ngp2 = a->ngp2, ngcgp = a->ngcgp, nggg = a->nggg, ntp0 = a->ntp0;
  const int nmv = a->nm2v - a->nm1v + 1, nmtot = a->nm2 - a->nm1 + 1;
  if (ngc == 0 || nmv <= 0) return QSGW_OK;                        // :418 guard
  QSGW_ARG(ngc > 0 && ngp1 >= 1 && ngp2 >= 1 && ngcgp >= 1 && nggg >= 1 && ntp0 >= 1 && nmtot >= 1,
           "zmel_ipw: sizes ngc=%d ngp1=%d ngp2=%d ngcgp=%d nggg=%d ntp0=%d", ngc, ngp1, ngp2, ngcgp, nggg, ntp0);
  QSGW_ARG(a->nm1v >= a->nm1 && a->nm2v <= a->nm2, "zmel_ipw: valence %d..%d outside %d..%d", a->nm1v, a->nm2v,
           a->nm1, a->nm2);
  QSGW_ARG(a->ngvecpB1 && a->ngvecpB2 && a->ngveccR && a->nvgcgp2 && a->nvggg && a->ggg && a->phase && a->geigq_d &&
               a->dgeigqk_d && a->zmelt_d,
           "zmel_ipw: null pointer");
  QSGW_ARG(a->row0 >= 0 && a->ldz >= a->row0 + ngc && a->ldgq >= ngp1 && a->ldgk >= ngp2,
           "zmel_ipw: leading dimensions ldz=%d (row0=%d) ldgq=%d ldgk=%d", a->ldz, a->row0, a->ldgq, a->ldgk);
  Box bg, bc;
  bg.build(a->nvggg, nggg);
  bc.build(a->nvgcgp2, ngcgp);
  // branch of the reference (:439): G1 integral first when the middle states outnumber the targets
  const bool g1first = nmv > ntp0;
  const int ngA = g1first ? ngp1 : ngp2;                 // plane waves contracted with the ggg matrix
  const int ngB = g1first ? ngp2 : ngp1;                 // plane waves of the gathered contraction
  const int* vA = g1first ? a->ngvecpB1 : a->ngvecpB2;
  const int* vB = g1first ? a->ngvecpB2 : a->ngvecpB1;
  const int ncolT = g1first ? ntp0 : nmv, nbat = g1first ? ntp0 : nmv;
  // composite index of Gc + G2 (G1 first, :464-466) or Gc - G1 (G2 first, :507-509), validated here
  std::vector<int> cidx(static_cast<size_t>(ngc) * ngB);
  for (int g = 0; g < ngB; ++g)
    for (int c = 0; c < ngc; ++c) {
      const int sg = g1first ? 1 : -1;
      const int k = bc.find(a->ngveccR[3 * c] + sg * vB[3 * g], a->ngveccR[3 * c + 1] + sg * vB[3 * g + 1],
                            a->ngveccR[3 * c + 2] + sg * vB[3 * g + 2]);
      QSGW_ARG(k >= 0, "zmel_ipw: composite vector of Gc %d and plane wave %d is not in nvgcgp2", c + 1, g + 1);
      cidx[c + static_cast<size_t>(ngc) * g] = k;
    }
  cudaStream_t s = ctx().stream;
  // device tables: box map, cidx, vectors (ints); ggg, phase (complex)
  const size_t nbox = bg.map.size(), ni = nbox + cidx.size() + 3 * static_cast<size_t>(ngcgp) + 3 * static_cast<size_t>(ngA);
  const size_t ioff_c = nbox, ioff_vc = ioff_c + cidx.size(), ioff_va = ioff_vc + 3 * static_cast<size_t>(ngcgp);
  const size_t ibytes = ((ni * sizeof(int) + 15) / 16) * 16;
  rc = g_ipw_tab.ensure(ibytes + (static_cast<size_t>(nggg) + ngc) * sizeof(double2));
  if (rc) return rc;
  int* di = g_ipw_tab.as<int>();
  double2* dz = reinterpret_cast<double2*>(g_ipw_tab.as<char>() + ibytes);
  QSGW_CUDA(cudaMemcpyAsync(di, bg.map.data(), nbox * sizeof(int), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(di + ioff_c, cidx.data(), cidx.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(di + ioff_vc, a->nvgcgp2, 3 * static_cast<size_t>(ngcgp) * sizeof(int), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(di + ioff_va, vA, 3 * static_cast<size_t>(ngA) * sizeof(int), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(dz, a->ggg, static_cast<size_t>(nggg) * sizeof(double2), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(dz + nggg, a->phase, static_cast<size_t>(ngc) * sizeof(double2), cudaMemcpyHostToDevice, s));
  // scratch: M (ngcgp x ngA), T (ngcgp x ncolT), Tg (ngc x ngB x nbat), Z (ngc x nmv x ntp0)
  if ((rc = g_ipw_m.ensure(static_cast<size_t>(ngcgp) * ngA * sizeof(double2)))) return rc;
  if ((rc = g_ipw_t.ensure(static_cast<size_t>(ngcgp) * ncolT * sizeof(double2)))) return rc;
  if ((rc = g_ipw_tg.ensure(static_cast<size_t>(ngc) * ngB * nbat * sizeof(double2)))) return rc;
  if ((rc = g_ipw_z.ensure(static_cast<size_t>(ngc) * nmv * ntp0 * sizeof(double2)))) return rc;
  double2 *M = g_ipw_m.as<double2>(), *T = g_ipw_t.as<double2>(), *Tg = g_ipw_tg.as<double2>(),
          *Z = g_ipw_z.as<double2>();
  const double2* geigq = reinterpret_cast<const double2*>(a->geigq_d);
  const double2* dgk = reinterpret_cast<const double2*>(a->dgeigqk_d);
  const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
  ipw_gmat_kernel<<<ipw_grid(static_cast<long long>(ngcgp) * ngA), 256, 0, s>>>(
      M, ngcgp, ngA, di + ioff_vc, di + ioff_va, g1first ? 1 : -1, a->nadd[0], a->nadd[1], a->nadd[2], di, bg.x0, bg.nx,
      bg.y0, bg.ny, bg.z0, bg.nz, dz);
  count_launch();
  QSGW_LAUNCH_CHECK("ipw_gmat_kernel");
  // T = M * geigq (:458) or M * dgeigqk (:501)
  rc = zgemm_f64(0, 0, ngcgp, ncolT, ngA, one, M, ngcgp, 0, g1first ? geigq : dgk, g1first ? a->ldgq : a->ldgk, 0,
                 zero, T, ngcgp, 0, 1, s);
  if (rc) return rc;
  const long long nidx = static_cast<long long>(ngc) * ngB;
  gather_rows_kernel<<<ipw_grid(nidx * nbat), 256, 0, s>>>(Tg, T, ngcgp, di + ioff_c, nidx, nbat);
  count_launch();
  QSGW_LAUNCH_CHECK("gather_rows_kernel");
  if (g1first)   // Z(:, :, itp) = Tg(:, :, itp) * dgeigqk  (:470-479), batched over itp
    rc = zgemm_f64(0, 0, ngc, nmv, ngp2, one, Tg, ngc, nidx, dgk, a->ldgk, 0, zero, Z, ngc,
                   static_cast<long long>(ngc) * nmv, ntp0, s);
  else           // Z(:, it, :) = Tg(:, :, it) * geigq  (:513-521), batched over it
    rc = zgemm_f64(0, 0, ngc, ntp0, ngp1, one, Tg, ngc, nidx, geigq, a->ldgq, 0, zero, Z,
                   static_cast<long long>(ngc) * nmv, ngc, nmv, s);
  if (rc) return rc;
  ipw_scatter_kernel<<<ipw_grid(static_cast<long long>(ngc) * nmv * ntp0), 256, 0, s>>>(
      reinterpret_cast<double2*>(a->zmelt_d), a->ldz, a->row0, a->nm1v - a->nm1, nmtot, Z, ngc, nmv, ntp0, dz + nggg);
  count_launch();
  QSGW_LAUNCH_CHECK("ipw_scatter_kernel");
  QSGW_CUDA(cudaStreamSynchronize(s));                                // host tables above die on return
  return QSGW_OK;
}
