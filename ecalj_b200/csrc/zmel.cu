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
  static bool attr = false;
  if (!attr) {
    QSGW_CUDA(cudaFuncSetAttribute(zmel_mt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(3 * ZM_NVMAX * ZM_T * sizeof(double2) + ZM_NVMAX * ZM_NVMAX * sizeof(double))));
    attr = true;
  }
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
