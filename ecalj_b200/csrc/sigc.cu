// Correlation self-energy of one task: get_correlation_block of
// sxcf_scz_correlation (m_sxcf_gemm.f90:407-612).
//
//   1. wgtim(0:niw, it, itp) on the GPU in FP64 (:432-458).
//   2. Pole entries (it, itp) -> (ixs, wgt3) on the host, in the reference's
//      loop order (:511-552, wfacx2/weavx2 of wfacx.f90:19-49).
//   3. ONE launch of the segmented DMMA GEMM:
//        czmelwc(:, c) = sum_{iw=0..niw} Wc_i(iw)^H (wgtim(iw, c) z_c)
//                      + sum_{i=0..2}  Wsym(ixs_c-1+i)^H (wgt3_i(c) z_c)
//      Columns are grouped by ixs so every 64-column tile shares one list of
//      W matrices; every column is written once (no scatter races).
//   4. zsec += czmelwc^H zmel (:599) with split-K, then Im zsec_ii <= 0 (:601-607).
#include <cmath>
#include <map>
#include <set>
#include <string>
#include <algorithm>
#include <vector>
#include "zgemm_f64.cuh"
#include "split_f16.cuh"
#include "ozaki_i8.cuh"
#include "autotune.cuh"
#include "hoststage.cuh"

namespace qsgw {

static constexpr double kPi = 3.14159265358979323846264338327950288;

__global__ void wgtim_kernel(double* __restrict__ wg, int niw, int ns1, int nm, int ntqxx, int nctot,
                             const double* __restrict__ omega, const double* __restrict__ ekc,
                             double esmr, double wkkr, double ua, const double* __restrict__ x,
                             const double* __restrict__ wt, const double* __restrict__ expa) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nm * ntqxx) return;
  const int itl = c % nm, itp = c / nm;
  const int it = ns1 + itl;
  const double pi = kPi;
  const double we = 0.5 * (omega[itp] - ekc[it - 1]);
  const double aw = fabs(ua * we), aw2 = aw * aw;
  const double sig2 = 2.0 * (0.5 * esmr) * (0.5 * esmr);
  const double sgn = signbit(we) ? -1.0 : 1.0;
  double* out = wg + static_cast<long long>(c) * (niw + 1);
  if (it <= nctot) {
    double s0 = 0.0;
    for (int i = 0; i < niw; ++i) {
      const double cons = 1.0 / (we * we * x[i] * x[i] + (1.0 - x[i]) * (1.0 - x[i]));
      const double w = we * cons * wt[i] * (-1.0 / pi);
      out[1 + i] = wkkr * w;
      s0 += w * expa[i];
    }
    double w0 = 0.0;
    if (fabs(we) < 2.0 / ua) w0 = -s0 - 0.5 * sgn * exp(we * we * ua * ua) * erfc(ua * fabs(we));
    out[0] = wkkr * w0;
  } else {
    double s0 = 0.0;
    for (int i = 0; i < niw; ++i) {
      const double omd = 1.0 / x[i] - 1.0;
      const double omd2w = omd * omd + we * we;
      const double r = omd2w / sig2;
      double cons;
      if (r > 5e-3) {
        cons = (1.0 - exp(-r)) / omd2w;
      } else {
        cons = 1.0 / sig2 - omd2w / (sig2 * sig2) / 2.0 + omd2w * omd2w / (sig2 * sig2 * sig2) / 6.0 -
               omd2w * omd2w * omd2w / (sig2 * sig2 * sig2 * sig2) / 24.0 +
               omd2w * omd2w * omd2w * omd2w / (sig2 * sig2 * sig2 * sig2 * sig2) / 120.0 -
               omd2w * omd2w * omd2w * omd2w * omd2w / (sig2 * sig2 * sig2 * sig2 * sig2 * sig2) / 720.0;
      }
      out[1 + i] = wkkr * (-we * cons * wt[i] / (x[i] * x[i]) / pi);
      s0 += cons * expa[i] * wt[i] / (x[i] * x[i]);
    }
    const double w0 = we * s0 / pi + sgn * 0.5 * exp(aw2) * (erfc(sqrt(aw2 + we * we / sig2)) - erfc(aw));
    out[0] = wkkr * w0;
  }
}

// full Hermitian (ld = n) from a packed upper triangle, column order (j, i <= j) (:327-358, :468-474)
__global__ void unpack_upper_kernel(double2* __restrict__ w, const double2* __restrict__ up, int n,
                                    int nmat) {
  const long long np = static_cast<long long>(n) * (n + 1) / 2;
  const long long tot = static_cast<long long>(n) * n * nmat;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n);
    const long long r = e / n;
    const int j = static_cast<int>(r % n);
    const long long m = r / n;
    double2 v;
    if (i < j) {
      v = up[m * np + static_cast<long long>(j) * (j + 1) / 2 + i];
    } else if (i == j) {
      // wc(i,j) = up then wc(j,i) = conjg(up) in the same iteration: the
      // diagonal ends up conjugated (m_sxcf_gemm.f90:470-473)
      const double2 u = up[m * np + static_cast<long long>(j) * (j + 1) / 2 + i];
      v = make_double2(u.x, -u.y);
    } else {
      const double2 u = up[m * np + static_cast<long long>(i) * (i + 1) / 2 + j];
      v = make_double2(u.x, -u.y);
    }
    w[e] = v;
  }
}

// (W + W^H)/2 of selected records (:573)
// out[q](i, j) = (W_recs[q](i, j) + conj(W_recs[q](j, i))) / 2: block (32, 8) per 32 x 32 tile
// (grid x, y) of record q (grid z); the transposed tile goes through shared memory so both
// reads are coalesced
__global__ void hermitize_kernel(double2* __restrict__ out, const double2* __restrict__ in,
                                 const int* __restrict__ recs, int n, long long ld, int nrec) {
  __shared__ double2 tile[32][33];
  const int q = blockIdx.z;
  const double2* W = in + static_cast<long long>(recs[q]) * ld * ld;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int b = threadIdx.y; b < 32; b += 8) {          // tile[x][b] = W(j0 + x, i0 + b)
    const int jj = j0 + threadIdx.x, ii = i0 + b;
    if (jj < n && ii < n) tile[threadIdx.x][b] = W[jj + static_cast<long long>(ii) * ld];
  }
  __syncthreads();
  for (int b = threadIdx.y; b < 32; b += 8) {
    const int i = i0 + threadIdx.x, j = j0 + b;
    if (i < n && j < n) {
      const double2 a = W[i + static_cast<long long>(j) * ld], t = tile[b][threadIdx.x];   // t = W(j, i)
      out[static_cast<long long>(q) * ld * ld + i + static_cast<long long>(j) * ld] =
          make_double2(0.5 * (a.x + t.x), 0.5 * (a.y - t.y));
    }
  }
}

__global__ void clamp_diag_kernel(double2* zsec, int ntqxx, int ntq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ntqxx) {
    double2 v = zsec[i + static_cast<long long>(i) * ntq];
    if (v.y > 0.0) v.y = 0.0;
    zsec[i + static_cast<long long>(i) * ntq] = v;
  }
}

// ---- host restatement of the pole weights (wfacx.f90:19-49, m_sxcf_gemm.f90:511-552)
static double wfacx2_h(double e1, double e2, double ek, double esmr) {
  const double el = std::min(e1, e2), eh = std::max(e1, e2);
  if (eh - el < 1e-6) return 0.0;
  if (esmr == 0.0) return (el <= ek && ek < eh) ? 1.0 : 0.0;
  return 0.5 * std::erfc(-(eh - ek) / std::sqrt(2.0) / esmr) - 0.5 * std::erfc(-(el - ek) / std::sqrt(2.0) / esmr);
}
static double weavx2_h(double e1, double e2, double ek, double esmr) {
  const double el = std::min(e1, e2), eh = std::max(e1, e2);
  const double wtt = 0.5 * std::erfc(-(eh - ek) / std::sqrt(2.0) / esmr) -
                     0.5 * std::erfc(-(el - ek) / std::sqrt(2.0) / esmr);
  const double sig2 = 2.0 * esmr * esmr;
  const double pi = 3.1415926535897932;
  return ek + esmr / std::sqrt(2.0 * pi) * (-std::exp(-(eh - ek) * (eh - ek) / sig2) +
                                            std::exp(-(el - ek) * (el - ek) / sig2)) / wtt;
}
static void inverse33_h(const double m[3][3], double inv[3][3]) {
  // columns of the cofactor matrix (m_sxcf_gemm.f90:658-668), then transpose / det
  double c[3][3];
  auto cross = [](const double* a, const double* b, double* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
  };
  double col[3][3];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) col[j][i] = m[i][j];
  cross(col[1], col[2], c[0]);
  cross(col[2], col[0], c[1]);
  cross(col[0], col[1], c[2]);
  const double det = col[0][0] * c[0][0] + col[0][1] * c[0][1] + col[0][2] * c[0][2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) inv[i][j] = c[i][j] / det;   // inv = transpose(cof) / det
}

struct PoleEntry { int col; int ixs; double w3[3]; };

static int pole_table_h(const qsgw_sxcf_args& a, std::vector<PoleEntry>& out) {
  const int nm = a.ns2 - a.ns1 + 1;
  int nt0p = 0, nt0m = 0;
  for (int i = 0; i < a.nekc; ++i) {
    if (a.ekc[i] < a.ef + 10.0 * a.esmr) ++nt0p;
    if (a.ekc[i] < a.ef - 10.0 * a.esmr) ++nt0m;
  }
  for (int itp = 1; itp <= a.ntqxx; ++itp) {
    const double omg = a.omega[itp - 1];
    const int itini = omg >= a.ef ? std::max(a.ns1, nt0m + 1) : a.ns1;
    const int itend = omg >= a.ef ? a.ns2r : std::min(nt0p, a.ns2r);
    for (int it = itini; it <= itend; ++it) {
      double wf = wfacx2_h(omg, a.ef, a.ekc[it - 1], it <= a.nctot ? 0.0 : a.esmr);
      if (wf < 1e-8) continue;
      wf = wf * a.wkkr * (std::signbit(omg - a.ef) ? -1.0 : 1.0);
      const double we = 0.5 * std::fabs(omg - weavx2_h(omg, a.ef, a.ekc[it - 1], a.esmr));
      int ixs = 0;
      for (int i = 1; i <= a.nw; ++i)
        if (a.freq_r[i] > we) { ixs = i; break; }
      if (ixs == 0 || ixs + 1 > a.nw) {
        set_error("sxcf: pole frequency %g outside the real-axis mesh (freq_r(nw)=%g)", we, a.freq_r[a.nw]);
        return QSGW_ERR_ARG;
      }
      double am[3][3], inv[3][3];
      for (int r = 0; r < 3; ++r) {
        const double xi = a.freq_r[ixs - 1 + r];
        am[r][0] = 1.0; am[r][1] = xi * xi; am[r][2] = xi * xi * xi * xi;
      }
      inverse33_h(am, inv);
      const double v[3] = {1.0, we * we, we * we * we * we};
      PoleEntry e;
      e.col = (it - a.ns1) + nm * (itp - 1);
      e.ixs = ixs;
      for (int j = 0; j < 3; ++j) e.w3[j] = wf * (v[0] * inv[0][j] + v[1] * inv[1][j] + v[2] * inv[2][j]);
      out.push_back(e);
    }
  }
  return QSGW_OK;
}

static DevBuf g_sc_wg, g_sc_w3, g_sc_cz, g_sc_wi, g_sc_wr, g_sc_tabs, g_sc_recs, g_sc_tmp;
static DevBuf g_sc_host_zs;
static DevBuf g_sc_trial;                // Sigma_c of the slice-count trials
// zmel, W(i omega), W(omega) records of the host-pointer calls: twelve slots (about 0.6 GB each
// at ngb = 600), so the inputs of the next tasks keep the copy engine busy through a long kernel
static HostRing g_sc_ring(12);

static int grid_for(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 16LL * ctx().sm_count)));
}

static int sxcf_check(const qsgw_sxcf_args* a) {
  QSGW_ARG(a, "sxcf: null args");
  QSGW_ARG(a->ngb >= 1 && a->ntqxx >= 0 && a->ntq >= a->ntqxx && a->niw >= 1 && a->nw >= 2,
           "sxcf: ngb=%d ntqxx=%d ntq=%d niw=%d nw=%d", a->ngb, a->ntqxx, a->ntq, a->niw, a->nw);
  QSGW_ARG(a->keepwv || a->nblochpmx >= a->ngb, "sxcf: nblochpmx=%d < ngb", a->nblochpmx);
  QSGW_ARG(a->ns1 >= 1 && a->ns2 <= a->nekc && a->ns2r <= a->ns2, "sxcf: middle states %d..%d (pole ..%d) vs nekc=%d",
           a->ns1, a->ns2, a->ns2r, a->nekc);
  QSGW_ARG(a->nwxi >= 0 && a->nwx <= a->nw, "sxcf: real window %d..%d, nw=%d", a->nwxi, a->nwx, a->nw);
  QSGW_ARG(a->omega && a->ekc && a->freqx && a->wwx && a->expa && a->freq_r, "sxcf: null table");
  QSGW_ARG(a->zmel && a->wc_imag && a->wc_real && a->zsec, "sxcf: null array");
  QSGW_ARG(a->ua > 0.0 && a->esmr > 0.0, "sxcf: ua=%g esmr=%g must be positive", a->ua, a->esmr);
  return QSGW_OK;
}

// ---- one task, split into the steps a batch of tasks interleaves
// host plan: pole entries, the real-axis records they read, and the column tiles.  Columns are
// sorted by their pole bin ixs (0 = no pole) and cut into tiles of the kernel's column width; a
// tile's segments are the niw+1 imaginary slots and the union of its columns' real-axis bins.
// scale_bin[r][col] = the column's pole weight on record r (zero when the column has no pole
// there), so mixing bins in a tile adds no padding columns.
struct SxcfPlan {
  int nm = 0;
  long long ncol = 0;
  std::vector<int> recs;                 // real-axis bins used, in record order
  std::vector<double> scale_bin;         // [nrec][ncol]
  std::vector<int> tile_cols, tile_group, gseg_off, gnseg, seg_slot;   // slot niw+1+r = record r
};

static int sxcf_plan(const qsgw_sxcf_args& a, int tilew, SxcfPlan& pl) {
  const int niw = a.niw;
  pl.nm = a.ns2 - a.ns1 + 1;
  pl.ncol = static_cast<long long>(pl.nm) * a.ntqxx;
  const long long ncol = pl.ncol;
  std::vector<PoleEntry> poles;
  int rc = pole_table_h(a, poles);
  if (rc) return rc;
  // bins needed by the pole entries, restricted to [nwxi, nwx] (:557)
  std::map<int, int> bin_slot;
  for (const auto& e : poles)
    for (int i = 0; i < 3; ++i) {
      const int b = e.ixs - 1 + i;
      if (b >= a.nwxi && b <= a.nwx && !bin_slot.count(b)) bin_slot.emplace(b, 0);
    }
  pl.recs.clear();
  for (auto& kv : bin_slot) { kv.second = static_cast<int>(pl.recs.size()); pl.recs.push_back(kv.first); }
  const int nrec = static_cast<int>(pl.recs.size());
  std::vector<int> key(ncol, 0);
  for (const auto& e : poles) key[e.col] = e.ixs;
  pl.scale_bin.assign(static_cast<size_t>(std::max(nrec, 1)) * ncol, 0.0);
  for (const auto& e : poles)
    for (int i = 0; i < 3; ++i) {
      auto it = bin_slot.find(e.ixs - 1 + i);
      if (it != bin_slot.end()) pl.scale_bin[static_cast<size_t>(it->second) * ncol + e.col] = e.w3[i];
    }
  std::vector<int> order(ncol);
  for (long long c = 0; c < ncol; ++c) order[c] = static_cast<int>(c);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key[x] < key[y]; });
  pl.tile_cols.clear(); pl.tile_group.clear(); pl.gseg_off.clear(); pl.gnseg.clear(); pl.seg_slot.clear();
  int gidx = 0;
  for (long long t0 = 0; t0 < ncol; t0 += tilew) {
    const long long t1 = std::min<long long>(ncol, t0 + tilew);
    pl.gseg_off.push_back(static_cast<int>(pl.seg_slot.size()));
    for (int sgi = 0; sgi <= niw; ++sgi) pl.seg_slot.push_back(sgi);
    std::set<int> rset;                          // records used by the tile's columns
    for (long long j = t0; j < t1; ++j) {
      const int k = key[order[j]];
      if (k <= 0) continue;
      for (int i = 0; i < 3; ++i) {
        auto it = bin_slot.find(k - 1 + i);
        if (it != bin_slot.end()) rset.insert(it->second);
      }
    }
    for (int r : rset) pl.seg_slot.push_back(niw + 1 + r);
    pl.gnseg.push_back(static_cast<int>(pl.seg_slot.size()) - pl.gseg_off.back());
    pl.tile_group.push_back(gidx++);
    for (int j = 0; j < tilew; ++j) pl.tile_cols.push_back(t0 + j < t1 ? order[t0 + j] : -1);
  }
  return QSGW_OK;
}

// Per-task device buffers: the imaginary-axis weights, the pole weights and czmelwc live until the
// contraction and the final product have run; the W operands (unpacked / hermitised records) only
// until the contraction has read them (the int8 batch slices them at once).
struct SxcfBufs {
  DevBuf *wg, *w3, *cz, *wi, *wr;
};

// device side of the plan: wgtim (:432-458), the W operands, the pole weights; fills sa (the
// segments point into the task's buffers) with out = czmelwc
static int sxcf_bind(const qsgw_sxcf_args& a, SxcfPlan& pl, const SxcfBufs& b, SigcSplitArgs& sa) {
  cudaStream_t s = ctx().stream;
  const int ngb = a.ngb, niw = a.niw;
  const long long ncol = pl.ncol;
  // ---- 1. imaginary-axis weights on the GPU
  int rc = g_sc_tabs.ensure((4 * niw + a.ntq + a.nekc + 8) * sizeof(double));
  if (rc) return rc;
  double* dt = g_sc_tabs.as<double>();
  double *d_x = dt, *d_wt = dt + niw, *d_ex = dt + 2 * niw, *d_om = dt + 3 * niw, *d_ekc = d_om + a.ntq;
  if ((rc = h2d(d_x, a.freqx, niw * sizeof(double), s))) return rc;
  if ((rc = h2d(d_wt, a.wwx, niw * sizeof(double), s))) return rc;
  if ((rc = h2d(d_ex, a.expa, niw * sizeof(double), s))) return rc;
  if ((rc = h2d(d_om, a.omega, a.ntq * sizeof(double), s))) return rc;
  if ((rc = h2d(d_ekc, a.ekc, a.nekc * sizeof(double), s))) return rc;
  if ((rc = b.wg->ensure(ncol * (niw + 1) * sizeof(double)))) return rc;
  wgtim_kernel<<<static_cast<int>((ncol + 127) / 128), 128, 0, s>>>(
      b.wg->as<double>(), niw, a.ns1, pl.nm, a.ntqxx, a.nctot, d_om, d_ekc, a.esmr, a.wkkr, a.ua, d_x, d_wt, d_ex);
  count_launch();
  QSGW_LAUNCH_CHECK("wgtim_kernel");
  // ---- W operands
  const long long ldw = a.keepwv ? ngb : a.nblochpmx;
  const long long wsz = ldw * ldw;
  const double2* wi = reinterpret_cast<const double2*>(a.wc_imag);
  const double2* wr_src = reinterpret_cast<const double2*>(a.wc_real);
  if (a.keepwv) {
    if ((rc = b.wi->ensure(wsz * (niw + 1) * sizeof(double2)))) return rc;
    unpack_upper_kernel<<<grid_for(wsz * (niw + 1)), 256, 0, s>>>(b.wi->as<double2>(), wi, ngb, niw + 1);
    count_launch();
    QSGW_LAUNCH_CHECK("unpack_upper_kernel");
    wi = b.wi->as<double2>();
  }
  const int nrec = static_cast<int>(pl.recs.size());
  const double2* wr = nullptr;
  if (nrec > 0) {
    if ((rc = b.wr->ensure(wsz * nrec * sizeof(double2)))) return rc;
    if (a.keepwv) {
      // packed records are already (W+W^H)/2; unpack only the used ones
      const long long np = static_cast<long long>(ngb) * (ngb + 1) / 2;
      for (int q = 0; q < nrec; ++q) {
        unpack_upper_kernel<<<grid_for(wsz), 256, 0, s>>>(b.wr->as<double2>() + q * wsz, wr_src + pl.recs[q] * np,
                                                          ngb, 1);
        count_launch();
        QSGW_LAUNCH_CHECK("unpack_upper_kernel");
      }
    } else {
      if ((rc = g_sc_recs.ensure(nrec * sizeof(int)))) return rc;
      if ((rc = h2d(g_sc_recs.p, pl.recs.data(), nrec * sizeof(int), s))) return rc;
      hermitize_kernel<<<dim3((ngb + 31) / 32, (ngb + 31) / 32, nrec), dim3(32, 8), 0, s>>>(
          b.wr->as<double2>(), wr_src, g_sc_recs.as<int>(), ngb, ldw, nrec);
      count_launch();
      QSGW_LAUNCH_CHECK("hermitize_kernel");
    }
    wr = b.wr->as<double2>();
  }
  if ((rc = b.w3->ensure(pl.scale_bin.size() * sizeof(double)))) return rc;
  if ((rc = h2d(b.w3->p, pl.scale_bin.data(), pl.scale_bin.size() * sizeof(double), s))) return rc;
  if ((rc = b.cz->ensure(static_cast<size_t>(ngb) * ncol * sizeof(double2)))) return rc;
  sa = SigcSplitArgs();
  sa.ngb = ngb; sa.ldw = ldw;
  sa.wi = wi; sa.nimag = niw + 1;
  sa.wr = wr; sa.nreal = nrec;
  sa.zmel = reinterpret_cast<const double2*>(a.zmel); sa.ncol = ncol;
  sa.wgt = b.wg->as<double>(); sa.nwgt = ncol * (niw + 1);
  sa.w3 = b.w3->as<double>(); sa.nw3 = nrec == 0 ? 0 : static_cast<long long>(nrec) * ncol;
  sa.tile_cols = pl.tile_cols; sa.tile_group = pl.tile_group;
  sa.group_seg_off = pl.gseg_off; sa.group_nseg = pl.gnseg; sa.seg_slot = pl.seg_slot;
  sa.segs.resize(pl.seg_slot.size());
  for (size_t i = 0; i < pl.seg_slot.size(); ++i) {
    const int sl = pl.seg_slot[i];
    sa.segs[i] = sl <= niw ? ZSeg{wi + sl * wsz, sa.wgt + sl, niw + 1, 0}
                           : ZSeg{wr + (sl - niw - 1) * wsz, sa.w3 + static_cast<long long>(sl - niw - 1) * ncol, 1, 0};
  }
  sa.out = b.cz->as<double2>();
  return QSGW_OK;
}

// ---- 4. zsec += czmelwc^H zmel (:599) and the Im clamp (:601-607)
static int sxcf_finish(const qsgw_sxcf_args& a, const double2* cz) {
  cudaStream_t s = ctx().stream;
  const long long kk = static_cast<long long>(a.ngb) * (a.ns2 - a.ns1 + 1);
  const double2* zmel = reinterpret_cast<const double2*>(a.zmel);
  // a thin product (ntqxx x ntqxx over K = ngb nm): padded to 16 x 8 fragments instead of 64 x 64 tiles
  int rc = a.ntqxx <= 64
               ? zgemm_hn_thin(a.ntqxx, kk, cz, kk, zmel, kk, reinterpret_cast<double2*>(a.zsec), a.ntq, s)
               : zgemm_f64(2, 0, a.ntqxx, a.ntqxx, static_cast<int>(kk), make_double2(1, 0), cz, kk, 0, zmel, kk, 0,
                           make_double2(1, 0), reinterpret_cast<double2*>(a.zsec), a.ntq, 0, 1, s);
  if (rc) return rc;
  clamp_diag_kernel<<<(a.ntqxx + 127) / 128, 128, 0, s>>>(reinterpret_cast<double2*>(a.zsec), a.ntqxx, a.ntq);
  count_launch();
  QSGW_LAUNCH_CHECK("clamp_diag_kernel");
  return QSGW_OK;
}

static std::string sigc_slice_key(const qsgw_sxcf_args& a) {
  char key[200];
  std::snprintf(key, sizeof(key), "sigc_i8 slices ngb=%d nm=%d ntq=%d niw=%d", a.ngb, a.ns2 - a.ns1 + 1, a.ntqxx,
                a.niw);
  return key;
}

// slice count of the int8 contraction of task a (sa bound): the fixed count, or the smallest whose
// Sigma_c diagonal (this call's contribution, the quantity the QP energies take) stays within the
// target of the 4-slice one
static int sxcf_i8_slices(const qsgw_sxcf_args& a, const SigcSplitArgs& sa, int* ns_out) {
  cudaStream_t s = ctx().stream;
  int ns = ctx().nslices;
  if (ns == 0) {
    const long long kk = static_cast<long long>(a.ngb) * (a.ns2 - a.ns1 + 1);
    const double2* zmel = reinterpret_cast<const double2*>(a.zmel);
    std::vector<double> ref, cur;
    auto diag = [&](int n, std::vector<double>& d) -> int {
      int r = sigc_split_i8(sa, n, s);
      if (r) return r;
      r = g_sc_trial.ensure(static_cast<size_t>(a.ntqxx) * a.ntqxx * sizeof(double2));
      if (r) return r;
      r = zgemm_f64(2, 0, a.ntqxx, a.ntqxx, static_cast<int>(kk), make_double2(1, 0), sa.out, kk, 0, zmel, kk, 0,
                    make_double2(0, 0), g_sc_trial.as<double2>(), a.ntqxx, 0, 1, s);
      if (r) return r;
      std::vector<double2> h(static_cast<size_t>(a.ntqxx) * a.ntqxx);
      QSGW_CUDA(cudaMemcpyAsync(h.data(), g_sc_trial.p, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
      QSGW_CUDA(cudaStreamSynchronize(s));
      d.resize(a.ntqxx);
      for (int i = 0; i < a.ntqxx; ++i) d[i] = h[static_cast<size_t>(i) * (a.ntqxx + 1)].x;
      return QSGW_OK;
    };
    auto err = [&](int n, double* e) -> int {
      int r = ref.empty() ? diag(4, ref) : QSGW_OK;
      if (r) return r;
      r = diag(n, cur);
      if (r) return r;
      *e = 0.0;
      for (int i = 0; i < a.ntqxx; ++i) *e = std::max(*e, std::fabs(cur[i] - ref[i]));
      return QSGW_OK;
    };
    // the estimate comes from this call; later calls of the shape (other q, other bands) vary
    // by a few times, so the choice keeps a factor 4 of margin
    int rc = tuned_slices(sigc_slice_key(a), {2, 3}, 4, 0.25 * ctx().sigc_qp_tol, err, 4, &ns);
    if (rc) return rc;
  }
  *ns_out = ns;
  return QSGW_OK;
}

// steps 1-3 of one non-empty task: czmelwc into sa.out
static int sxcf_contract(const qsgw_sxcf_args& a, SigcSplitArgs& sa) {
  cudaStream_t s = ctx().stream;
  const bool split = ctx().prec_mode != QSGW_PREC_FP64;
  const bool i8 = ctx().prec_mode == QSGW_PREC_SPLIT_I8;
  // column tile of the int8 / split-FP16 / FP64 kernel
  const int tilew = i8 ? kOzTileN : (split ? sigc_split_tile_width() : ZG_BN);
  SxcfPlan pl;
  int rc = sxcf_plan(a, tilew, pl);
  if (rc) return rc;
  rc = sxcf_bind(a, pl, SxcfBufs{&g_sc_wg, &g_sc_w3, &g_sc_cz, &g_sc_wi, &g_sc_wr}, sa);
  if (rc) return rc;
  if (i8) {
    // ---- 3. imaginary axis + poles: int8 slices on tcgen05
    int ns = 0;
    if ((rc = sxcf_i8_slices(a, sa, &ns))) return rc;
    rc = sigc_split_i8(sa, ns, s);
  } else if (split) {
    // ---- 3'. the same contraction in split FP16 on tcgen05
    rc = sigc_split_f16(sa, s);
  } else {
    const size_t tb = sa.segs.size() * sizeof(ZSeg) +
                      (sa.group_seg_off.size() + sa.group_nseg.size() + sa.tile_group.size() + sa.tile_cols.size()) *
                          sizeof(int);
    rc = g_sc_tmp.ensure(tb + 16 * 5);
    if (rc) return rc;
    unsigned char* tbase = g_sc_tmp.as<unsigned char>();
    size_t off = 0;
    int cprc = 0;
    auto put = [&](const void* src, size_t n) -> const void* {
      void* dst = tbase + off;
      if (!cprc) cprc = h2d(dst, src, n, s);
      off += (n + 15) & ~size_t(15);
      return dst;
    };
    ZParams p{};
    p.segs = reinterpret_cast<const ZSeg*>(put(sa.segs.data(), sa.segs.size() * sizeof(ZSeg)));
    p.group_seg_off = reinterpret_cast<const int*>(put(sa.group_seg_off.data(), sa.group_seg_off.size() * sizeof(int)));
    p.group_nseg = reinterpret_cast<const int*>(put(sa.group_nseg.data(), sa.group_nseg.size() * sizeof(int)));
    p.tile_group = reinterpret_cast<const int*>(put(sa.tile_group.data(), sa.tile_group.size() * sizeof(int)));
    p.tile_cols = reinterpret_cast<const int*>(put(sa.tile_cols.data(), sa.tile_cols.size() * sizeof(int)));
    if (cprc) return cprc;
    // ---- 3. imaginary axis + poles in one launch
    p.M = a.ngb; p.K = a.ngb;
    p.a_rs = sa.ldw; p.a_ks = 1; p.a_conj = 1;          // Wc^H (:492 opA = m_op_C)
    p.B = sa.zmel; p.b_rs = a.ngb; p.b_ks = 1; p.b_conj = 0;
    p.C = sa.out; p.ldc = a.ngb; p.beta_zero = 1;
    rc = zgemm_seg_launch(p, static_cast<int>(sa.tile_group.size()), s);
  }
  return rc;
}

int sxcf_device(const qsgw_sxcf_args& a) {
  if (a.ns1 > a.ns2 || a.ntqxx == 0) return QSGW_OK;   // :418
  SigcSplitArgs sa;
  int rc;
  if (ctx().prec_mode == QSGW_PREC_SPLIT_F16 && !sigc_kind_fixed()) {
    // the split-FP16 kernel (64 x 128 tiles, CTA pairs, 64 x 256 tiles): timed once per shape
    // on this call's data when tuning is on, else the 64 x 256 one
    char key[200];
    std::snprintf(key, sizeof(key), "sigc_f16 kernel ngb=%d nm=%d ntq=%d niw=%d", a.ngb, a.ns2 - a.ns1 + 1,
                  a.ntqxx, a.niw);
    int kind = 2;
    bool tried = false;
    rc = tuned_choice(key, {0, 1, 2}, 2, [&](int k) { sigc_kind_use(k); return sxcf_contract(a, sa); },
                      ctx().stream, &kind, &tried);
    if (rc) return rc;
    sigc_kind_use(kind);
  }
  if ((rc = sxcf_contract(a, sa))) return rc;
  return sxcf_finish(a, sa.out);
}

// Tasks of one shape in SPLIT_I8 share the launches of the int8 contraction: the tasks of a group
// are planned on the host, then each is bound and sliced into the batch buffers (its W operands
// are read once, so the next task's records can reuse the same scratch), then one launch runs every
// tile of the group, then the final products run task by task.  Groups are cut where the shape or
// the slice count changes or the group's scratch passes kSigcBatchBytes.
static constexpr size_t kSigcBatchBytes = size_t(8) << 30;
static std::vector<DevBuf> g_sb_wg, g_sb_w3, g_sb_cz;   // per task of a group

int sxcf_batch_device(const qsgw_sxcf_args* t, int n) {
  if (ctx().prec_mode != QSGW_PREC_SPLIT_I8) {
    for (int i = 0; i < n; ++i) {
      const int rc = sxcf_device(t[i]);
      if (rc) return rc;
    }
    return QSGW_OK;
  }
  cudaStream_t s = ctx().stream;
  int i = 0;
  while (i < n) {
    const qsgw_sxcf_args& a0 = t[i];
    if (a0.ns1 > a0.ns2 || a0.ntqxx == 0) { ++i; continue; }   // :418
    int ns = ctx().nslices;
    if (ns == 0 && !tuned_lookup(sigc_slice_key(a0), &ns)) {
      // the first task of a shape chooses the slice count on its own data
      const int rc = sxcf_device(a0);
      if (rc) return rc;
      ++i;
      continue;
    }
    // the group: following tasks of the same ngb and slice count within the scratch budget
    std::vector<int> members;
    std::vector<SxcfPlan> plans;
    long long nslot = 0, ntiles = 0;
    size_t bytes = 0;
    for (int j = i; j < n; ++j) {
      const qsgw_sxcf_args& a = t[j];
      if (a.ns1 > a.ns2 || a.ntqxx == 0) {
        if (members.empty()) continue;
        break;
      }
      int nsj = ctx().nslices;
      if (a.ngb != a0.ngb || (nsj == 0 && (!tuned_lookup(sigc_slice_key(a), &nsj) || nsj != ns))) break;
      SxcfPlan pl;
      int rc = sxcf_plan(a, kOzTileN, pl);
      if (rc) return rc;
      const long long sl = a.niw + 1 + static_cast<long long>(pl.recs.size());
      const long long nt = static_cast<long long>(pl.tile_group.size());
      const size_t add = OzSigcBatch::bytes_per(ns, a.ngb, a.ngb, sl, nt) +
                         static_cast<size_t>(a.ngb) * pl.ncol * sizeof(double2);
      if (!members.empty() && bytes + add > kSigcBatchBytes) break;
      members.push_back(j);
      plans.push_back(std::move(pl));
      nslot += sl;
      ntiles += nt;
      bytes += add;
    }
    const int ng = static_cast<int>(members.size());
    if (static_cast<int>(g_sb_wg.size()) < ng) {
      g_sb_wg.resize(ng); g_sb_w3.resize(ng); g_sb_cz.resize(ng);
    }
    OzSigcBatch batch;
    int rc = batch.reserve(ns, a0.ngb, a0.ngb, a0.ngb, nslot, ntiles);
    if (rc) return rc;
    for (int g = 0; g < ng; ++g) {
      SigcSplitArgs sa;
      rc = sxcf_bind(t[members[g]], plans[g], SxcfBufs{&g_sb_wg[g], &g_sb_w3[g], &g_sb_cz[g], &g_sc_wi, &g_sc_wr}, sa);
      if (rc) return rc;
      if ((rc = batch.add(sa, s))) return rc;
    }
    if ((rc = batch.launch(s))) return rc;
    for (int g = 0; g < ng; ++g)
      if ((rc = sxcf_finish(t[members[g]], g_sb_cz[g].as<double2>()))) return rc;
    i = members.back() + 1;
  }
  return QSGW_OK;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_sxcf_correlation_d(const qsgw_sxcf_args* args) {
  int rc = require_init();
  if (rc) return rc;
  rc = sxcf_check(args);
  if (rc) return rc;
  QSGW_ARG((reinterpret_cast<uintptr_t>(args->zmel) & 15) == 0 &&
               (reinterpret_cast<uintptr_t>(args->wc_imag) & 15) == 0 &&
               (reinterpret_cast<uintptr_t>(args->wc_real) & 15) == 0 &&
               (reinterpret_cast<uintptr_t>(args->zsec) & 15) == 0,
           "sxcf: complex arrays must be 16-byte aligned");
  return sxcf_device(*args);
}

extern "C" int qsgw_sxcf_correlation_batch_d(const qsgw_sxcf_args* tasks, int ntask) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(ntask >= 0 && (tasks || ntask == 0), "sxcf batch: %d tasks at %p", ntask, static_cast<const void*>(tasks));
  for (int i = 0; i < ntask; ++i) {
    rc = sxcf_check(&tasks[i]);
    if (rc) return rc;
    const qsgw_sxcf_args* a = &tasks[i];
    QSGW_ARG((reinterpret_cast<uintptr_t>(a->zmel) & 15) == 0 && (reinterpret_cast<uintptr_t>(a->wc_imag) & 15) == 0 &&
                 (reinterpret_cast<uintptr_t>(a->wc_real) & 15) == 0 && (reinterpret_cast<uintptr_t>(a->zsec) & 15) == 0,
             "sxcf batch: task %d: complex arrays must be 16-byte aligned", i);
  }
  return sxcf_batch_device(tasks, ntask);
}

extern "C" int qsgw_sxcf_correlation(const qsgw_sxcf_args* args) {
  int rc = require_init();
  if (rc) return rc;
  rc = sxcf_check(args);
  if (rc) return rc;
  const qsgw_sxcf_args& a = *args;
  cudaStream_t s = ctx().stream;
  const int nm = std::max(0, a.ns2 - a.ns1 + 1);
  const size_t zb = static_cast<size_t>(a.ngb) * nm * a.ntqxx * 16;
  const size_t wrec = a.keepwv ? static_cast<size_t>(a.ngb) * (a.ngb + 1) / 2 * 16
                               : static_cast<size_t>(a.nblochpmx) * a.nblochpmx * 16;
  const size_t wib = wrec * (a.niw + 1), wrb = wrec * (a.nw + 1);
  const size_t sb = static_cast<size_t>(a.ntq) * a.ntq * 16;
  HostSlot* sl = nullptr;
  cudaStream_t cs = nullptr;
  rc = g_sc_ring.begin(&sl, &cs); if (rc) return rc;
  DevBuf &dz = sl->buf[0], &dwi = sl->buf[1], &dwr = sl->buf[2];
  rc = dz.ensure(zb); if (rc) return rc;
  rc = dwi.ensure(wib); if (rc) return rc;
  rc = dwr.ensure(wrb); if (rc) return rc;
  // inputs on the copy stream (the asynchronous mode overlaps them with the previous call)
  if (zb) QSGW_CUDA(cudaMemcpyAsync(dz.p, a.zmel, zb, cudaMemcpyHostToDevice, cs));
  QSGW_CUDA(cudaMemcpyAsync(dwi.p, a.wc_imag, wib, cudaMemcpyHostToDevice, cs));
  // only the real-axis records the pole part reads travel (as the reference
  // reads __WVR records by index, m_sxcf_gemm.f90:570)
  {
    std::vector<PoleEntry> poles;
    if (a.ns1 <= a.ns2 && a.ntqxx > 0) {
      rc = pole_table_h(a, poles);
      if (rc) return rc;
    }
    std::vector<char> need(a.nw + 1, 0);
    for (const auto& e : poles)
      for (int i = 0; i < 3; ++i) {
        const int b = e.ixs - 1 + i;
        if (b >= a.nwxi && b <= a.nwx) need[b] = 1;
      }
    for (int b = 0; b <= a.nw; ++b)
      if (need[b])
        QSGW_CUDA(cudaMemcpyAsync(dwr.as<char>() + b * wrec, reinterpret_cast<const char*>(a.wc_real) + b * wrec,
                                  wrec, cudaMemcpyHostToDevice, cs));
  }
  rc = g_sc_ring.ready(*sl, cs);
  if (rc) return rc;
  // zsec accumulates: synchronous calls copy it in and out; asynchronous calls accumulate into
  // one device image per host array until qsgw_synchronize
  void* zs_dev = nullptr;
  if (host_async()) {
    rc = host_acc_target(a.zsec, sb, s, &zs_dev);
    if (rc) return rc;
  } else {
    rc = g_sc_host_zs.ensure(sb); if (rc) return rc;
    zs_dev = g_sc_host_zs.p;
    QSGW_CUDA(cudaMemcpyAsync(zs_dev, a.zsec, sb, cudaMemcpyHostToDevice, s));
  }
  qsgw_sxcf_args d = a;
  d.zmel = dz.as<double>();
  d.wc_imag = dwi.as<double>();
  d.wc_real = dwr.as<double>();
  d.zsec = static_cast<double*>(zs_dev);
  rc = sxcf_device(d);
  if (rc) return rc;
  QSGW_CUDA(cudaMemcpyAsync(a.zsec, zs_dev, sb, cudaMemcpyDeviceToHost, s));
  return g_sc_ring.finish(*sl);
}

extern "C" int qsgw_sxcf_wgtim_d(double* wgtim_d, int niw, int ns1, int ns2, int ntqxx, int nctot,
                                 const double* omega, const double* ekc, int nekc, double esmr,
                                 double wkkr, double ua, const double* freqx, const double* wwx,
                                 const double* expa) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(wgtim_d && omega && ekc && freqx && wwx && expa, "sxcf_wgtim: null pointer");
  QSGW_ARG(niw >= 1 && ns1 >= 1 && ns2 >= ns1 && ns2 <= nekc && ntqxx >= 1, "sxcf_wgtim: bad sizes");
  QSGW_ARG(esmr > 0.0 && ua > 0.0, "sxcf_wgtim: esmr and ua must be positive");
  cudaStream_t s = ctx().stream;
  const int nm = ns2 - ns1 + 1;
  rc = g_sc_tabs.ensure((4 * niw + ntqxx + nekc + 8) * sizeof(double));
  if (rc) return rc;
  double* dt = g_sc_tabs.as<double>();
  double *d_x = dt, *d_wt = dt + niw, *d_ex = dt + 2 * niw, *d_om = dt + 3 * niw, *d_ekc = d_om + ntqxx;
  QSGW_CUDA(cudaMemcpyAsync(d_x, freqx, niw * sizeof(double), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(d_wt, wwx, niw * sizeof(double), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(d_ex, expa, niw * sizeof(double), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(d_om, omega, ntqxx * sizeof(double), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(d_ekc, ekc, nekc * sizeof(double), cudaMemcpyHostToDevice, s));
  const long long ncol = static_cast<long long>(nm) * ntqxx;
  wgtim_kernel<<<static_cast<int>((ncol + 127) / 128), 128, 0, s>>>(wgtim_d, niw, ns1, nm, ntqxx, nctot, d_om, d_ekc,
                                                                    esmr, wkkr, ua, d_x, d_wt, d_ex);
  count_launch();
  QSGW_LAUNCH_CHECK("wgtim_kernel");
  return QSGW_OK;
}
