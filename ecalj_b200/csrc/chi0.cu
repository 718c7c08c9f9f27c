// chi0 rank-k accumulation.
//   qsgw_x0gemm / qsgw_x0gemm_d : drop-in for x0gemm (x0gemm.f90:2-97).
//   qsgw_chi0_lorentz_d          : every k and every iw in one launch, with
//                                  the Lorentzian pair weights built on the
//                                  GPU in FP64.
// The host builds the (jpm, iw) bin lists in the reference's icoun order
// (x0gemm.f90:37-64); the GPU never materialises zw / wzw: the pair gather
// and the weight are folded into the operand loads of the DMMA engine.
#include <memory>
#include <cmath>
#include <vector>
#include "zgemm_f64.cuh"
#include "autotune.cuh"
#include "split_f16.cuh"
#include "ozaki_i8.cuh"
#include "hoststage.cuh"

namespace qsgw {

static DevBuf g_x0_idx, g_x0_w, g_x0_bins, g_x0_zm, g_x0_rc;

struct BinTables {
  std::vector<int> colidx;
  std::vector<double> wts;
  std::vector<int> cnt, slab;
  std::vector<long long> off;
  int maxcnt = 0;
};

// Returns the number of chunks of the longest bin.
static int upload_bins(const BinTables& bt, ZParams& p, cudaStream_t s, int& rc) {
  const size_t nb = bt.cnt.size();
  const size_t ni = bt.colidx.size();
  rc = g_x0_idx.ensure(std::max<size_t>(ni, 1) * sizeof(int));
  if (rc) return 0;
  rc = g_x0_w.ensure(std::max<size_t>(ni, 1) * sizeof(double));
  if (rc) return 0;
  const size_t bin_bytes = nb * (2 * sizeof(int) + sizeof(long long));
  rc = g_x0_bins.ensure(std::max<size_t>(bin_bytes, 64));
  if (rc) return 0;
  std::vector<unsigned char> hb(bin_bytes);
  memcpy(hb.data(), bt.off.data(), nb * sizeof(long long));
  memcpy(hb.data() + nb * sizeof(long long), bt.cnt.data(), nb * sizeof(int));
  memcpy(hb.data() + nb * (sizeof(long long) + sizeof(int)), bt.slab.data(), nb * sizeof(int));
  if (ni) {
    rc = check_cuda(cudaMemcpyAsync(g_x0_idx.p, bt.colidx.data(), ni * sizeof(int), cudaMemcpyHostToDevice, s), "H2D pair columns");
    if (rc) return 0;
    rc = check_cuda(cudaMemcpyAsync(g_x0_w.p, bt.wts.data(), ni * sizeof(double), cudaMemcpyHostToDevice, s), "H2D pair weights");
    if (rc) return 0;
  }
  rc = check_cuda(cudaMemcpyAsync(g_x0_bins.p, hb.data(), bin_bytes, cudaMemcpyHostToDevice, s), "H2D bins");
  if (rc) return 0;
  // the pageable copies above are staged before returning, hb may die now
  unsigned char* base = g_x0_bins.as<unsigned char>();
  p.bin_coff = reinterpret_cast<const long long*>(base);
  p.bin_woff = reinterpret_cast<const long long*>(base);
  p.bin_cnt = reinterpret_cast<const int*>(base + nb * sizeof(long long));
  p.bin_slab = reinterpret_cast<const int*>(base + nb * (sizeof(long long) + sizeof(int)));
  p.colidx = g_x0_idx.as<int>();
  p.wts = g_x0_w.as<double>();
  return (bt.maxcnt + ZG_BK - 1) / ZG_BK;
}

static int choose_splitk(int ntiles, int nbins, int maxch) {
  const long long ctas = static_cast<long long>(ntiles) * nbins;
  const long long slots = 2LL * ctx().sm_count;
  if (ctas >= slots || maxch < 16) return 1;
  int sk = static_cast<int>((slots + ctas - 1) / ctas);
  return std::max(1, std::min(sk, maxch / 8));
}

static int x0gemm_device(double2* rcxq, int npr, int ipr_col, int npr_col, int nwhis, int npm,
                         int ns1, int ns2, const double2* zmel, int nbb, int nm1, int nm2,
                         int nqtot, int icounkmink, int icounkmaxk, const int* itc, const int* itpc,
                         const int* jpmc, const int* iwini, const int* iwend, const int* icouini,
                         const double* whwc, int ncount) {
  cudaStream_t s = ctx().stream;
  const int nmz = nm2 - nm1 + 1;
  // ---- bin lists in icoun order (x0gemm.f90:37-64) ----
  const int nbins_all = nwhis * npm;
  std::vector<int> cnt(nbins_all, 0);
  for (int icoun = icounkmink; icoun <= icounkmaxk; ++icoun) {
    const int c = icoun - 1;
    const int jpm = jpmc[c], it = itc[c], itp = itpc[c];
    QSGW_ARG(jpm >= 1 && jpm <= npm, "x0gemm: jpmc(%d)=%d outside 1..npm", icoun, jpm);
    if (it < ns1 || it > ns2) continue;
    QSGW_ARG(it >= nm1 && it <= nm2, "x0gemm: itc(%d)=%d outside zmel bounds %d:%d", icoun, it, nm1, nm2);
    QSGW_ARG(itp >= 1 && itp <= nqtot, "x0gemm: itpc(%d)=%d outside 1..nqtot", icoun, itp);
    QSGW_ARG(iwini[c] >= 1 && iwend[c] <= nwhis, "x0gemm: bins %d..%d outside 1..nwhis", iwini[c], iwend[c]);
    QSGW_ARG(icouini[c] >= 1 && icouini[c] + (iwend[c] - iwini[c]) <= ncount,
             "x0gemm: icouini(%d)=%d outside whwc", icoun, icouini[c]);
    for (int iw = iwini[c]; iw <= iwend[c]; ++iw) cnt[(jpm - 1) * nwhis + (iw - 1)]++;
  }
  BinTables bt;
  std::vector<long long> start(nbins_all, 0);
  long long tot = 0;
  for (int jpm = 1; jpm <= npm; ++jpm)
    for (int iw = 1; iw <= nwhis; ++iw) {
      const int b = (jpm - 1) * nwhis + (iw - 1);
      start[b] = tot;
      if (cnt[b] > 0) {
        bt.cnt.push_back(cnt[b]);
        bt.off.push_back(tot);
        bt.slab.push_back(iw * (3 - 2 * jpm) - (1 - npm) * nwhis);
        bt.maxcnt = std::max(bt.maxcnt, cnt[b]);
      }
      tot += cnt[b];
    }
  if (bt.cnt.empty()) return QSGW_OK;
  bt.colidx.resize(tot);
  bt.wts.resize(tot);
  std::vector<long long> fill(start);
  for (int icoun = icounkmink; icoun <= icounkmaxk; ++icoun) {
    const int c = icoun - 1;
    const int jpm = jpmc[c], it = itc[c], itp = itpc[c];
    if (it < ns1 || it > ns2) continue;
    const int col = (it - nm1) + nmz * (itp - 1);
    for (int iw = iwini[c]; iw <= iwend[c]; ++iw) {
      const int b = (jpm - 1) * nwhis + (iw - 1);
      bt.colidx[fill[b]] = col;
      bt.wts[fill[b]] = whwc[iw - iwini[c] + icouini[c] - 1];   // x0gemm.f90:62
      fill[b]++;
    }
  }
  if (ctx().prec_mode == QSGW_PREC_SPLIT_I8) {
    // the same bins on the int8 tensor-core path: the pair columns and weights go to the device,
    // each bin's entries form one K range; rcxq accumulates (no tuning trials)
    int rc = g_x0_idx.ensure(std::max<size_t>(tot, 1) * sizeof(int));
    if (rc) return rc;
    rc = g_x0_w.ensure(std::max<size_t>(tot, 1) * sizeof(double));
    if (rc) return rc;
    if ((rc = h2d(g_x0_idx.p, bt.colidx.data(), tot * sizeof(int), s))) return rc;
    if ((rc = h2d(g_x0_w.p, bt.wts.data(), tot * sizeof(double), s))) return rc;
    OzChi0Bins ob;
    ob.ebeg = bt.off;
    ob.cnt = bt.cnt;
    ob.slab = bt.slab;
    int classes = 0;
    for (double w : bt.wts) classes |= (w < 0.0 ? 1 : 0) | (w > 0.0 ? 2 : 0);
    const bool herm = (ipr_col == 1 && npr_col == npr);
    const int ns = ctx().nslices > 0 ? ctx().nslices : 4;   // rcxq accumulates: no trials, the accurate count
    return chi0_split_i8(rcxq, npr, static_cast<long long>(npr) * npr_col, npr, npr_col, ipr_col - 1, herm, zmel, nbb,
                         static_cast<long long>(nmz) * nqtot, g_x0_idx.as<int>(), g_x0_w.as<double>(), ob, classes,
                         ns, s, nullptr);
  }
  ZParams p{};
  p.M = npr; p.N = npr_col;
  p.A = zmel; p.a_rs = 1; p.a_ks = nbb; p.a_conj = 1;               // zw^H   (:76, :88 opA=C)
  p.B = zmel + (ipr_col - 1); p.b_rs = 1; p.b_ks = nbb; p.b_conj = 0;  // wzw   (:84)
  p.C = rcxq; p.ldc = npr; p.c_bs = static_cast<long long>(npr) * npr_col;
  p.ntm = (npr + ZG_BM - 1) / ZG_BM; p.ntn = (npr_col + ZG_BN - 1) / ZG_BN;
  int rc = 0;
  const int maxch = upload_bins(bt, p, s, rc);
  if (rc) return rc;
  const int herm = (ipr_col == 1 && npr_col == npr) ? 1 : 0;
  const int ntiles = herm ? p.ntm * (p.ntm + 1) / 2 : p.ntm * p.ntn;
  const int nbins = static_cast<int>(bt.cnt.size());
  const int sk = choose_splitk(ntiles, nbins, maxch);
  p.kch_per_split = (maxch + sk - 1) / sk;
  rc = zgemm_chi0_launch(p, nbins, herm, sk, s);
  if (rc) return rc;
  // host vectors must outlive the async copies from pageable memory: they do,
  // because pageable cudaMemcpyAsync stages the data before returning.
  return QSGW_OK;
}

static int x0gemm_check(int npr, int ipr_col, int npr_col, int nwhis, int npm, int nbb, int nm1,
                        int nm2, int nqtot, int icounkmink, int icounkmaxk, int ncount,
                        const void* rcxq, const void* zmel) {
  QSGW_ARG(npr >= 1 && npr_col >= 1 && ipr_col >= 1, "x0gemm: bad npr=%d npr_col=%d ipr_col=%d", npr, npr_col, ipr_col);
  QSGW_ARG(npr <= nbb && ipr_col - 1 + npr_col <= nbb, "x0gemm: product-basis range exceeds nbb=%d", nbb);
  QSGW_ARG(npm == 1 || npm == 2, "x0gemm: npm=%d", npm);
  QSGW_ARG(nwhis >= 1, "x0gemm: nwhis=%d", nwhis);
  QSGW_ARG(nm2 >= nm1 && nqtot >= 1, "x0gemm: zmel bounds %d:%d nqtot=%d", nm1, nm2, nqtot);
  QSGW_ARG(icounkmink >= 1 && icounkmaxk >= icounkmink - 1, "x0gemm: icoun range %d..%d", icounkmink, icounkmaxk);
  QSGW_ARG(ncount >= 0, "x0gemm: ncount=%d", ncount);
  QSGW_ARG(rcxq && zmel, "x0gemm: null array");
  QSGW_ARG((reinterpret_cast<uintptr_t>(rcxq) & 15) == 0 && (reinterpret_cast<uintptr_t>(zmel) & 15) == 0,
           "x0gemm: complex arrays must be 16-byte aligned");
  return QSGW_OK;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_x0gemm_d(double* rcxq_d, int npr, int ipr_col, int npr_col, int nwhis, int npm,
                             int ns1, int ns2, const double* zmel_d, int nbb, int nm1, int nm2,
                             int nqtot, int icounkmink, int icounkmaxk, const int* itc,
                             const int* itpc, const int* jpmc, const int* iwini, const int* iwend,
                             const int* icouini, const double* whwc, int ncount) {
  int rc = require_init();
  if (rc) return rc;
  rc = x0gemm_check(npr, ipr_col, npr_col, nwhis, npm, nbb, nm1, nm2, nqtot, icounkmink, icounkmaxk,
                    ncount, rcxq_d, zmel_d);
  if (rc) return rc;
  if (icounkmaxk < icounkmink) return QSGW_OK;
  QSGW_ARG(itc && itpc && jpmc && iwini && iwend && icouini && whwc, "x0gemm: null index table");
  return x0gemm_device(reinterpret_cast<double2*>(rcxq_d), npr, ipr_col, npr_col, nwhis, npm, ns1,
                       ns2, reinterpret_cast<const double2*>(zmel_d), nbb, nm1, nm2, nqtot,
                       icounkmink, icounkmaxk, itc, itpc, jpmc, iwini, iwend, icouini, whwc, ncount);
}

extern "C" int qsgw_x0gemm(double* rcxq, int npr, int ipr_col, int npr_col, int nwhis, int npm,
                           int ns1, int ns2, const double* zmel, int nbb, int nm1, int nm2,
                           int nqtot, int icounkmink, int icounkmaxk, const int* itc,
                           const int* itpc, const int* jpmc, const int* iwini, const int* iwend,
                           const int* icouini, const double* whwc, int ncount) {
  int rc = require_init();
  if (rc) return rc;
  rc = x0gemm_check(npr, ipr_col, npr_col, nwhis, npm, nbb, nm1, nm2, nqtot, icounkmink, icounkmaxk,
                    ncount, rcxq, zmel);
  if (rc) return rc;
  if (icounkmaxk < icounkmink) return QSGW_OK;
  cudaStream_t s = ctx().stream;
  const size_t nslab = static_cast<size_t>(npm == 1 ? nwhis + 1 : 2 * nwhis + 1);
  const size_t rc_bytes = static_cast<size_t>(npr) * npr_col * nslab * 16;
  const size_t zm_bytes = static_cast<size_t>(nbb) * (nm2 - nm1 + 1) * nqtot * 16;
  rc = g_x0_rc.ensure(rc_bytes); if (rc) return rc;
  rc = g_x0_zm.ensure(zm_bytes); if (rc) return rc;
  QSGW_CUDA(cudaMemcpyAsync(g_x0_rc.p, rcxq, rc_bytes, cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(g_x0_zm.p, zmel, zm_bytes, cudaMemcpyHostToDevice, s));
  rc = qsgw_x0gemm_d(g_x0_rc.as<double>(), npr, ipr_col, npr_col, nwhis, npm, ns1, ns2,
                     g_x0_zm.as<double>(), nbb, nm1, nm2, nqtot, icounkmink, icounkmaxk, itc, itpc,
                     jpmc, iwini, iwend, icouini, whwc, ncount);
  if (rc) return rc;
  QSGW_CUDA(cudaMemcpyAsync(rcxq, g_x0_rc.p, rc_bytes, cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  return QSGW_OK;
}

// ---------------------------------------------------------------------------
// All-k chi0 with Lorentzian weights built on the device.
namespace qsgw {

__global__ void lorentz_weight_kernel(double* __restrict__ w, const int* __restrict__ peo,
                                      const int* __restrict__ peu, const double* __restrict__ eo,
                                      const double* __restrict__ eu, const double* __restrict__ fi,
                                      long long npair, int niw, double inv_nk) {
  const long long total = npair * niw;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long pr = i % npair;
    const int iw = static_cast<int>(i / npair);
    const double de = eu[peu[pr]] - eo[peo[pr]];
    const double om = fi[iw];
    w[i] = -2.0 * de / (de * de + om * om) * inv_nk;   // chi0(iw) <= 0 (dpsion5.f90:218)
  }
}

// Real frequency axis: f(w) = [1/(w - de + i eta) - 1/(w + de + i eta)] / nk, whose value at
// w = i nu is the imaginary-axis weight above.  Slot iw holds Re f, slot nw + iw holds Im f.
__global__ void lorentz_real_weight_kernel(double* __restrict__ w, const int* __restrict__ peo,
                                           const int* __restrict__ peu, const double* __restrict__ eo,
                                           const double* __restrict__ eu, const double* __restrict__ fr,
                                           long long npair, int nw, double eta, double inv_nk) {
  const long long total = npair * nw;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long pr = i % npair;
    const int iw = static_cast<int>(i / npair);
    const double de = eu[peu[pr]] - eo[peo[pr]];
    const double om = fr[iw];
    const double a = om - de, b = om + de, e2 = eta * eta;
    const double da = 1.0 / (a * a + e2), db = 1.0 / (b * b + e2);
    w[i] = (a * da - b * db) * inv_nk;
    w[static_cast<long long>(nw) * npair + i] = (-eta * da + eta * db) * inv_nk;
  }
}

static DevBuf g_lz_map, g_lz_e, g_lz_w, g_lz_bins, g_lz_fi;

// eta < 0: imaginary axis, nw slots of weights; eta >= 0: real axis, 2 nw slots (Re, Im).
// classes (out): bit 0 when a weight can be negative, bit 1 when one can be positive
int chi0_lorentz_weights(int niw, const double* freq_i, int nk, const int* nocc, const int* nun,
                         const double* eocc, const double* eunocc, long long& npair, double*& w_d,
                         cudaStream_t s, double eta = -1.0, int nk_norm = 0, int* classes = nullptr) {
  const double inv_nk = 1.0 / (nk_norm > 0 ? nk_norm : nk);   // 1/nk of the whole k mesh
  npair = 0;
  long long no_tot = 0, nu_tot = 0;
  for (int k = 0; k < nk; ++k) {
    QSGW_ARG(nocc[k] >= 0 && nun[k] >= 0, "chi0: negative band count at k=%d", k);
    npair += static_cast<long long>(nocc[k]) * nun[k];
    no_tot += nocc[k];
    nu_tot += nun[k];
  }
  std::vector<int> peo(npair), peu(npair);
  long long c = 0, oo = 0, uo = 0;
  for (int k = 0; k < nk; ++k) {
    // column order of zcols: (it - 1) + nocc_k * (itp - 1), as zmel(:, it, itp)
    for (int itp = 0; itp < nun[k]; ++itp)
      for (int it = 0; it < nocc[k]; ++it) {
        peo[c] = static_cast<int>(oo + it);
        peu[c] = static_cast<int>(uo + itp);
        ++c;
      }
    oo += nocc[k];
    uo += nun[k];
  }
  if (classes) {
    // imaginary axis: w = -2 de / (de^2 + w^2) / nk has the sign of -de; the real axis has both
    int cl = 0;
    if (eta >= 0.0) cl = 3;
    else
      for (long long i = 0; i < npair && cl != 3; ++i) {
        const double de = eunocc[peu[i]] - eocc[peo[i]];
        cl |= (de > 0.0 ? 1 : 0) | (de < 0.0 ? 2 : 0);
      }
    *classes = cl;
  }
  int rc = g_lz_map.ensure(2 * std::max<long long>(npair, 1) * sizeof(int));
  if (rc) return rc;
  rc = g_lz_e.ensure((no_tot + nu_tot + 1) * sizeof(double));
  if (rc) return rc;
  rc = g_lz_w.ensure(std::max<long long>(npair, 1) * niw * (eta >= 0.0 ? 2 : 1) * sizeof(double));
  if (rc) return rc;
  rc = g_lz_fi.ensure(niw * sizeof(double));
  if (rc) return rc;
  int* dpeo = g_lz_map.as<int>();
  int* dpeu = dpeo + npair;
  double* deo = g_lz_e.as<double>();
  double* deu = deo + no_tot;
  if ((rc = h2d(dpeo, peo.data(), npair * sizeof(int), s))) return rc;
  if ((rc = h2d(dpeu, peu.data(), npair * sizeof(int), s))) return rc;
  if ((rc = h2d(deo, eocc, no_tot * sizeof(double), s))) return rc;
  if ((rc = h2d(deu, eunocc, nu_tot * sizeof(double), s))) return rc;
  if ((rc = h2d(g_lz_fi.p, freq_i, niw * sizeof(double), s))) return rc;
  const long long tot = npair * niw;
  const int blocks = static_cast<int>(std::min<long long>((tot + 255) / 256, 8LL * ctx().sm_count));
  if (tot > 0 && eta < 0.0) {
    lorentz_weight_kernel<<<std::max(blocks, 1), 256, 0, s>>>(g_lz_w.as<double>(), dpeo, dpeu, deo, deu,
                                                              g_lz_fi.as<double>(), npair, niw, inv_nk);
    count_launch();
    QSGW_LAUNCH_CHECK("lorentz_weight_kernel");
  } else if (tot > 0) {
    lorentz_real_weight_kernel<<<std::max(blocks, 1), 256, 0, s>>>(g_lz_w.as<double>(), dpeo, dpeu, deo, deu,
                                                                   g_lz_fi.as<double>(), npair, niw, eta, inv_nk);
    count_launch();
    QSGW_LAUNCH_CHECK("lorentz_real_weight_kernel");
  }
  w_d = g_lz_w.as<double>();
  return QSGW_OK;
}

static DevBuf g_lz_ident;

__global__ void iota_kernel(int* a, long long n) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    a[i] = static_cast<int>(i);
}

// chi = Hre + i Him for the real axis (Hre, Him: the Re-weight and Im-weight slots)
__global__ void combine_re_im_kernel(double2* __restrict__ chi, const double2* __restrict__ hre,
                                     const double2* __restrict__ him, long long n) {
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double2 a = hre[e], b = him[e];
    chi[e] = make_double2(a.x - b.y, a.y + b.x);
  }
}

static DevBuf g_lzr_h;
static DevBuf g_lz_ref, g_lz_try;       // chi0 of the slice-count trials

}  // namespace qsgw

static int chi0_run(double* chi0_d, int npr, int niw, const double* zcols_d, int ldz, long long npair,
                    const double* w_d, cudaStream_t s, bool accumulate = false, int classes = 3);

extern "C" int qsgw_chi0_lorentz_d(double* chi0_d, int npr, int niw, const double* freq_i, int nk,
                                   const int* nocc, const int* nun, const double* eocc,
                                   const double* eunocc, const double* zcols_d, int ldz) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(chi0_d && zcols_d && freq_i && nocc && nun && eocc && eunocc, "chi0_lorentz: null pointer");
  QSGW_ARG(npr >= 1 && niw >= 1 && nk >= 1 && ldz >= npr, "chi0_lorentz: npr=%d niw=%d nk=%d ldz=%d", npr, niw, nk, ldz);
  QSGW_ARG((reinterpret_cast<uintptr_t>(chi0_d) & 15) == 0 && (reinterpret_cast<uintptr_t>(zcols_d) & 15) == 0,
           "chi0_lorentz: complex arrays must be 16-byte aligned");
  cudaStream_t s = ctx().stream;
  long long npair = 0;
  double* w_d = nullptr;
  int classes = 3;
  rc = chi0_lorentz_weights(niw, freq_i, nk, nocc, nun, eocc, eunocc, npair, w_d, s, -1.0, 0, &classes);
  if (rc) return rc;
  QSGW_ARG(npair < (1LL << 31), "chi0_lorentz: %lld pairs exceed the 32-bit column index", npair);
  return chi0_run(chi0_d, npr, niw, zcols_d, ldz, npair, w_d, s, false, classes);
}

// chi0 slots iw = conj(Z) diag(w[iw]) Z^T for precomputed weights w (nslot x npair), in the
// precision mode of the context; chi0_d is overwritten.
static int chi0_run(double* chi0_d, int npr, int niw, const double* zcols_d, int ldz, long long npair,
                    const double* w_d, cudaStream_t s, bool accumulate, int classes) {
  int rc = QSGW_OK;
  const size_t cbytes = static_cast<size_t>(npr) * npr * niw * 16;
  if (!accumulate) QSGW_CUDA(cudaMemsetAsync(chi0_d, 0, cbytes, s));
  if (npair == 0) return QSGW_OK;
  std::unique_ptr<TuneSuspend> hold(accumulate ? new TuneSuspend() : nullptr);   // trials would clear chi0
  if (ctx().prec_mode == QSGW_PREC_SPLIT_I8) {
    // one bin per frequency slot, every pair in every bin in column order (weights w[iw * npair + p])
    OzChi0Bins ob;
    for (int iw = 0; iw < niw; ++iw) {
      ob.ebeg.push_back(static_cast<long long>(iw) * npair);
      ob.cnt.push_back(static_cast<int>(npair));
      ob.slab.push_back(iw);
    }
    auto run_ns = [&](int ns, double2* out, const char* tune) {
      return chi0_split_i8(out, npr, static_cast<long long>(npr) * npr, npr, npr, 0, true,
                           reinterpret_cast<const double2*>(zcols_d), ldz, npair, nullptr, w_d, ob, classes, ns, s,
                           tune);
    };
    int ns = ctx().nslices;
    if (ns == 0) {
      // automatic slice count: the smallest whose chi0 stays within the relative target of the
      // 4-slice one (trials on scratch copies; accumulating calls take the choice already made)
      const long long nel = static_cast<long long>(npr) * npr * niw;
      bool have_ref = false;
      auto err = [&](int n, double* e) -> int {
        int r = g_lz_ref.ensure(nel * sizeof(double2));
        if (r) return r;
        r = g_lz_try.ensure(nel * sizeof(double2));
        if (r) return r;
        if (!have_ref) {
          QSGW_CUDA(cudaMemsetAsync(g_lz_ref.p, 0, nel * sizeof(double2), s));
          if ((r = run_ns(4, g_lz_ref.as<double2>(), nullptr))) return r;
          have_ref = true;
        }
        QSGW_CUDA(cudaMemsetAsync(g_lz_try.p, 0, nel * sizeof(double2), s));
        if ((r = run_ns(n, g_lz_try.as<double2>(), nullptr))) return r;
        return rel_diff_fro(g_lz_try.as<double2>(), g_lz_ref.as<double2>(), nel, s, e);
      };
      char key[160];
      std::snprintf(key, sizeof(key), "chi0_i8 slices npr=%d npair~2^%.3f niw=%d", npr,
                    std::round(8.0 * std::log2(static_cast<double>(npair))) / 8.0, niw);
      rc = tuned_slices(key, {2, 3}, 4, ctx().chi0_rel_tol, err, 3, &ns);
      if (rc) return rc;
    }
    return run_ns(ns, reinterpret_cast<double2*>(chi0_d), accumulate ? nullptr : "chi0_lorentz");
  }
  if (ctx().prec_mode == QSGW_PREC_SPLIT_F16) {
    return chi0_split_f16(reinterpret_cast<double2*>(chi0_d), npr, niw,
                          reinterpret_cast<const double2*>(zcols_d), ldz, npair, w_d, s);
  }
  rc = g_lz_ident.ensure(npair * sizeof(int));
  if (rc) return rc;
  iota_kernel<<<static_cast<int>(std::min<long long>((npair + 255) / 256, 4096)), 256, 0, s>>>(
      g_lz_ident.as<int>(), npair);
  count_launch();
  QSGW_LAUNCH_CHECK("iota_kernel");
  // one bin per iw, all pairs in every bin, bin iw's weights at offset iw*npair
  std::vector<long long> off(2 * niw);
  std::vector<int> cs(2 * niw);
  for (int iw = 0; iw < niw; ++iw) {
    off[iw] = 0;                                  // column offsets (shared identity list)
    off[niw + iw] = static_cast<long long>(iw) * npair;   // weight offsets
    cs[iw] = static_cast<int>(npair);
    cs[niw + iw] = iw;                            // slab
  }
  rc = g_lz_bins.ensure(2 * niw * (sizeof(long long) + sizeof(int)));
  if (rc) return rc;
  unsigned char* base = g_lz_bins.as<unsigned char>();
  if ((rc = h2d(base, off.data(), 2 * niw * sizeof(long long), s))) return rc;
  if ((rc = h2d(base + 2 * niw * sizeof(long long), cs.data(), 2 * niw * sizeof(int), s))) return rc;
  ZParams p{};
  p.M = npr; p.N = npr;
  p.A = reinterpret_cast<const double2*>(zcols_d); p.a_rs = 1; p.a_ks = ldz; p.a_conj = 1;
  p.B = reinterpret_cast<const double2*>(zcols_d); p.b_rs = 1; p.b_ks = ldz; p.b_conj = 0;
  p.C = reinterpret_cast<double2*>(chi0_d); p.ldc = npr; p.c_bs = static_cast<long long>(npr) * npr;
  p.ntm = p.ntn = (npr + ZG_BM - 1) / ZG_BM;
  p.bin_coff = reinterpret_cast<const long long*>(base);
  p.bin_woff = reinterpret_cast<const long long*>(base) + niw;
  p.bin_cnt = reinterpret_cast<const int*>(base + 2 * niw * sizeof(long long));
  p.bin_slab = p.bin_cnt + niw;
  p.colidx = g_lz_ident.as<int>();
  p.wts = w_d;
  const int maxch = static_cast<int>((npair + ZG_BK - 1) / ZG_BK);
  const int ntiles = p.ntm * (p.ntm + 1) / 2;
  const int heur = choose_splitk(ntiles, niw, maxch);
  // split K: the autotuner times the heuristic and its neighbours (x1/2, x2, x4) on this shape
  auto run = [&](int sk, bool clear) -> int {      // trials clear chi0 (it was cleared above)
    ZParams q = p;
    q.kch_per_split = (maxch + sk - 1) / sk;
    if (clear) QSGW_CUDA(cudaMemsetAsync(chi0_d, 0, cbytes, s));
    return zgemm_chi0_launch(q, niw, 1, sk, s);
  };
  std::vector<int> cands;
  for (int c : {heur / 2, heur, heur * 2, heur * 4})
    if (c >= 1 && c <= maxch && (cands.empty() || cands.back() != c)) cands.push_back(c);
  char key[160];
  // pair counts within ~9% share a choice (they differ from q to q)
  std::snprintf(key, sizeof(key), "chi0_dmma npr=%d npair~2^%.3f niw=%d", npr,
                std::round(8.0 * std::log2(static_cast<double>(npair))) / 8.0, niw);
  int sk = heur;
  bool tried = false;
  rc = tuned_choice(key, cands, heur, [&](int c) { return run(c, true); }, s, &sk, &tried);
  if (rc) return rc;
  return run(sk, tried);
}

extern "C" int qsgw_chi0_lorentz_acc_d(double* chi0_d, int npr, int niw, const double* freq_i, int nk_total,
                                       int nkb, const int* nocc, const int* nun, const double* eocc,
                                       const double* eunocc, const double* zcols_d, int ldz) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(chi0_d && zcols_d && freq_i && nocc && nun && eocc && eunocc, "chi0_lorentz_acc: null pointer");
  QSGW_ARG(npr >= 1 && niw >= 1 && nkb >= 1 && nk_total >= nkb && ldz >= npr,
           "chi0_lorentz_acc: npr=%d niw=%d nkb=%d nk_total=%d ldz=%d", npr, niw, nkb, nk_total, ldz);
  QSGW_ARG((reinterpret_cast<uintptr_t>(chi0_d) & 15) == 0 && (reinterpret_cast<uintptr_t>(zcols_d) & 15) == 0,
           "chi0_lorentz_acc: complex arrays must be 16-byte aligned");
  cudaStream_t s = ctx().stream;
  long long npair = 0;
  double* w_d = nullptr;
  int classes = 3;
  rc = chi0_lorentz_weights(niw, freq_i, nkb, nocc, nun, eocc, eunocc, npair, w_d, s, -1.0, nk_total, &classes);
  if (rc) return rc;
  QSGW_ARG(npair < (1LL << 31), "chi0_lorentz_acc: %lld pairs exceed the 32-bit column index", npair);
  return chi0_run(chi0_d, npr, niw, zcols_d, ldz, npair, w_d, s, true, classes);
}

extern "C" int qsgw_chi0_lorentz_real_d(double* chi0_d, int npr, int nw, const double* freq_r, double eta, int nk,
                                        const int* nocc, const int* nun, const double* eocc,
                                        const double* eunocc, const double* zcols_d, int ldz) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(chi0_d && zcols_d && freq_r && nocc && nun && eocc && eunocc, "chi0_lorentz_real: null pointer");
  QSGW_ARG(npr >= 1 && nw >= 1 && nk >= 1 && ldz >= npr && eta >= 0.0,
           "chi0_lorentz_real: npr=%d nw=%d nk=%d ldz=%d eta=%g", npr, nw, nk, ldz, eta);
  QSGW_ARG((reinterpret_cast<uintptr_t>(chi0_d) & 15) == 0 && (reinterpret_cast<uintptr_t>(zcols_d) & 15) == 0,
           "chi0_lorentz_real: complex arrays must be 16-byte aligned");
  cudaStream_t s = ctx().stream;
  long long npair = 0;
  double* w_d = nullptr;
  rc = chi0_lorentz_weights(nw, freq_r, nk, nocc, nun, eocc, eunocc, npair, w_d, s, eta);
  if (rc) return rc;
  QSGW_ARG(npair < (1LL << 31), "chi0_lorentz_real: %lld pairs exceed the 32-bit column index", npair);
  const long long nn = static_cast<long long>(npr) * npr * nw;
  rc = g_lzr_h.ensure(static_cast<size_t>(2 * nn) * sizeof(double2));
  if (rc) return rc;
  double2* h = g_lzr_h.as<double2>();
  // both Hermitian parts in one run over 2 nw weight slots
  rc = chi0_run(reinterpret_cast<double*>(h), npr, 2 * nw, zcols_d, ldz, npair, w_d, s);
  if (rc) return rc;
  combine_re_im_kernel<<<static_cast<int>(std::min<long long>((nn + 255) / 256, 16LL * ctx().sm_count)), 256, 0,
                         s>>>(reinterpret_cast<double2*>(chi0_d), h, h + nn, nn);
  count_launch();
  QSGW_LAUNCH_CHECK("combine_re_im_kernel");
  return QSGW_OK;
}

static qsgw::DevBuf g_lzh_c;
static qsgw::HostRing g_lzh_ring(2);    // zcols of the host-pointer calls

extern "C" int qsgw_chi0_lorentz(double* chi0, int npr, int niw, const double* freq_i, int nk,
                                 const int* nocc, const int* nun, const double* eocc,
                                 const double* eunocc, const double* zcols, int ldz) {
  using namespace qsgw;
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(chi0 && zcols && nocc && nun, "chi0_lorentz: null pointer");
  QSGW_ARG(npr >= 1 && niw >= 1 && nk >= 1 && ldz >= npr, "chi0_lorentz: npr=%d niw=%d nk=%d ldz=%d", npr, niw, nk, ldz);
  long long ncol = 0;
  for (int k = 0; k < nk; ++k) ncol += static_cast<long long>(nocc[k]) * nun[k];
  cudaStream_t s = ctx().stream;
  const size_t zb = static_cast<size_t>(ldz) * ncol * 16;
  const size_t cb = static_cast<size_t>(npr) * npr * niw * 16;
  HostSlot* sl = nullptr;
  cudaStream_t cs = nullptr;
  rc = g_lzh_ring.begin(&sl, &cs); if (rc) return rc;
  DevBuf& dz = sl->buf[0];
  rc = dz.ensure(zb); if (rc) return rc;
  rc = g_lzh_c.ensure(cb); if (rc) return rc;   // one output image, reused in stream order
  QSGW_CUDA(cudaMemcpyAsync(dz.p, zcols, zb, cudaMemcpyHostToDevice, cs));
  rc = g_lzh_ring.ready(*sl, cs);
  if (rc) return rc;
  rc = qsgw_chi0_lorentz_d(g_lzh_c.as<double>(), npr, niw, freq_i, nk, nocc, nun, eocc, eunocc,
                           dz.as<double>(), ldz);
  if (rc) return rc;
  QSGW_CUDA(cudaMemcpyAsync(chi0, g_lzh_c.p, cb, cudaMemcpyDeviceToHost, s));
  return g_lzh_ring.finish(*sl);
}
