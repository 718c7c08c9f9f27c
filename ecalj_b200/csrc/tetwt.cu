// Tetrahedron histogram weights of chi0 on the GPU (FP64 scalar geometry per
// (tetrahedron, occupied band, unoccupied band)): the Rath-Freeman microcell
// integral of SRC/subroutines/tetwt5.f90 (lindtet6 :514-600, inttetra6
// :601-672, inttetrac6 :673-713, intttvc6 :714-787 with
// tetrahedron_matrix_linear = F, midk/midk3), integtetn (m_tetrakbt.f90:441-466)
// and the corner accumulation of tetwt5x_dtet4 (:304-341, npm = 1, wtet = 1/4):
//     w(ihis, jb, ib, k) += wtthis(ihis) * pi / (4 voltot)   for each corner k.
// The reference's sparse (ibjb, ihw, nhw, jhw, whw) storage is replaced by this
// dense array.  Its symmetrisation over degenerate bands (tetwt5.f90:347-423) is
// the host-only qsgw_tetwt_symmetrize, applied to the host copy of the array
// that qsgw_x0_lists reads.
#include <algorithm>
#include <cmath>
#include <vector>
#include "common.cuh"

namespace qsgw {

struct TetCtx {
  const double* frhis;
  int nwhis;
  double* out;        // w + bin offset of this (jb, ib): out[ihis + stride_k * corner_k]
  long long stride_k;
  int corner[4];
  double fac;
  int* flag;
};

// insertion sort of util.f90:574-594 (ascending index order)
__device__ __forceinline__ void sort4(const double* v, int* o) {
  for (int i = 0; i < 4; ++i) o[i] = i;
  for (int ix = 1; ix < 4; ++ix)
    for (int i = ix; i >= 1 && v[o[i - 1]] > v[o[i]]; --i) {
      const int t = o[i - 1];
      o[i - 1] = o[i];
      o[i] = t;
    }
}

__device__ double integtetn_d(const double* e, double ee) {
  const double e1 = e[0] - 3e-8, e2 = e[1] - 2e-8, e3 = e[2] - 1e-8, e4 = e[3];
  const double v1 = ee - e1, v2 = ee - e2, v4 = ee - e4;
  if (ee < e1) return 0.0;
  if (ee < e2) return v1 * v1 * v1 / ((e4 - e1) * (e3 - e1) * (e2 - e1));
  if (ee < e3) {
    const double a = v1 / cbrt((e4 - e1) * (e3 - e1) * (e2 - e1));
    const double b = v2 / cbrt(-(e4 - e2) * (e3 - e2) * (e1 - e2));
    return (a - b) * (a * a + a * b + b * b);
  }
  if (ee < e4) return 1.0 - v4 * v4 * v4 / ((e1 - e4) * (e2 - e4) * (e3 - e4));
  return 1.0;
}

// intttvc6: histogram of omega = -v over a tetrahedron of volume voltet, added to every corner
__device__ void intttvc_d(const double* v, double voltet, const TetCtx& c) {
  double nv[4];
  for (int i = 0; i < 4; ++i) nv[i] = -v[i];
  int o[4];
  sort4(nv, o);
  double ww[4];
  for (int i = 0; i < 4; ++i) ww[i] = nv[o[i]];
  int inihis = -1, iedhis = -1, ix = 0;
  for (int ihis = 0; ihis < c.nwhis; ++ihis) {
    if (ix == 0 && ww[0] < c.frhis[ihis + 1]) { inihis = ihis; ix = 3; }
    if (ix == 3 && ww[3] < c.frhis[ihis + 1]) { iedhis = ihis; break; }
  }
  if (inihis < 0 || iedhis < 0) {                  // outside the histogram: the reference stops (rx)
    atomicExch(c.flag, 1);
    return;
  }
  const double norm = integtetn_d(ww, ww[3]);
  const double pvn = voltet / norm;
  double intega = 0.0;
  for (int ihis = inihis; ihis <= iedhis; ++ihis) {
    const double integb = (c.frhis[ihis + 1] > ww[3]) ? norm : integtetn_d(ww, c.frhis[ihis + 1]);
    const double add = pvn * (integb - intega) * c.fac;
    if (add != 0.0)
      for (int k = 0; k < 4; ++k) atomicAdd(c.out + ihis + c.stride_k * c.corner[k], add);
    intega = integb;
  }
}

__device__ void inttetrac_d(const double (*kk)[3], const double* xx, int i0, int i1, int i2, int i3,
                            const TetCtx& c) {
  const int it[4] = {i0, i1, i2, i3};
  double am[3][3];
  for (int d = 0; d < 3; ++d)
    for (int j = 0; j < 3; ++j) am[d][j] = kk[it[j]][d] - kk[it[3]][d];
  const double det = am[0][0] * (am[1][1] * am[2][2] - am[1][2] * am[2][1]) -
                     am[0][1] * (am[1][0] * am[2][2] - am[1][2] * am[2][0]) +
                     am[0][2] * (am[1][0] * am[2][1] - am[1][1] * am[2][0]);
  const double v[4] = {xx[i0], xx[i1], xx[i2], xx[i3]};
  intttvc_d(v, fabs(det / 6.0), c);
}

__device__ void mid_d(double (*kk)[3], const double* ee, double* xx, double* yy, int i, int j, int slot) {
  const double r = ee[i] / (ee[i] - ee[j]);
  for (int d = 0; d < 3; ++d) kk[slot][d] = kk[i][d] + r * (kk[j][d] - kk[i][d]);
  xx[slot] = xx[i] + r * (xx[j] - xx[i]);
  if (yy) yy[slot] = yy[i] + r * (yy[j] - yy[i]);
}

// inttetra6: the part of the sub-tetrahedron (corners it of the 8-point set) where eb > ef
__device__ void inttetra_d(const double (*kk8)[3], const double* xx8, const double* ebf8, int i0, int i1, int i2,
                           int i3, const TetCtx& c) {
  const int it[4] = {i0, i1, i2, i3};
  double ein[4];
  for (int i = 0; i < 4; ++i) ein[i] = ebf8[it[i]];
  int o[4];
  sort4(ein, o);
  double kk[8][3], ee[4], xx[8];
  for (int i = 0; i < 4; ++i) {
    for (int d = 0; d < 3; ++d) kk[i][d] = kk8[it[o[i]]][d];
    ee[i] = ein[o[i]];
    xx[i] = xx8[it[o[i]]];
  }
  if (0.0 >= ee[3]) return;
  if (ee[3] > 0.0 && 0.0 >= ee[2]) {               // Fig 1
    mid_d(kk, ee, xx, nullptr, 3, 1, 4); mid_d(kk, ee, xx, nullptr, 3, 0, 5); mid_d(kk, ee, xx, nullptr, 3, 2, 6);
    inttetrac_d(kk, xx, 3, 4, 5, 6, c);
  } else if (ee[2] > 0.0 && 0.0 >= ee[1]) {        // Fig 2
    mid_d(kk, ee, xx, nullptr, 3, 1, 4); mid_d(kk, ee, xx, nullptr, 3, 0, 5);
    mid_d(kk, ee, xx, nullptr, 2, 0, 6); mid_d(kk, ee, xx, nullptr, 2, 1, 7);
    inttetrac_d(kk, xx, 3, 2, 4, 5, c);
    inttetrac_d(kk, xx, 2, 5, 6, 4, c);
    inttetrac_d(kk, xx, 2, 4, 6, 7, c);
  } else if (ee[1] > 0.0 && 0.0 >= ee[0]) {        // Fig 3
    mid_d(kk, ee, xx, nullptr, 0, 3, 4); mid_d(kk, ee, xx, nullptr, 0, 1, 5); mid_d(kk, ee, xx, nullptr, 0, 2, 6);
    inttetrac_d(kk, xx, 2, 3, 6, 1, c);
    inttetrac_d(kk, xx, 3, 4, 5, 6, c);
    inttetrac_d(kk, xx, 3, 1, 5, 6, c);
  } else {                                         // Fig 4
    inttetrac_d(kk, xx, 0, 1, 2, 3, c);
  }
}

// One thread = one (tetrahedron, ib, jb).  ek, ekq: (nband, nk) column-major; qbzw: (3, nk).
__global__ void tetwt_hist_kernel(double* __restrict__ w, int nk, int nocc, int nunocc, int nwhis,
                                  const int* __restrict__ idtet, int ntet, const double* __restrict__ qbzw,
                                  const double* __restrict__ ek, const double* __restrict__ ekq, int nband,
                                  double efermi, const double* __restrict__ frhis, double fac,
                                  int* __restrict__ flag) {
  const long long tot = static_cast<long long>(ntet) * nocc * nunocc;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int jb = static_cast<int>(e % nunocc);
    const long long r = e / nunocc;
    const int ib = static_cast<int>(r % nocc);
    const int t = static_cast<int>(r / nocc);
    int kc[4];
    double ea[4], eb[4];
    double emin = 1e300, emax = -1e300, dmax = -1e300;
    for (int i = 0; i < 4; ++i) {
      kc[i] = idtet[4 * t + i];
      ea[i] = ek[ib + static_cast<long long>(nband) * kc[i]];
      eb[i] = ekq[jb + static_cast<long long>(nband) * kc[i]];
      emin = fmin(emin, ea[i]);
      emax = fmax(emax, eb[i]);
      dmax = fmax(dmax, eb[i] - ea[i]);
    }
    if (!(emin <= efermi && emax >= efermi) || dmax < 0.0) continue;        // tetwt5.f90:283-288
    TetCtx c;
    c.frhis = frhis;
    c.nwhis = nwhis;
    c.out = w + static_cast<long long>(nwhis) * (jb + static_cast<long long>(nunocc) * ib);
    c.stride_k = static_cast<long long>(nwhis) * nunocc * nocc;
    for (int i = 0; i < 4; ++i) c.corner[i] = kc[i];
    c.fac = fac;
    c.flag = flag;
    // lindtet6: corners in descending order of ea; the occupied part (ea < ef)
    int o[4];
    sort4(ea, o);
    double kk[8][3], ee[4], xx[8], ebf[8];
    for (int i = 0; i < 4; ++i) {
      const int s = o[3 - i];
      for (int d = 0; d < 3; ++d) kk[i][d] = qbzw[3 * kc[s] + d];
      ee[i] = ea[s] - efermi;
      xx[i] = 0.5 * (ea[s] - eb[s]);
      ebf[i] = eb[s] - efermi;
    }
    if (0.0 <= ee[3]) continue;
    if (ee[3] < 0.0 && 0.0 <= ee[2]) {               // Fig 1
      mid_d(kk, ee, xx, ebf, 3, 1, 4); mid_d(kk, ee, xx, ebf, 3, 0, 5); mid_d(kk, ee, xx, ebf, 3, 2, 6);
      inttetra_d(kk, xx, ebf, 3, 4, 5, 6, c);
    } else if (ee[2] < 0.0 && 0.0 <= ee[1]) {        // Fig 2
      mid_d(kk, ee, xx, ebf, 3, 1, 4); mid_d(kk, ee, xx, ebf, 3, 0, 5);
      mid_d(kk, ee, xx, ebf, 2, 0, 6); mid_d(kk, ee, xx, ebf, 2, 1, 7);
      inttetra_d(kk, xx, ebf, 3, 2, 4, 5, c);
      inttetra_d(kk, xx, ebf, 2, 5, 6, 4, c);
      inttetra_d(kk, xx, ebf, 2, 4, 6, 7, c);
    } else if (ee[1] < 0.0 && 0.0 <= ee[0]) {        // Fig 3
      mid_d(kk, ee, xx, ebf, 0, 3, 4); mid_d(kk, ee, xx, ebf, 0, 1, 5); mid_d(kk, ee, xx, ebf, 0, 2, 6);
      inttetra_d(kk, xx, ebf, 2, 3, 6, 1, c);
      inttetra_d(kk, xx, ebf, 3, 4, 5, 6, c);
      inttetra_d(kk, xx, ebf, 3, 1, 5, 6, c);
    } else {                                         // Fig 4
      inttetra_d(kk, xx, ebf, 0, 1, 2, 3, c);
    }
  }
}

static DevBuf g_tw_tab;

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_tetwt_hist_d(double* w_d, int nk, int nocc, int nunocc, int nwhis, const int* idtet, int ntet,
                                 const double* qbzw, const double* ek, const double* ekq, int nband, double efermi,
                                 const double* frhis, double* voltot) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(w_d && idtet && qbzw && ek && ekq && frhis, "tetwt_hist: null pointer");
  QSGW_ARG(nk >= 1 && nocc >= 1 && nunocc >= 1 && nwhis >= 1 && ntet >= 1 && nband >= nocc && nband >= nunocc,
           "tetwt_hist: nk=%d nocc=%d nunocc=%d nwhis=%d ntet=%d nband=%d", nk, nocc, nunocc, nwhis, ntet, nband);
  for (long long i = 0; i < 4LL * ntet; ++i)
    QSGW_ARG(idtet[i] >= 0 && idtet[i] < nk, "tetwt_hist: corner %lld = %d outside 0..%d", i, idtet[i], nk - 1);
  for (int i = 0; i < nwhis; ++i) QSGW_ARG(frhis[i] < frhis[i + 1], "tetwt_hist: bins not increasing at %d", i);
  // total volume of the tetrahedra (tetwt5x_dtet4 :200-206)
  double vt = 0.0;
  for (int t = 0; t < ntet; ++t) {
    double am[3][3];
    const double* k3 = qbzw + 3 * idtet[4 * t + 3];
    for (int j = 0; j < 3; ++j)
      for (int d = 0; d < 3; ++d) am[d][j] = qbzw[3 * idtet[4 * t + j] + d] - k3[d];
    vt += std::fabs((am[0][0] * (am[1][1] * am[2][2] - am[1][2] * am[2][1]) -
                     am[0][1] * (am[1][0] * am[2][2] - am[1][2] * am[2][0]) +
                     am[0][2] * (am[1][0] * am[2][1] - am[1][1] * am[2][0])) / 6.0);
  }
  QSGW_ARG(vt > 0.0, "tetwt_hist: the tetrahedra have no volume");
  if (voltot) *voltot = vt;
  cudaStream_t s = ctx().stream;
  const size_t bi = static_cast<size_t>(4) * ntet * sizeof(int);
  const size_t bq = static_cast<size_t>(3) * nk * sizeof(double), be = static_cast<size_t>(nband) * nk * sizeof(double);
  const size_t off_q = ((bi + 255) / 256) * 256, off_e = off_q + ((bq + 255) / 256) * 256;
  const size_t off_f = off_e + 2 * ((be + 255) / 256) * 256;
  rc = g_tw_tab.ensure(off_f + (nwhis + 1) * sizeof(double));
  if (rc) return rc;
  char* b = g_tw_tab.as<char>();
  if ((rc = h2d(b, idtet, bi, s))) return rc;
  if ((rc = h2d(b + off_q, qbzw, bq, s))) return rc;
  if ((rc = h2d(b + off_e, ek, be, s))) return rc;
  if ((rc = h2d(b + off_e + ((be + 255) / 256) * 256, ekq, be, s))) return rc;
  if ((rc = h2d(b + off_f, frhis, (nwhis + 1) * sizeof(double), s))) return rc;
  const long long tot = static_cast<long long>(ntet) * nocc * nunocc;
  const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((tot + 127) / 128, 64LL * ctx().sm_count)));
  tetwt_hist_kernel<<<grid, 128, 0, s>>>(w_d, nk, nocc, nunocc, nwhis, reinterpret_cast<const int*>(b), ntet,
                                         reinterpret_cast<const double*>(b + off_q),
                                         reinterpret_cast<const double*>(b + off_e),
                                         reinterpret_cast<const double*>(b + off_e + ((be + 255) / 256) * 256), nband,
                                         efermi, reinterpret_cast<const double*>(b + off_f), M_PI / (4.0 * vt),
                                         ctx().d_flags);
  count_launch();
  QSGW_LAUNCH_CHECK("tetwt_hist_kernel");
  return QSGW_OK;
}

// Pair/bin lists of x0gemm from the dense weights (host logic): the index
// accumulation of X0kf_v4hz_init (x0kf_v4h.f90:48-142) for npm = 1, no core
// states, no cRPA.  For every k (k-major, then occupied ib, then jb) the pair
// gets one entry when any of its bins has a nonzero weight: the contiguous bin
// range from its first to its last nonzero bin, with the weights of that range
// appended to whwc.  job 0 counts, job 1 fills (arrays of the counted sizes).
extern "C" int qsgw_x0_lists(const double* w, int nk, int nocc, int nunocc, int nwhis, int job, int* ncoun,
                             int* ncount, int* itc, int* itpc, int* jpmc, int* iwini, int* iwend, int* icouini,
                             double* whwc, int* icounkmin, int* icounkmax) {
  QSGW_ARG(w && ncoun && ncount && nk >= 1 && nocc >= 0 && nunocc >= 0 && nwhis >= 1 && (job == 0 || job == 1),
           "x0_lists: nk=%d nocc=%d nunocc=%d nwhis=%d job=%d", nk, nocc, nunocc, nwhis, job);
  const int cap_coun = *ncoun, cap_count = *ncount;
  QSGW_ARG(job == 0 || (itc && itpc && jpmc && iwini && iwend && icouini && whwc && icounkmin && icounkmax),
           "x0_lists: job 1 needs every output array");
  long long icoun = 0, icount = 0;
  for (int k = 0; k < nk; ++k) {
    if (job == 1) icounkmin[k] = static_cast<int>(icoun + 1);
    for (int ib = 0; ib < nocc; ++ib)
      for (int jb = 0; jb < nunocc; ++jb) {
        const double* wp = w + static_cast<size_t>(nwhis) * (jb + static_cast<size_t>(nunocc) * (ib + static_cast<size_t>(nocc) * k));
        int first = -1, last = -1;
        for (int h = 0; h < nwhis; ++h)
          if (wp[h] != 0.0) {
            if (first < 0) first = h;
            last = h;
          }
        if (first < 0) continue;
        if (job == 1) {
          QSGW_ARG(icoun < cap_coun && icount + (last - first + 1) <= cap_count,
                   "x0_lists: the job 1 arrays are smaller than job 0 counted");
          itc[icoun] = ib + 1;
          itpc[icoun] = jb + 1;
          jpmc[icoun] = 1;
          iwini[icoun] = first + 1;
          iwend[icoun] = last + 1;
          icouini[icoun] = static_cast<int>(icount + 1);
          for (int h = first; h <= last; ++h) whwc[icount + (h - first)] = wp[h];
        }
        ++icoun;
        icount += last - first + 1;
      }
    if (job == 1) icounkmax[k] = static_cast<int>(icoun);
  }
  QSGW_ARG(icount <= 2147483647LL, "x0_lists: %lld weights exceed the int range", icount);
  *ncoun = static_cast<int>(icoun);
  *ncount = static_cast<int>(icount);
  return QSGW_OK;
}

// Degenerate groups of chkdgn (tetwt5.f90:868-912): a new group wherever two neighbouring levels
// differ by more than 1e-4; start[g] .. start[g+1]-1 is group g.
static void degenerate_groups(const double* e, int n, std::vector<int>& start) {
  start.clear();
  if (n < 1) return;
  start.push_back(0);
  for (int i = 1; i < n; ++i)
    if (std::fabs(e[i] - e[i - 1]) > 1e-4) start.push_back(i);
  start.push_back(n);
}

extern "C" int qsgw_tetwt_symmetrize(double* w, int nk, int nocc, int nunocc, int nwhis, const double* ek,
                                     const double* ekq, int nband) {
  QSGW_ARG(w && ek && ekq && nk >= 1 && nocc >= 0 && nunocc >= 0 && nwhis >= 1 && nband >= nocc && nband >= nunocc,
           "tetwt_symmetrize: nk=%d nocc=%d nunocc=%d nwhis=%d nband=%d", nk, nocc, nunocc, nwhis, nband);
  std::vector<int> ga, gb;
  std::vector<double> acc(nwhis);
  const size_t pair = static_cast<size_t>(nwhis);
  for (int k = 0; k < nk; ++k) {
    degenerate_groups(ek + static_cast<size_t>(nband) * k, nocc, ga);
    degenerate_groups(ekq + static_cast<size_t>(nband) * k, nunocc, gb);
    double* wk = w + pair * nunocc * nocc * k;
    for (size_t a = 0; a + 1 < ga.size(); ++a)
      for (size_t b = 0; b + 1 < gb.size(); ++b) {
        const int i0 = ga[a], i1 = ga[a + 1], j0 = gb[b], j1 = gb[b + 1];
        const int cnt = (i1 - i0) * (j1 - j0);
        if (cnt == 1) continue;
        // tetwt5.f90:403-423: the block's histograms summed ib-major, then divided by its size
        std::fill(acc.begin(), acc.end(), 0.0);
        for (int ib = i0; ib < i1; ++ib)
          for (int jb = j0; jb < j1; ++jb) {
            const double* p = wk + pair * (jb + static_cast<size_t>(nunocc) * ib);
            for (int h = 0; h < nwhis; ++h) acc[h] = acc[h] + p[h];
          }
        for (int h = 0; h < nwhis; ++h) acc[h] = acc[h] / cnt;
        for (int ib = i0; ib < i1; ++ib)
          for (int jb = j0; jb < j1; ++jb)
            std::copy(acc.begin(), acc.end(), wk + pair * (jb + static_cast<size_t>(nunocc) * ib));
      }
  }
  return QSGW_OK;
}
