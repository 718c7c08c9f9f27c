// Hilbert transform of the chi0 histogram: drop-in for dpsion_init +
// dpsion_chiq (dpsion5.f90:77-137, 174-292) with time reversal (npm = 1),
// no chi+-, with the optional SmearX0 Gaussian filter.
//
// x0gemm leaves rcxq(npr, npr_col, 0:nwhis) = spectral weights on the
// histogram bins [frhis(i), frhis(i+1)].  The reference normalises the bins
// in place (rcxq <- -wfac / (R - L) rcxq, :215-220), then
//     chi0(i w_j)   = sum_i rcxq(i) imatt(j, i)                 (:229, one GEMM)
//     chi0(w_r(t))  = i rcxq(t) + sum_i rcxq(i) rmatt(t, i)     (:243-257)
// with imatt, rmatt from hilbertmat (hilbertmat.f90:14-79, FP64 logs).  Here
// the normalisation and the i rcxq(t) term are folded into one small complex
// matrix B (slots 0..nwhis x [niw imaginary | nw+1 real] columns), built on
// the host in FP64 as the reference's dpsion_init builds its matrices, and
// the N^2-sized work is two passes of the DMMA GEMM over rcxq:
//     zxqi = rcxq . B[:, imag],   zxq = rcxq . B[:, real].
// rcxq is not modified (the reference leaves chi0(w_r) in rcxq(:, :, 0:nw);
// here it goes to zxq).
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <complex>
#include <vector>
#include "zgemm_f64.cuh"

namespace qsgw {
namespace {

using cd = std::complex<double>;

// int_a^b (m w + n) / (w - z) dw = m facm + n facn  (hilbertmat.f90:57-69)
void hm2(cd z, double a, double b, cd& facm, cd& facn) {
  const cd db = z - b, da = z - a;
  facm = facn = cd(0.0, 0.0);
  if (std::abs(da) > 1e-8 && std::abs(db) > 1e-8) {
    facn = std::log(db / da);
    facm = z * facn + (b - a);
  }
}

// rmat over bins -nwhis..nwhis (index i + nwhis): H(z) = sum rmat(i) f(i) for f linear between
// the bin centres, zero at w = 0 and at the outer edges (hilbertmat.f90:14-56)
void hilbertmat_h(cd z, int nwhis, const std::vector<double>& L, const std::vector<double>& C,
                  const std::vector<double>& R, std::vector<cd>& rmat) {
  rmat.assign(2 * nwhis + 1, cd(0.0, 0.0));
  const cd zz = z + cd(0.0, 1e-13);
  cd facm, facn;
  for (int iw = -nwhis; iw <= nwhis; ++iw) {
    if (iw == 0) continue;
    const int k = iw + nwhis;
    const double ci = C[k];
    const double cim = (iw == -nwhis) ? L[k] : (iw == 1 ? 0.0 : C[k - 1]);
    hm2(zz, L[k], C[k], facm, facn);
    rmat[k] += (facm - facn * cim) / (ci - cim);
    if (iw != -nwhis && iw != 1) rmat[k - 1] += (-facm + facn * ci) / (ci - cim);
    const double cip = (iw == nwhis) ? R[k] : (iw == -1 ? 0.0 : C[k + 1]);
    hm2(zz, C[k], R[k], facm, facn);
    rmat[k] += (-facm + facn * cip) / (cip - ci);
    if (iw != nwhis && iw != -1) rmat[k + 1] += (facm - facn * ci) / (cip - ci);
  }
}

// The transform matrix B (rows = rcxq slots 0..nwhis, columns = niw imaginary then nw+1 real
// frequencies, column-major): imatt and rmatt of dpsion_init (dpsion5.f90:93-107, 123-128) with
// the bin normalisation -wfac / (R - L) (:215-220) and the i rcxq(t) term (:255) folded in.
void build_transform(int nwhis, const double* frhis, int niw, const double* freq_i, int nw, const double* freq_r,
                     double ecut, double smear, std::vector<cd>& B) {
  // bins -nwhis..nwhis (dpsion5.f90:87-89)
  std::vector<double> L(2 * nwhis + 1), R(2 * nwhis + 1), C(2 * nwhis + 1);
  for (int i = 1; i <= nwhis; ++i) {
    L[nwhis + i] = frhis[i - 1];
    R[nwhis + i] = frhis[i];
    L[nwhis - i] = -frhis[i];
    R[nwhis - i] = -frhis[i - 1];
  }
  L[nwhis] = R[nwhis] = 0.0;
  for (int k = 0; k <= 2 * nwhis; ++k) C[k] = 0.5 * (L[k] + R[k]);
  // bin normalisation (dpsion5.f90:215-220)
  std::vector<double> fnorm(nwhis + 1, 1.0);
  for (int i = 1; i <= nwhis; ++i) {
    const double c = C[nwhis + i];
    const double wfac = (ecut < 1e9) ? std::exp(-(c / ecut) * (c / ecut)) : 1.0;
    fnorm[i] = -wfac / (R[nwhis + i] - L[nwhis + i]);
  }
  // B: rows = rcxq slots 0..nwhis, columns = niw imaginary then nw+1 real frequencies
  const int K = nwhis + 1, ncol = niw + (nw + 1);
  B.assign(static_cast<size_t>(K) * ncol, cd(0.0, 0.0));
  std::vector<cd> rm;
  const double pi = 3.14159265358979323846;
  for (int j = 0; j < niw; ++j) {                  // imatt (dpsion5.f90:123-128)
    hilbertmat_h(cd(0.0, freq_i[j]), nwhis, L, C, R, rm);
    for (int i = 1; i <= nwhis; ++i)
      B[static_cast<size_t>(j) * K + i] = fnorm[i] * (std::real(rm[nwhis + i] - rm[nwhis - i]) / pi);
  }
  for (int t = 0; t <= nw; ++t) {                  // rmatt (dpsion5.f90:93-107) and i rcxq(t) (:255)
    hilbertmat_h(cd(freq_r[t], 0.0), nwhis, L, C, R, rm);
    cd* col = B.data() + static_cast<size_t>(niw + t) * K;
    for (int i = 1; i <= nwhis; ++i)
      col[i] = fnorm[i] * (std::real(rm[nwhis + i]) / pi - std::real(rm[nwhis - i]) / pi);
    col[t] += cd(0.0, fnorm[t]);                   // slot 0 is not normalised: fnorm[0] = 1
  }
  // SmearX0 (dpsion5.f90:174-193): rcxq(bins) <- rcxq(bins) . gfmat^T before the normalisation,
  // folded in as B(bins, :) <- gfmat^T B(bins, :); gfmat(j, i) = exp(-(c_i - c_j)^2 / (2 smear^2))
  // normalised over j (gaussianfilterhis, :459-483)
  if (std::fabs(smear) > 1e-15) {
    std::vector<double> c(nwhis), g(static_cast<size_t>(nwhis) * nwhis);
    for (int i = 0; i < nwhis; ++i) c[i] = 0.5 * (frhis[i] + frhis[i + 1]);
    for (int i = 0; i < nwhis; ++i) {
      double sum = 0.0;
      for (int j = 0; j < nwhis; ++j) {
        const double d = c[i] - c[j];
        g[j + static_cast<size_t>(nwhis) * i] = std::exp(-d * d / (2.0 * smear * smear));
        sum += g[j + static_cast<size_t>(nwhis) * i];
      }
      for (int j = 0; j < nwhis; ++j) g[j + static_cast<size_t>(nwhis) * i] /= sum;
    }
    std::vector<cd> tmp(nwhis);
    for (int col = 0; col < ncol; ++col) {
      cd* bc = B.data() + static_cast<size_t>(col) * K;
      for (int k = 0; k < nwhis; ++k) {          // new row k+1 = sum_b gfmat(b, k) old row b+1
        cd acc(0.0, 0.0);
        for (int b = 0; b < nwhis; ++b) acc += g[b + static_cast<size_t>(nwhis) * k] * bc[b + 1];
        tmp[k] = acc;
      }
      for (int k = 0; k < nwhis; ++k) bc[k + 1] = tmp[k];
    }
  }
}

}  // namespace

static DevBuf g_dp_b;

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_dpsion_chiq_d(const double* rcxq, int npr, int npr_col, int nwhis, const double* frhis,
                                  int niw, const double* freq_i, int nw, const double* freq_r, double ecut,
                                  double smearx0, double* zxqi, double* zxq) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(rcxq && frhis && npr >= 1 && npr_col >= 1 && nwhis >= 1 && niw >= 0 && nw >= -1,
           "dpsion_chiq: npr=%d npr_col=%d nwhis=%d niw=%d nw=%d", npr, npr_col, nwhis, niw, nw);
  QSGW_ARG(niw == 0 || (zxqi && freq_i), "dpsion_chiq: niw=%d needs zxqi and freq_i", niw);
  QSGW_ARG(nw < 0 || (zxq && freq_r), "dpsion_chiq: nw=%d needs zxq and freq_r", nw);
  // dpsion5.f90:208-209
  QSGW_ARG(nw < nwhis, "dpsion_chiq: nwhis=%d <= nw=%d", nwhis, nw);
  QSGW_ARG(nw < 0 || freq_r[0] == 0.0, "dpsion_chiq: freq_r(0) = %g, must be 0", nw < 0 ? 0.0 : freq_r[0]);
  QSGW_ARG(frhis[0] >= 0.0, "dpsion_chiq: frhis(1) = %g < 0", frhis[0]);
  for (int i = 0; i < nwhis; ++i)
    QSGW_ARG(frhis[i + 1] > frhis[i], "dpsion_chiq: frhis not increasing at bin %d", i + 1);
  const long long M = static_cast<long long>(npr) * npr_col;
  QSGW_ARG(M <= INT_MAX, "dpsion_chiq: npr*npr_col = %lld too large", M);
  QSGW_ARG(((reinterpret_cast<uintptr_t>(rcxq) | reinterpret_cast<uintptr_t>(zxqi) |
             reinterpret_cast<uintptr_t>(zxq)) & 15) == 0, "dpsion_chiq: complex arrays must be 16-byte aligned");
  std::vector<cd> B;
  build_transform(nwhis, frhis, niw, freq_i, nw, freq_r, ecut, smearx0, B);
  const int K = nwhis + 1;
  cudaStream_t s = ctx().stream;
  rc = g_dp_b.ensure(B.size() * sizeof(cd));
  if (rc) return rc;
  if ((rc = h2d(g_dp_b.p, B.data(), B.size() * sizeof(cd), s))) return rc;
  const double2* A = reinterpret_cast<const double2*>(rcxq);
  const double2* Bd = g_dp_b.as<double2>();
  const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
  if (niw > 0) {
    rc = zgemm_f64(0, 0, static_cast<int>(M), niw, K, one, A, M, 0, Bd, K, 0, zero,
                   reinterpret_cast<double2*>(zxqi), M, 0, 1, s);
    if (rc) return rc;
  }
  if (nw >= 0) {
    rc = zgemm_f64(0, 0, static_cast<int>(M), nw + 1, K, one, A, M, 0, Bd + static_cast<size_t>(niw) * K, K, 0, zero,
                   reinterpret_cast<double2*>(zxq), M, 0, 1, s);
    if (rc) return rc;
  }
  return QSGW_OK;
}

extern "C" int qsgw_dpsion_matrix(int nwhis, const double* frhis, int niw, const double* freq_i, int nw,
                                  const double* freq_r, double ecut, double smearx0, double* b) {
  QSGW_ARG(frhis && b && nwhis >= 1 && niw >= 0 && nw >= -1 && nw < nwhis,
           "dpsion_matrix: nwhis=%d niw=%d nw=%d", nwhis, niw, nw);
  QSGW_ARG(niw == 0 || freq_i, "dpsion_matrix: niw=%d needs freq_i", niw);
  QSGW_ARG(nw < 0 || (freq_r && freq_r[0] == 0.0), "dpsion_matrix: freq_r must start at 0");
  for (int i = 0; i < nwhis; ++i)
    QSGW_ARG(frhis[i + 1] > frhis[i], "dpsion_matrix: frhis not increasing at bin %d", i + 1);
  std::vector<cd> B;
  build_transform(nwhis, frhis, niw, freq_i, nw, freq_r, ecut, smearx0, B);
  std::copy(B.begin(), B.end(), reinterpret_cast<cd*>(b));
  return QSGW_OK;
}
