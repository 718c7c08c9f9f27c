// A C++ caller of libqsgw_b200 written the way a Fortran or C host would use it:
// plain pointers to column-major complex(8) arrays, status codes, no torch.
//   cabi_caller          checks that calls before qsgw_init fail cleanly and builds x0gemm
//                        pair/bin lists with the host-only qsgw_x0_lists, and writes and
//                        reads a __Vcoud file (no GPU needed)
//   cabi_caller gpu      also multiplies Fortran-layout matrices with qsgw_zmm (host
//                        pointers, op(A) = A^H) and compares with a plain triple loop
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "qsgw_b200.h"

typedef std::complex<double> cd;

static int fail(const char* what) {
  char msg[512];
  qsgw_last_error(msg, sizeof(msg));
  std::printf("FAIL %s: %s\n", what, msg);
  return 1;
}

int main(int argc, char** argv) {
  // before init: every entry point returns QSGW_ERR_NOTINIT and sets a message
  double dummy[2] = {0, 0};
  if (qsgw_zmm(dummy, dummy, dummy, 1, 1, 1, 0, 0, dummy, dummy, 1, 1, 1) != QSGW_ERR_NOTINIT)
    return fail("qsgw_zmm before init");
  char msg[256];
  qsgw_last_error(msg, sizeof(msg));
  if (std::strstr(msg, "qsgw_init") == nullptr) return fail("error text");
  {
    // host-only: x0gemm pair/bin lists from dense tetrahedron weights w(ihis, jb, ib, k)
    const int nk = 2, nocc = 2, nunocc = 2, nwhis = 4;
    std::vector<double> w(static_cast<size_t>(nwhis) * nunocc * nocc * nk, 0.0);
    auto W = [&](int h, int jb, int ib, int k) -> double& { return w[h + nwhis * (jb + nunocc * (ib + nocc * k))]; };
    W(1, 0, 1, 0) = 0.5;                      // k = 1: pair (it = 2, itp = 1), bins 2..4 with a hole at 3
    W(3, 0, 1, 0) = 0.25;
    W(0, 1, 0, 1) = 1.0;                      // k = 2: pair (it = 1, itp = 2), bin 1
    int ncoun = 0, ncount = 0;
    if (qsgw_x0_lists(w.data(), nk, nocc, nunocc, nwhis, 0, &ncoun, &ncount, nullptr, nullptr, nullptr, nullptr,
                      nullptr, nullptr, nullptr, nullptr, nullptr) != QSGW_OK || ncoun != 2 || ncount != 4)
      return fail("qsgw_x0_lists job 0");
    std::vector<int> itc(ncoun), itpc(ncoun), jpmc(ncoun), iwini(ncoun), iwend(ncoun), icouini(ncoun), kmin(nk), kmax(nk);
    std::vector<double> whwc(ncount);
    if (qsgw_x0_lists(w.data(), nk, nocc, nunocc, nwhis, 1, &ncoun, &ncount, itc.data(), itpc.data(), jpmc.data(),
                      iwini.data(), iwend.data(), icouini.data(), whwc.data(), kmin.data(), kmax.data()) != QSGW_OK)
      return fail("qsgw_x0_lists job 1");
    const bool ok = itc[0] == 2 && itpc[0] == 1 && iwini[0] == 2 && iwend[0] == 4 && icouini[0] == 1 &&
                    itc[1] == 1 && itpc[1] == 2 && iwini[1] == 1 && iwend[1] == 1 && icouini[1] == 4 &&
                    jpmc[0] == 1 && jpmc[1] == 1 && whwc[0] == 0.5 && whwc[1] == 0.0 && whwc[2] == 0.25 &&
                    whwc[3] == 1.0 && kmin[0] == 1 && kmax[0] == 1 && kmin[1] == 2 && kmax[1] == 2;
    if (!ok) return fail("qsgw_x0_lists tables");
  }
  {
    // host-only: the Hilbert transform matrix; chi0(i w) of one bin of weight 1 is b(bin, j)
    const int nwhis = 6, niw = 2, nw = 2;
    const double frhis[nwhis + 1] = {0.0, 0.01, 0.03, 0.06, 0.1, 0.15, 0.21};
    const double freq_i[niw] = {0.05, 0.5}, freq_r[nw + 1] = {0.0, 0.005, 0.02};
    std::vector<cd> b(static_cast<size_t>(nwhis + 1) * (niw + nw + 1));
    if (qsgw_dpsion_matrix(nwhis, frhis, niw, freq_i, nw, freq_r, 1e10, 0.0, reinterpret_cast<double*>(b.data())) !=
        QSGW_OK)
      return fail("qsgw_dpsion_matrix");
    // a positive weight (x0gemm's sign) gives chi0(i w) < 0, decreasing in magnitude with w
    const cd c0 = b[3 + 0 * (nwhis + 1)], c1 = b[3 + 1 * (nwhis + 1)];
    if (!(c0.real() < 0.0 && c1.real() < 0.0 && std::abs(c1) < std::abs(c0) && c0.imag() == 0.0))
      return fail("qsgw_dpsion_matrix values");
    if (qsgw_dpsion_matrix(nwhis, frhis, niw, freq_i, nwhis, freq_r, 1e10, 0.0,
                           reinterpret_cast<double*>(b.data())) != QSGW_ERR_ARG)   // nw >= nwhis
      return fail("qsgw_dpsion_matrix argument check");
  }
  {
    // host-only: a __Vcoud file written and read back beside this executable
    const std::string path = std::string(argv[0]) + ".Vcoud.1";
    const int ngb = 5;
    const double q[3] = {0.125, -0.25, 0.5};
    std::vector<double> v(ngb);
    std::vector<cd> z(static_cast<size_t>(ngb) * ngb);
    for (int i = 0; i < ngb; ++i) v[i] = 0.5 + i * i;
    for (size_t i = 0; i < z.size(); ++i) z[i] = cd(std::cos(0.7 * i), std::sin(0.3 * i));
    if (qsgw_vcoud_write(path.c_str(), ngb, q, v.data(), reinterpret_cast<const double*>(z.data())) != QSGW_OK)
      return fail("qsgw_vcoud_write");
    int n = 0;
    double q2[3];
    std::vector<double> v2(ngb), vs(ngb);
    std::vector<cd> z2(z.size());
    if (qsgw_vcoud_read(path.c_str(), ngb, &n, q2, v2.data(), vs.data(), reinterpret_cast<double*>(z2.data())) !=
        QSGW_OK)
      return fail("qsgw_vcoud_read");
    bool ok = n == ngb && q2[0] == q[0] && q2[1] == q[1] && q2[2] == q[2] && v2 == v && z2 == z;
    for (int i = 0; i < ngb; ++i) ok = ok && vs[i] == std::sqrt(v[i]);
    if (!ok) return fail("qsgw_vcoud_read values");
    if (qsgw_vcoud_read(path.c_str(), ngb - 1, &n, q2, v2.data(), nullptr, nullptr) != QSGW_ERR_ARG)
      return fail("qsgw_vcoud_read capacity check");
    std::remove(path.c_str());
  }
  if (argc < 2 || std::strcmp(argv[1], "gpu") != 0) {
    std::printf("OK cpu\n");
    return 0;
  }
  if (qsgw_init(0) != QSGW_OK) return fail("qsgw_init");
  const int m = 37, n = 29, k = 41, lda = k + 3, ldb = k + 1, ldc = m + 2;
  std::vector<cd> a(static_cast<size_t>(lda) * m), b(static_cast<size_t>(ldb) * n), c(static_cast<size_t>(ldc) * n);
  unsigned s = 12345u;
  auto rnd = [&]() { s = s * 1664525u + 1013904223u; return (s >> 8) / 16777216.0 - 0.5; };
  for (auto& x : a) x = cd(rnd(), rnd());
  for (auto& x : b) x = cd(rnd(), rnd());
  for (auto& x : c) x = cd(rnd(), rnd());
  std::vector<cd> ref = c;
  const cd alpha(0.5, -1.25), beta(2.0, 0.5);
  // C = alpha A^H B + beta C, A stored (k x m), column-major
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      cd acc = 0;
      for (int l = 0; l < k; ++l) acc += std::conj(a[l + static_cast<size_t>(lda) * i]) * b[l + static_cast<size_t>(ldb) * j];
      ref[i + static_cast<size_t>(ldc) * j] = alpha * acc + beta * c[i + static_cast<size_t>(ldc) * j];
    }
  const double al[2] = {alpha.real(), alpha.imag()}, be[2] = {beta.real(), beta.imag()};
  if (qsgw_zmm(reinterpret_cast<double*>(a.data()), reinterpret_cast<double*>(b.data()),
               reinterpret_cast<double*>(c.data()), m, n, k, 2, 0, al, be, lda, ldb, ldc) != QSGW_OK)
    return fail("qsgw_zmm");
  double num = 0, den = 0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      num += std::norm(c[i + static_cast<size_t>(ldc) * j] - ref[i + static_cast<size_t>(ldc) * j]);
      den += std::norm(ref[i + static_cast<size_t>(ldc) * j]);
    }
  const double rel = std::sqrt(num / den);
  qsgw_finalize();
  if (!(rel <= 1e-13)) {
    std::printf("FAIL relative error %.3e\n", rel);
    return 1;
  }
  std::printf("OK gpu %.3e\n", rel);
  return 0;
}
