// Hermitian eigensolver on the GPU in FP64: the Coulomb-matrix
// diagonalisation that feeds v^1/2 and the E basis (main_hvccfp0.f90:322-367,
// zhgv_d / zhgv_h in m_lapack.f90:64-104, 203-229).
//
// Parallel cyclic two-sided Jacobi: each step applies N/2 disjoint plane
// rotations chosen by a round-robin tournament ordering; a sweep is N-1
// steps.  Per step three small kernels: the 2x2 angles, the column update
// A <- A J (and V <- V J), the row update A <- J^H A.  The complex
// rotation first removes the phase of a_pq, then applies the real Jacobi
// rotation with t = sgn(tau) / (|tau| + sqrt(1 + tau^2)).  Sweeps stop when
// the off-diagonal norm is below 1e-14 of the Frobenius norm.
// The generalised problem (-v) z = lambda O z is reduced with O^-1/2 built
// from a Jacobi solve of O.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>
#include "zgemm_f64.cuh"

namespace qsgw {

struct Rot {
  int p, q;
  double c, s;        // real rotation
  double2 ph;         // e^{-i phi}, b = a_pq = |b| e^{i phi}
};

__device__ __forceinline__ void pair_of(int t, int k, int ne, int& p, int& q) {
  // round-robin: player ne-1 fixed, the others rotate
  if (k == 0) { p = ne - 1; q = t; }
  else { p = (t + k) % (ne - 1); q = (t - k + (ne - 1)) % (ne - 1); }
  if (p > q) { const int x = p; p = q; q = x; }
}

__global__ void jacobi_angles_kernel(const double2* __restrict__ A, long long lda, int n, int ne, int t,
                                     Rot* __restrict__ rot) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne / 2) return;
  int p, q;
  pair_of(t, k, ne, p, q);
  Rot r{p, q, 1.0, 0.0, make_double2(1.0, 0.0)};
  if (q < n) {
    const double a = A[p + p * lda].x, d = A[q + q * lda].x;
    const double2 b = A[p + q * lda];
    const double ab = hypot(b.x, b.y);
    if (ab > 1e-300 && ab > 1e-18 * sqrt(fabs(a * d))) {
      const double tau = (d - a) / (2.0 * ab);
      const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
      r.c = 1.0 / sqrt(1.0 + tt * tt);
      r.s = tt * r.c;
      r.ph = make_double2(b.x / ab, -b.y / ab);
    }
  }
  rot[k] = r;
}

// A <- A J and V <- V J on columns (p, q):
//   col_p' = c col_p - s e^{-i phi} col_q,   col_q' = s col_p + c e^{-i phi} col_q
__global__ void jacobi_cols_kernel(double2* __restrict__ A, long long lda, double2* __restrict__ V, long long ldv,
                                   int n, int npair, const Rot* __restrict__ rot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (i >= n || k >= npair) return;
  const Rot r = rot[k];
  if (r.q >= n || r.s == 0.0) return;
  double2* M[2] = {A, V};
  const long long ld[2] = {lda, ldv};
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    double2& xp = M[m][i + r.p * ld[m]];
    double2& xq = M[m][i + r.q * ld[m]];
    const double2 a = xp, b = xq;
    const double2 eb = make_double2(r.ph.x * b.x - r.ph.y * b.y, r.ph.x * b.y + r.ph.y * b.x);
    xp = make_double2(r.c * a.x - r.s * eb.x, r.c * a.y - r.s * eb.y);
    xq = make_double2(r.s * a.x + r.c * eb.x, r.s * a.y + r.c * eb.y);
  }
}

// A <- J^H A on rows (p, q):
//   row_p' = c row_p - s e^{i phi} row_q,   row_q' = s row_p + c e^{i phi} row_q
__global__ void jacobi_rows_kernel(double2* __restrict__ A, long long lda, int n, int npair,
                                   const Rot* __restrict__ rot) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (j >= n || k >= npair) return;
  const Rot r = rot[k];
  if (r.q >= n || r.s == 0.0) return;
  double2& xp = A[r.p + j * lda];
  double2& xq = A[r.q + j * lda];
  const double2 a = xp, b = xq;
  const double2 cph = make_double2(r.ph.x, -r.ph.y);
  const double2 eb = make_double2(cph.x * b.x - cph.y * b.y, cph.x * b.y + cph.y * b.x);
  xp = make_double2(r.c * a.x - r.s * eb.x, r.c * a.y - r.s * eb.y);
  xq = make_double2(r.s * a.x + r.c * eb.x, r.s * a.y + r.c * eb.y);
}

// off-diagonal and total squared norms -> out[0], out[1]
__global__ void offdiag_norm_kernel(const double2* __restrict__ A, long long lda, int n, double* out) {
  double off = 0.0, tot = 0.0;
  const long long nn = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nn;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    const double2 v = A[i + j * lda];
    const double m = v.x * v.x + v.y * v.y;
    tot += m;
    if (i != j) off += m;
  }
  for (int o = 16; o; o >>= 1) {
    off += __shfl_xor_sync(0xffffffffu, off, o);
    tot += __shfl_xor_sync(0xffffffffu, tot, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(out, off); atomicAdd(out + 1, tot); }
}

__global__ void set_identity_kernel(double2* V, long long ldv, int n) {
  const long long nn = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nn;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    V[i + j * ldv] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
}

__global__ void diag_kernel(const double2* A, long long lda, int n, double* d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = A[i + i * lda].x;
}

// out(:, j) = V(:, perm[j]) * colscale[j]
__global__ void permute_cols_kernel(double2* __restrict__ out, long long ldo, const double2* __restrict__ V,
                                    long long ldv, int n, const int* __restrict__ perm) {
  const long long nn = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nn;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    out[i + j * ldo] = V[i + static_cast<long long>(perm[j]) * ldv];
  }
}

// M(:, j) *= f[j]
__global__ void scale_cols_kernel(double2* M, long long ld, int n, const double* f) {
  const long long nn = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nn;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    double2& v = M[i + j * ld];
    v.x *= f[j]; v.y *= f[j];
  }
}

static DevBuf g_jc_rot, g_jc_norm, g_jc_d, g_jc_v, g_jc_w, g_jc_x, g_jc_perm;

static int grid_for(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 16LL * ctx().sm_count)));
}

// In place: A (n x n Hermitian) -> diagonal; V (n x n) <- eigenvectors; d <- unsorted eigenvalues (host).
static int jacobi_solve(double2* A, long long lda, double2* V, int n, std::vector<double>& d, cudaStream_t s) {
  const int ne = n + (n & 1);
  const int npair = ne / 2;
  int rc = g_jc_rot.ensure(npair * sizeof(Rot));
  if (rc) return rc;
  rc = g_jc_norm.ensure(2 * sizeof(double));
  if (rc) return rc;
  rc = g_jc_d.ensure(n * sizeof(double));
  if (rc) return rc;
  Rot* rot = g_jc_rot.as<Rot>();
  set_identity_kernel<<<grid_for(static_cast<long long>(n) * n), 256, 0, s>>>(V, n, n);
  count_launch();
  bool converged = (n <= 1);
  for (int sweep = 0; sweep < 40 && !converged; ++sweep) {
    for (int t = 0; t < ne - 1; ++t) {
      jacobi_angles_kernel<<<(npair + 127) / 128, 128, 0, s>>>(A, lda, n, ne, t, rot);
      jacobi_cols_kernel<<<dim3((n + 127) / 128, npair), 128, 0, s>>>(A, lda, V, n, n, npair, rot);
      jacobi_rows_kernel<<<dim3((n + 127) / 128, npair), 128, 0, s>>>(A, lda, n, npair, rot);
      count_launch(3);
    }
    QSGW_LAUNCH_CHECK("jacobi sweep");
    QSGW_CUDA(cudaMemsetAsync(g_jc_norm.p, 0, 2 * sizeof(double), s));
    offdiag_norm_kernel<<<grid_for(static_cast<long long>(n) * n), 256, 0, s>>>(A, lda, n, g_jc_norm.as<double>());
    count_launch();
    double h[2] = {0.0, 0.0};
    QSGW_CUDA(cudaMemcpyAsync(h, g_jc_norm.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    QSGW_CUDA(cudaStreamSynchronize(s));
    if (!std::isfinite(h[0]) || !std::isfinite(h[1])) {
      set_error("zhegv: non-finite matrix entries");
      return QSGW_ERR_NUMERIC;
    }
    converged = h[0] <= 1e-28 * h[1];
  }
  if (!converged) {
    set_error("zhegv: Jacobi sweeps did not converge");
    return QSGW_ERR_NUMERIC;
  }
  diag_kernel<<<(n + 127) / 128, 128, 0, s>>>(A, lda, n, g_jc_d.as<double>());
  count_launch();
  d.resize(n);
  QSGW_CUDA(cudaMemcpyAsync(d.data(), g_jc_d.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  return QSGW_OK;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_zhegv_d(double* v_d, const double* o_d, int n, int lda, double* vcoud) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(v_d && vcoud && n >= 1 && lda >= n, "zhegv: n=%d lda=%d", n, lda);
  cudaStream_t s = ctx().stream;
  const long long nn = static_cast<long long>(n) * n;
  rc = g_jc_v.ensure(nn * sizeof(double2));
  if (rc) return rc;
  rc = g_jc_w.ensure(nn * sizeof(double2));
  if (rc) return rc;
  double2* V = g_jc_v.as<double2>();
  double2* W = g_jc_w.as<double2>();
  double2* A = reinterpret_cast<double2*>(v_d);
  double2* Oh = nullptr;                         // O^-1/2 when an overlap is given
  if (o_d) {
    rc = g_jc_x.ensure(2 * nn * sizeof(double2));
    if (rc) return rc;
    double2* X = g_jc_x.as<double2>();           // working copy of O, then O^-1/2
    double2* Y = X + nn;
    QSGW_CUDA(cudaMemcpy2DAsync(X, n * sizeof(double2), o_d, lda * sizeof(double2), n * sizeof(double2), n,
                                cudaMemcpyDeviceToDevice, s));
    std::vector<double> mu;
    rc = jacobi_solve(X, n, V, n, mu, s);
    if (rc) return rc;
    std::vector<double> f(n);
    for (int j = 0; j < n; ++j) {
      if (!(mu[j] > 0.0)) {
        set_error("zhegv: overlap matrix is not positive definite");
        return QSGW_ERR_NUMERIC;
      }
      f[j] = 1.0 / std::sqrt(mu[j]);
    }
    rc = g_jc_d.ensure(n * sizeof(double));
    if (rc) return rc;
    QSGW_CUDA(cudaMemcpyAsync(g_jc_d.p, f.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    // Y = U diag(mu^-1/2), X = Y U^H = O^-1/2
    QSGW_CUDA(cudaMemcpyAsync(Y, V, nn * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    scale_cols_kernel<<<grid_for(nn), 256, 0, s>>>(Y, n, n, g_jc_d.as<double>());
    count_launch();
    rc = zgemm_f64(0, 2, n, n, n, make_double2(1, 0), Y, n, 0, V, n, 0, make_double2(0, 0), X, n, 0, 1, s);
    if (rc) return rc;
    // A <- O^-1/2 v O^-1/2
    rc = zgemm_f64(0, 0, n, n, n, make_double2(1, 0), A, lda, 0, X, n, 0, make_double2(0, 0), W, n, 0, 1, s);
    if (rc) return rc;
    rc = zgemm_f64(0, 0, n, n, n, make_double2(1, 0), X, n, 0, W, n, 0, make_double2(0, 0), A, lda, 0, 1, s);
    if (rc) return rc;
    Oh = X;
  }
  std::vector<double> lam;
  rc = jacobi_solve(A, lda, V, n, lam, s);
  if (rc) return rc;
  // descending eigenvalues of v = ascending eigenvalues of -v (main_hvccfp0.f90:339, vcoud = -eb)
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return lam[a] > lam[b]; });
  for (int j = 0; j < n; ++j) vcoud[j] = lam[perm[j]];
  rc = g_jc_perm.ensure(n * sizeof(int));
  if (rc) return rc;
  QSGW_CUDA(cudaMemcpyAsync(g_jc_perm.p, perm.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
  if (Oh) {
    // z = O^-1/2 y
    rc = zgemm_f64(0, 0, n, n, n, make_double2(1, 0), Oh, n, 0, V, n, 0, make_double2(0, 0), W, n, 0, 1, s);
    if (rc) return rc;
    permute_cols_kernel<<<grid_for(nn), 256, 0, s>>>(A, lda, W, n, n, g_jc_perm.as<int>());
  } else {
    permute_cols_kernel<<<grid_for(nn), 256, 0, s>>>(A, lda, V, n, n, g_jc_perm.as<int>());
  }
  count_launch();
  QSGW_LAUNCH_CHECK("permute_cols_kernel");
  QSGW_CUDA(cudaStreamSynchronize(s));
  return QSGW_OK;
}
