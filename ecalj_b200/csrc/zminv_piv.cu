// Batched inverse of general complex matrices with partial pivoting (stands
// in for zminv = zgetrf + zgetri, m_lapack.f90:108-176, where eps~ is not
// Hermitian: the real frequency axis, WVRllwR m_llw.f90:49-264).
//
// Blocked Gauss-Jordan exchange with row pivots.  For a panel of columns C
// (width nb) the panel kernel picks pivot rows pi by partial pivoting on the
// running Schur complement and sweeps the n x nb panel in place, which gives
// P^-1 on the pivot rows and R P^-1 on the others (P = A[pi, C]); then one
// rank-nb update on the DMMA engine,
//     A <- A - Rb Qb,  Rb = panel result + e_k on pivot row pi_k,
//                      Qb = A[pi, :] with P - I on the columns C,
// completes the exchange of the pair (pi, C) for the whole matrix.  After all
// panels the matrix holds A^-1 with rows and columns permuted:
//     A^-1[a, b] = R[piv[a], pinv[b]],  piv[c] = pivot row of column c.
#include "zgemm_f64.cuh"

namespace qsgw {

constexpr int PV_NB = 32;
constexpr int PV_THREADS = 512;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One CTA per matrix.  X: n x nb panel scratch (ld n), Rb: n x nb, Qb: nb x n (ld nb),
// used: n flags, piv: n pivot rows; flag <- 1 on a zero or non-finite pivot.
__global__ void __launch_bounds__(PV_THREADS) piv_panel_kernel(const double2* __restrict__ A, int n, long long lda,
                                                               long long a_bs, double2* __restrict__ Xall,
                                                               double2* __restrict__ Rball, double2* __restrict__ Qball,
                                                               int* __restrict__ usedall, int* __restrict__ pivall,
                                                               int c0, int w, int* __restrict__ flag) {
  __shared__ double2 rowp[PV_NB];
  __shared__ double sv[PV_THREADS / 32];
  __shared__ int si[PV_THREADS / 32];
  __shared__ int sp;
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double2* Ab = A + b * a_bs;
  double2* X = Xall + static_cast<long long>(b) * n * PV_NB;
  double2* Rb = Rball + static_cast<long long>(b) * n * PV_NB;
  double2* Qb = Qball + static_cast<long long>(b) * n * PV_NB;
  int* used = usedall + static_cast<long long>(b) * n;
  int* piv = pivall + static_cast<long long>(b) * n;
  for (long long e = tid; e < static_cast<long long>(n) * w; e += PV_THREADS) {
    const int r = static_cast<int>(e % n), l = static_cast<int>(e / n);
    X[r + static_cast<long long>(n) * l] = Ab[r + lda * (c0 + l)];
  }
  __syncthreads();
  for (int j = 0; j < w; ++j) {
    // pivot: the unused row with the largest |X[r, j]| (smallest index on ties)
    double best = -1.0;
    int bi = n;
    for (int r = tid; r < n; r += PV_THREADS) {
      if (used[r]) continue;
      const double2 v = X[r + static_cast<long long>(n) * j];
      const double m = v.x * v.x + v.y * v.y;
      if (m > best || (m == best && r < bi)) { best = m; bi = r; }
    }
    for (int o = 16; o; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (lane == 0) { sv[wid] = best; si[wid] = bi; }
    __syncthreads();
    if (tid == 0) {
      double m = sv[0];
      int p = si[0];
      for (int k = 1; k < PV_THREADS / 32; ++k)
        if (sv[k] > m || (sv[k] == m && si[k] < p)) { m = sv[k]; p = si[k]; }
      if (!(m > 0.0) || !isfinite(m) || p >= n) {
        atomicExch(flag, 1);
        p = -1;
      } else {
        used[p] = 1;
        piv[c0 + j] = p;
      }
      sp = p;
    }
    __syncthreads();
    const int p = sp;
    if (p < 0) return;                                  // singular: the caller reports the flag
    if (tid < w) rowp[tid] = X[p + static_cast<long long>(n) * tid];
    __syncthreads();
    const double2 a = rowp[j];
    const double den = a.x * a.x + a.y * a.y;
    const double2 ainv = make_double2(a.x / den, -a.y / den);
    // sweep on (p, j): [[a, q], [r, S]] -> [[1/a, -q/a], [r/a, S - r q / a]]
    for (int r = tid; r < n; r += PV_THREADS) {
      if (r == p) {
        for (int l = 0; l < w; ++l) {
          const double2 q = rowp[l];
          const double2 v = (l == j) ? ainv : cmul(make_double2(-q.x, -q.y), ainv);
          X[p + static_cast<long long>(n) * l] = v;
        }
      } else {
        const double2 xr = cmul(X[r + static_cast<long long>(n) * j], ainv);
        for (int l = 0; l < w; ++l) {
          double2* xp = X + r + static_cast<long long>(n) * l;
          if (l == j) {
            *xp = xr;
          } else {
            const double2 t = cmul(xr, rowp[l]);
            *xp = make_double2(xp->x - t.x, xp->y - t.y);
          }
        }
      }
    }
    __syncthreads();
  }
  // Rb = panel result + e_k on pivot row pi_k; Qb = A[pi, :] - [c = c0 + l]
  for (long long e = tid; e < static_cast<long long>(n) * w; e += PV_THREADS) {
    const int r = static_cast<int>(e % n), l = static_cast<int>(e / n);
    double2 v = X[r + static_cast<long long>(n) * l];
    if (r == piv[c0 + l]) v.x += 1.0;
    Rb[r + static_cast<long long>(n) * l] = v;
  }
  for (long long e = tid; e < static_cast<long long>(n) * w; e += PV_THREADS) {
    const int l = static_cast<int>(e % w), c = static_cast<int>(e / w);
    double2 v = Ab[piv[c0 + l] + lda * c];
    if (c == c0 + l) v.x -= 1.0;
    Qb[l + static_cast<long long>(PV_NB) * c] = v;
  }
}

// out[a + ld b] = R[piv[a] + lda pinv[b]]  (pinv built here from piv)
__global__ void piv_permute_kernel(double2* __restrict__ out, long long ldo, long long o_bs,
                                   const double2* __restrict__ R, long long lda, long long a_bs,
                                   const int* __restrict__ pivall, int n) {
  extern __shared__ int pinv[];
  const int b = blockIdx.y;
  const int* piv = pivall + static_cast<long long>(b) * n;
  // a singular matrix (flagged by the panel kernel) may leave piv incomplete: keep every index in range
  for (int c = threadIdx.x; c < n; c += blockDim.x) pinv[c] = 0;
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const int r = piv[c];
    if (r >= 0 && r < n) pinv[r] = c;
  }
  __syncthreads();
  const double2* Rb = R + b * a_bs;
  double2* ob = out + b * o_bs;
  const long long tot = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(e % n), bb = static_cast<int>(e / n);
    const int r = min(max(piv[a], 0), n - 1);
    ob[a + ldo * bb] = Rb[r + lda * pinv[bb]];
  }
}

static DevBuf g_pv_x, g_pv_r, g_pv_q, g_pv_i, g_pv_t;

int zminv_general_batched(double2* A, int n, long long lda, long long a_bs, int nbatch, cudaStream_t s) {
  if (n <= 0 || nbatch <= 0) return QSGW_OK;
  const size_t pbytes = static_cast<size_t>(n) * PV_NB * nbatch * sizeof(double2);
  int rc;
  if ((rc = g_pv_x.ensure(pbytes))) return rc;
  if ((rc = g_pv_r.ensure(pbytes))) return rc;
  if ((rc = g_pv_q.ensure(pbytes))) return rc;
  if ((rc = g_pv_i.ensure(2 * static_cast<size_t>(n) * nbatch * sizeof(int)))) return rc;
  if ((rc = g_pv_t.ensure(static_cast<size_t>(n) * n * nbatch * sizeof(double2)))) return rc;
  int* used = g_pv_i.as<int>();
  int* piv = used + static_cast<size_t>(n) * nbatch;
  QSGW_CUDA(cudaMemsetAsync(used, 0, 2 * static_cast<size_t>(n) * nbatch * sizeof(int), s));   // used and piv
  QSGW_CUDA(cudaMemsetAsync(ctx().d_flags, 0, sizeof(int), s));
  for (int c0 = 0; c0 < n; c0 += PV_NB) {
    const int w = std::min(PV_NB, n - c0);
    piv_panel_kernel<<<nbatch, PV_THREADS, 0, s>>>(A, n, lda, a_bs, g_pv_x.as<double2>(), g_pv_r.as<double2>(),
                                                   g_pv_q.as<double2>(), used, piv, c0, w, ctx().d_flags);
    count_launch();
    QSGW_LAUNCH_CHECK("piv_panel_kernel");
    rc = zgemm_f64(0, 0, n, n, w, make_double2(-1.0, 0.0), g_pv_r.as<double2>(), n,
                   static_cast<long long>(n) * PV_NB, g_pv_q.as<double2>(), PV_NB, static_cast<long long>(n) * PV_NB,
                   make_double2(1.0, 0.0), A, lda, a_bs, nbatch, s);
    if (rc) return rc;
  }
  // undo the permutation: T = permuted(A), then A = T
  const long long nn = static_cast<long long>(n) * n;
  const dim3 grid(static_cast<unsigned>(std::max<long long>(1, std::min<long long>((nn + 255) / 256, 4096))), nbatch);
  const size_t shm = static_cast<size_t>(n) * sizeof(int);
  if (shm > 48 * 1024) {
    QSGW_CUDA(cudaFuncSetAttribute(piv_permute_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(shm)));
  }
  piv_permute_kernel<<<grid, 256, shm, s>>>(g_pv_t.as<double2>(), n, nn, A, lda, a_bs, piv, n);
  count_launch();
  QSGW_LAUNCH_CHECK("piv_permute_kernel");
  QSGW_CUDA(cudaMemcpy2DAsync(A, lda * sizeof(double2), g_pv_t.as<double2>(), n * sizeof(double2),
                              n * sizeof(double2), static_cast<size_t>(n), cudaMemcpyDeviceToDevice, s));
  for (int bb = 1; bb < nbatch; ++bb) {
    QSGW_CUDA(cudaMemcpy2DAsync(A + bb * a_bs, lda * sizeof(double2), g_pv_t.as<double2>() + bb * nn,
                                n * sizeof(double2), n * sizeof(double2), static_cast<size_t>(n),
                                cudaMemcpyDeviceToDevice, s));
  }
  return QSGW_OK;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_zminv_batched_d(double* a, int n, int lda, int nbatch) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(a && n >= 0 && lda >= std::max(1, n) && nbatch >= 0, "zminv: n=%d lda=%d nbatch=%d", n, lda, nbatch);
  QSGW_ARG((reinterpret_cast<uintptr_t>(a) & 15) == 0, "zminv: array must be 16-byte aligned");
  return zminv_general_batched(reinterpret_cast<double2*>(a), n, lda, static_cast<long long>(lda) * n, nbatch,
                               ctx().stream);
}
