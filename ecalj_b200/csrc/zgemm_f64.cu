// Host side of the FP64 complex GEMM engine and the ZGEMM entry points that
// replace the reference's BLAS shim zmm_h / zmm_d (m_blas.f90:198-228,
// 469-498).
#include <algorithm>
#include <type_traits>
#include "zgemm_f64.cuh"

namespace qsgw {

template <int MODE, bool A_RC, bool B_RC>
static int launch_kernel(const ZParams& p, dim3 grid, cudaStream_t s) {
  auto kern = zgemm_f64_kernel<MODE, A_RC, B_RC>;
  static uint64_t attr_done = 0;                  // one bit per device
  int rc = smem_limit_once(reinterpret_cast<const void*>(kern), static_cast<int>(sizeof(ZSmem)), attr_done);
  if (rc) return rc;
  const char* tag = MODE == ZM_CHI0 ? "chi0_dmma" : (MODE == ZM_SEG ? "sigc_seg_dmma" : "gemm_dmma");
  const int pi = prof_begin(tag, s);
  kern<<<grid, ZG_THREADS, sizeof(ZSmem), s>>>(p);
  prof_end(pi, s);
  count_launch();
  QSGW_LAUNCH_CHECK("zgemm_f64_kernel");
  return QSGW_OK;
}

// ---- thin A^H B: C(0:n, 0:n) += A^H B for complex A, B of K x n (column-major, leading dimensions
// lda, ldb), n <= 64 and K large: the last contraction of Sigma_c, zsec += czmelwc^H zmel over
// K = ngb (ns2 - ns1 + 1) (m_sxcf_gemm.f90:599).  The general engine's 64 x 64 tiles would run
// 2.6x the needed DMMA work at n = 40; here n is padded only to 16 (rows, MB m16 blocks) and 8
// (columns, NB n8 blocks: 48 x 40 at n = 40).  A CTA (4 warps) takes a K range; the MB x NB
// fragments (m16 x n8) of the output are dealt round-robin to its warps, which share the staged
// operands; the CTA's partial sums go to C by FP64 atomics.
constexpr int TH_BK = 16;                          // k per stage
template <int MB>
constexpr int thin_smem_bytes() { return 2 * 2 * TH_BK * (MB * 16 + 2) * static_cast<int>(sizeof(double2)); }
template <int MB, int NB>
__global__ void __launch_bounds__(128) zgemm_hn_thin_kernel(const double2* __restrict__ A, long long lda,
                                                            const double2* __restrict__ B, long long ldb, int n,
                                                            long long K, long long kper, double2* __restrict__ C,
                                                            long long ldc) {
  static_assert(NB <= 2 * MB, "the staged B columns cover 16 MB");
  constexpr int NF = MB * NB, FPW = (NF + 3) / 4;
  constexpr int R = MB * 16, PR = R + 2;           // padded rows of A^H (= columns of B); pitch
  extern __shared__ __align__(16) unsigned char th_smem[];       // thin_smem_bytes<MB>()
  double2 (*sa)[TH_BK][PR] = reinterpret_cast<double2 (*)[TH_BK][PR]>(th_smem);
  double2 (*sb)[TH_BK][PR] = reinterpret_cast<double2 (*)[TH_BK][PR]>(th_smem + 2 * TH_BK * PR * sizeof(double2));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const long long k0 = blockIdx.x * kper, k1 = min(K, k0 + kper);
  if (k0 >= k1) return;
  const int nch = static_cast<int>((k1 - k0 + TH_BK - 1) / TH_BK);
  auto load = [&](int c, int st) {
#pragma unroll
    for (int e = tid; e < TH_BK * R; e += 128) {
      const int kk = e % TH_BK, r = e / TH_BK;
      const long long k = k0 + static_cast<long long>(c) * TH_BK + kk;
      const bool ok = r < n && k < k1;
      cp_async16(&sa[st][kk][r], ok ? A + r * lda + k : A, ok);
      cp_async16(&sb[st][kk][r], ok ? B + r * ldb + k : B, ok);
    }
  };
  double accr[FPW][4], acci[FPW][4];
#pragma unroll
  for (int u = 0; u < FPW; ++u)
#pragma unroll
    for (int e = 0; e < 4; ++e) accr[u][e] = acci[u][e] = 0.0;
  load(0, 0);
  cp_async_commit();
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) load(c + 1, (c + 1) & 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int st = c & 1;
#pragma unroll
    for (int k8 = 0; k8 < TH_BK / 8; ++k8) {
      const int ka = k8 * 8 + t, kb = ka + 4;
#pragma unroll
      for (int u = 0; u < FPW; ++u) {
        const int f = warp + 4 * u;
        if (f >= NF) break;
        const int i = f / NB, j = f % NB;
        const int r0 = i * 16 + g, nn = j * 8 + g;
        const double2 v[4] = {sa[st][ka][r0], sa[st][ka][r0 + 8], sa[st][kb][r0], sa[st][kb][r0 + 8]};
        double ar[4], ai[4], nai[4];                 // a = conj(A(k, m))
#pragma unroll
        for (int e = 0; e < 4; ++e) { ar[e] = v[e].x; ai[e] = -v[e].y; nai[e] = v[e].y; }
        const double2 b0 = sb[st][ka][nn], b1 = sb[st][kb][nn];
        dmma16(accr[u], ar, b0.x, b1.x);
        dmma16(accr[u], nai, b0.y, b1.y);
        dmma16(acci[u], ar, b0.y, b1.y);
        dmma16(acci[u], ai, b0.x, b1.x);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < FPW; ++u) {
    const int f = warp + 4 * u;
    if (f >= NF) break;
    const int i = f / NB, j = f % NB;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int row = i * 16 + g + (e >= 2 ? 8 : 0), col = j * 8 + 2 * t + (e & 1);
      if (row < n && col < n) {
        double* d = reinterpret_cast<double*>(C + row + static_cast<long long>(col) * ldc);
        atomicAdd(d, accr[u][e]);
        atomicAdd(d + 1, acci[u][e]);
      }
    }
  }
}

int zgemm_hn_thin(int n, long long K, const double2* A, long long lda, const double2* B, long long ldb, double2* C,
                  long long ldc, cudaStream_t s) {
  QSGW_ARG(n >= 1 && n <= 64 && K >= 0, "zgemm_hn_thin: n=%d (1..64), K=%lld", n, K);
  if (K == 0) return QSGW_OK;
  const long long nch = (K + TH_BK - 1) / TH_BK;
  auto run = [&](auto mb, auto nb) -> int {
    constexpr int MB = decltype(mb)::value, NB = decltype(nb)::value;
    auto kern = zgemm_hn_thin_kernel<MB, NB>;
    static uint64_t attr = 0;                       // one bit per device
    int rc = smem_limit_once(reinterpret_cast<const void*>(kern), thin_smem_bytes<MB>(), attr);
    if (rc) return rc;
    // one wave: as many K ranges as CTAs fit on the GPU at once (occupancy queried once)
    static int per_sm = 0;
    if (per_sm == 0)
      QSGW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, thin_smem_bytes<MB>()));
    const long long nsplit = std::max<long long>(1, std::min<long long>(nch, std::max(per_sm, 1) * 1LL * ctx().sm_count));
    const long long kper = ((nch + nsplit - 1) / nsplit) * TH_BK;
    const unsigned grid = static_cast<unsigned>((K + kper - 1) / kper);
    kern<<<grid, 128, thin_smem_bytes<MB>(), s>>>(A, lda, B, ldb, n, K, kper, C, ldc);
    return QSGW_OK;
  };
  using std::integral_constant;
  const int pi = prof_begin("gemm_dmma", s);
  int rc;
  const bool odd8 = ((n + 7) / 8) % 2 == 1;        // n8 column blocks: 2 MB - 1 or 2 MB
  if (n <= 16) rc = odd8 ? run(integral_constant<int, 1>(), integral_constant<int, 1>())
                         : run(integral_constant<int, 1>(), integral_constant<int, 2>());
  else if (n <= 32) rc = odd8 ? run(integral_constant<int, 2>(), integral_constant<int, 3>())
                              : run(integral_constant<int, 2>(), integral_constant<int, 4>());
  else if (n <= 48) rc = odd8 ? run(integral_constant<int, 3>(), integral_constant<int, 5>())
                              : run(integral_constant<int, 3>(), integral_constant<int, 6>());
  else rc = odd8 ? run(integral_constant<int, 4>(), integral_constant<int, 7>())
                 : run(integral_constant<int, 4>(), integral_constant<int, 8>());
  if (rc) return rc;
  prof_end(pi, s);
  count_launch();
  QSGW_LAUNCH_CHECK("zgemm_hn_thin_kernel");
  return QSGW_OK;
}

__global__ void zscale_kernel(double2* C, long long ldc, long long c_bs, int m, int n,
                              double2 beta, int beta_zero) {
  const long long b = blockIdx.y;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       idx < static_cast<long long>(m) * n; idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = idx % m, j = idx / m;
    double2* d = C + b * c_bs + i + j * ldc;
    if (beta_zero) {
      *d = make_double2(0.0, 0.0);
    } else {
      const double2 o = *d;
      *d = make_double2(beta.x * o.x - beta.y * o.y, beta.x * o.y + beta.y * o.x);
    }
  }
}

int zgemm_f64(int opa, int opb, int m, int n, int k, double2 alpha,
              const double2* A, long long lda, long long a_bs,
              const double2* B, long long ldb, long long b_bs, double2 beta,
              double2* C, long long ldc, long long c_bs, int nbatch, cudaStream_t s) {
  if (m <= 0 || n <= 0 || nbatch <= 0) return QSGW_OK;
  ZParams p{};
  p.M = m; p.N = n; p.K = k;
  p.A = A; p.a_bs = a_bs; p.a_conj = (opa == 2);
  if (opa == 0) { p.a_rs = 1; p.a_ks = lda; } else { p.a_rs = lda; p.a_ks = 1; }
  p.B = B; p.b_bs = b_bs; p.b_conj = (opb == 2);
  if (opb == 0) { p.b_rs = ldb; p.b_ks = 1; } else { p.b_rs = 1; p.b_ks = ldb; }
  p.C = C; p.ldc = ldc; p.c_bs = c_bs;
  p.alpha = alpha; p.beta = beta;
  p.beta_zero = (beta.x == 0.0 && beta.y == 0.0);
  p.ntm = (m + ZG_BM - 1) / ZG_BM; p.ntn = (n + ZG_BN - 1) / ZG_BN;
  if (k <= 0) {  // C = beta C
    dim3 g(static_cast<unsigned>(std::min<long long>((static_cast<long long>(m) * n + 255) / 256, 4096)),
           nbatch);
    zscale_kernel<<<g, 256, 0, s>>>(C, ldc, c_bs, m, n, beta, p.beta_zero);
    count_launch();
    QSGW_LAUNCH_CHECK("zscale_kernel");
    return QSGW_OK;
  }
  const int nch = (k + ZG_BK - 1) / ZG_BK;
  const long long tiles = static_cast<long long>(p.ntm) * p.ntn * nbatch;
  const int slots = 2 * ctx().sm_count;
  int splitk = 1;
  if (tiles < slots && nch >= 8) {
    splitk = static_cast<int>((slots + tiles - 1) / tiles);
    splitk = std::min(splitk, nch / 4);
    splitk = std::max(splitk, 1);
  }
  p.kch_per_split = (nch + splitk - 1) / splitk;
  splitk = (nch + p.kch_per_split - 1) / p.kch_per_split;
  p.splitk = splitk;
  if (splitk > 1) {
    // beta applied up front; the tiles then add alpha*acc atomically
    dim3 g(static_cast<unsigned>(std::min<long long>((static_cast<long long>(m) * n + 255) / 256, 4096)),
           nbatch);
    zscale_kernel<<<g, 256, 0, s>>>(C, ldc, c_bs, m, n, beta, p.beta_zero);
    count_launch();
    QSGW_LAUNCH_CHECK("zscale_kernel");
  }
  dim3 grid(static_cast<unsigned>(p.ntm * p.ntn), nbatch, splitk);
  const bool arc = (opa == 0), brc = (opb != 0);
  if (arc && brc) return launch_kernel<ZM_GEMM, true, true>(p, grid, s);
  if (arc && !brc) return launch_kernel<ZM_GEMM, true, false>(p, grid, s);
  if (!arc && brc) return launch_kernel<ZM_GEMM, false, true>(p, grid, s);
  return launch_kernel<ZM_GEMM, false, false>(p, grid, s);
}

int zgemm_chi0_launch(ZParams p, int nbins, int herm, int splitk, cudaStream_t s) {
  p.herm = herm;
  p.splitk = splitk;
  const int ntiles = herm ? p.ntm * (p.ntm + 1) / 2 : p.ntm * p.ntn;
  dim3 grid(static_cast<unsigned>(ntiles), nbins, splitk);
  return launch_kernel<ZM_CHI0, true, true>(p, grid, s);
}

int zgemm_seg_launch(ZParams p, int ncol_tiles, cudaStream_t s) {
  if (ncol_tiles > 65535) {
    set_error("segmented GEMM: %d column tiles exceed the grid limit", ncol_tiles);
    return QSGW_ERR_UNSUPPORTED;
  }
  p.ntm = (p.M + ZG_BM - 1) / ZG_BM;
  p.splitk = 1;
  dim3 grid(static_cast<unsigned>(p.ntm), ncol_tiles, 1);
  // A = op(W): 'C' / 'T' -> k-contiguous rows, 'N' -> row-contiguous
  if (p.a_rs == 1) return launch_kernel<ZM_SEG, true, false>(p, grid, s);
  return launch_kernel<ZM_SEG, false, false>(p, grid, s);
}

}  // namespace qsgw

using namespace qsgw;

static int zmm_check(int m, int n, int k, int opa, int opb, int lda, int ldb, int ldc) {
  QSGW_ARG(m >= 0 && n >= 0 && k >= 0, "qsgw_zmm: negative size m=%d n=%d k=%d", m, n, k);
  QSGW_ARG(opa >= 0 && opa <= 2 && opb >= 0 && opb <= 2, "qsgw_zmm: op must be 0 (N), 1 (T) or 2 (C)");
  QSGW_ARG(lda >= std::max(1, opa == 0 ? m : k), "qsgw_zmm: lda=%d too small", lda);
  QSGW_ARG(ldb >= std::max(1, opb == 0 ? k : n), "qsgw_zmm: ldb=%d too small", ldb);
  QSGW_ARG(ldc >= std::max(1, m), "qsgw_zmm: ldc=%d too small", ldc);
  return QSGW_OK;
}

extern "C" int qsgw_zmm_d(const double* a, const double* b, double* c, int m, int n, int k,
                          int opa, int opb, const double* alpha, const double* beta,
                          int lda, int ldb, int ldc) {
  int rc = require_init();
  if (rc) return rc;
  rc = zmm_check(m, n, k, opa, opb, lda, ldb, ldc);
  if (rc) return rc;
  QSGW_ARG(alpha && beta, "qsgw_zmm: alpha/beta must point to (re, im) pairs");
  return zgemm_f64(opa, opb, m, n, k, make_double2(alpha[0], alpha[1]),
                   reinterpret_cast<const double2*>(a), lda, 0,
                   reinterpret_cast<const double2*>(b), ldb, 0,
                   make_double2(beta[0], beta[1]), reinterpret_cast<double2*>(c), ldc, 0, 1,
                   ctx().stream);
}

extern "C" int qsgw_zmm(const double* a, const double* b, double* c, int m, int n, int k,
                        int opa, int opb, const double* alpha, const double* beta,
                        int lda, int ldb, int ldc) {
  int rc = require_init();
  if (rc) return rc;
  rc = zmm_check(m, n, k, opa, opb, lda, ldb, ldc);
  if (rc) return rc;
  QSGW_ARG(alpha && beta, "qsgw_zmm: alpha/beta must point to (re, im) pairs");
  cudaStream_t s = ctx().stream;
  const size_t na = static_cast<size_t>(lda) * (opa == 0 ? k : m);
  const size_t nb = static_cast<size_t>(ldb) * (opb == 0 ? n : k);
  const size_t nc = static_cast<size_t>(ldc) * n;
  DevBuf da, db, dc;
  rc = da.ensure(na * 16); if (rc) return rc;
  rc = db.ensure(nb * 16); if (rc) { da.release(); return rc; }
  rc = dc.ensure(nc * 16); if (rc) { da.release(); db.release(); return rc; }
  auto done = [&](int r) { da.release(); db.release(); dc.release(); return r; };
  if (na) { rc = check_cuda(cudaMemcpyAsync(da.p, a, na * 16, cudaMemcpyHostToDevice, s), "H2D a"); if (rc) return done(rc); }
  if (nb) { rc = check_cuda(cudaMemcpyAsync(db.p, b, nb * 16, cudaMemcpyHostToDevice, s), "H2D b"); if (rc) return done(rc); }
  rc = check_cuda(cudaMemcpyAsync(dc.p, c, nc * 16, cudaMemcpyHostToDevice, s), "H2D c");
  if (rc) return done(rc);
  rc = zgemm_f64(opa, opb, m, n, k, make_double2(alpha[0], alpha[1]), da.as<double2>(), lda, 0,
                 db.as<double2>(), ldb, 0, make_double2(beta[0], beta[1]), dc.as<double2>(), ldc, 0,
                 1, s);
  if (rc) return done(rc);
  rc = check_cuda(cudaMemcpyAsync(c, dc.p, nc * 16, cudaMemcpyDeviceToHost, s), "D2H c");
  if (rc) return done(rc);
  rc = check_cuda(cudaStreamSynchronize(s), "qsgw_zmm sync");
  return done(rc);
}
