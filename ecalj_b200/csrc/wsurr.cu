// Learned interpolator of W_c(q, i w) across the imaginary-frequency grid.
//
// The plain method computes W_c exactly at a few anchor frequencies; the
// network predicts W_c at the other frequencies of the grid.
//
// One sample = one real channel (re or im) of one element of W_c(q) and one
// target frequency t.  Features (16): the channel at the na anchor
// frequencies divided by s = max |anchor value|, the Gauss-Legendre x of the
// target, 1, zero padding.  Output (normalised by s):
//     y = sum_i C[t][i] x_i  +  MLP(x),     MLP: 16 -> 256 -> 256 -> 1, ReLU.
// C is a per-target linear head (FP32); rows >= 64 are linear only (no MLP
// term), for the part of the matrix outside the dominant block.  The MLP has
// BF16 weights (FP32
// master copy for Adam) and accumulates in FP32.  Loss: the s^2-weighted
// mean squared error, i.e. the squared Frobenius error of the un-normalised
// prediction.  Every kernel here is hand-written: projection of W_c on the
// dominant Coulomb eigenvectors, features, forward, backward, Adam, the
// full-matrix linear head and the scatter of the block predictions.
#include <cuda_bf16.h>
#include <cmath>
#include <vector>
#include "common.cuh"

namespace qsgw {
namespace ws {

// Head rows 0..NMLP-1 carry the MLP correction (dominant block); rows NMLP..NTMAX-1
// are linear only (the rest of the matrix).
constexpr int NIN = 16, NH = 256, NTMAX = 128, NMLP = 64;
// parameter layout: W1[NIN][NH], b1[NH], W2[NH][NH], b2[NH], W3[NH], b3, C[NTMAX][NIN]
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NIN * NH, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH, OFF_C = OFF_B3 + 1, NPARAM = OFF_C + NTMAX * NIN;

struct State {
  bool ready = false;
  float* master = nullptr;     // FP32 parameters
  __nv_bfloat16* w16 = nullptr;
  float* grad = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* red = nullptr;        // [0] = sum of w e^2, [1] = sum of w
  double* lsq = nullptr;       // normal equations of the heads: G[NTMAX][NIN*NIN], then H[NTMAX][NIN]
  int step = 0;
  int cap = 0;                 // batch capacity of the buffers below
  __nv_bfloat16* w2t = nullptr;  // W2 transposed [n][k] (BF16), the forward GEMM's B operand
  __nv_bfloat16* h1 = nullptr;   // layer-1 activations (batch x NH, BF16: the layer-2 GEMM's operand)
  __nv_bfloat16* h1t = nullptr;  // the same transposed (NH x cap), the weight-gradient GEMM's operand
  float* h2 = nullptr;
  float* g1 = nullptr;         // dL/dpre1
  float* g2 = nullptr;         // dL/dpre2 (FP32, for db2)
  __nv_bfloat16* g2b = nullptr;  // dL/dpre2 in BF16 (batch x NH) and transposed (NH x cap)
  __nv_bfloat16* g2t = nullptr;
  float* head = nullptr;       // linear-head term of every row
  float* out = nullptr;
  float* xb = nullptr;         // gathered mini-batch
  float* yb = nullptr;
  float* wb = nullptr;
  int* tb = nullptr;
};
static State g;

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__global__ void init_params_kernel(float* p, unsigned long long seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  const unsigned long long z = mix64(seed + 0x9E3779B97F4A7C15ULL * (i + 1));
  const float u = static_cast<float>(z >> 40) / static_cast<float>(1ULL << 24) * 2.f - 1.f;  // [-1, 1)
  float scale = 0.f;                                   // biases and the linear head start at zero
  if (i < OFF_B1) scale = sqrtf(6.f / NIN);
  else if (i >= OFF_W2 && i < OFF_B2) scale = sqrtf(6.f / NH);
  else if (i >= OFF_W3 && i < OFF_B3) scale = sqrtf(3.f / NH) * 0.01f;   // small initial correction
  p[i] = u * scale;
}

__global__ void to_bf16_kernel(const float* __restrict__ p, __nv_bfloat16* __restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NPARAM) w[i] = __float2bfloat16_rn(p[i]);
}

// Forward pass, layer 1 and the linear head: one block = 32 samples, thread = hidden unit.
// h1 = relu(x W1 + b1) in BF16 (row-major, and transposed into h1t when training, rows
// beyond the batch up to the 32-row block zero); head[r] = C[t_r] . x_r (FP32 master
// parameters).  With wt and sumw (training) the sum of the sample weights is added to *sumw.
__global__ void __launch_bounds__(256) forward_l1_kernel(const float* __restrict__ x, const int* __restrict__ tix,
                                                         int batch, const __nv_bfloat16* __restrict__ w,
                                                         const float* __restrict__ master,
                                                         __nv_bfloat16* __restrict__ h1, __nv_bfloat16* __restrict__ h1t,
                                                         long long ldt, float* __restrict__ head,
                                                         const float* __restrict__ wt, float* __restrict__ sumw) {
  __shared__ float sx[32][NIN];
  const int s0 = blockIdx.x * 32;
  const int tid = threadIdx.x;
  for (int e = tid; e < 32 * NIN; e += blockDim.x) {
    const int r = e / NIN, c = e % NIN;
    sx[r][c] = (s0 + r < batch) ? x[static_cast<long long>(s0 + r) * NIN + c] : 0.f;
  }
  __syncthreads();
  if (tid < 32 && s0 + tid < batch) {
    float a = 0.f;
    const int t = tix[s0 + tid];
    if (t >= 0 && t < NTMAX) {                         // rows with a bad head index get no head term
      const float* c = master + OFF_C + t * NIN;
#pragma unroll
      for (int i = 0; i < NIN; ++i) a += c[i] * sx[tid][i];
    }
    head[s0 + tid] = a;
    if (wt && sumw) atomicAdd(sumw, wt[s0 + tid]);
  }
  float wcol[NIN];
#pragma unroll
  for (int i = 0; i < NIN; ++i) wcol[i] = bf(w[OFF_W1 + i * NH + tid]);
  const float b1 = bf(w[OFF_B1 + tid]);
  for (int r = 0; r < 32; ++r) {
    const bool in = s0 + r < batch;
    float a = b1;
#pragma unroll
    for (int i = 0; i < NIN; ++i) a += sx[r][i] * wcol[i];
    const __nv_bfloat16 v = __float2bfloat16_rn(in ? fmaxf(a, 0.f) : 0.f);
    if (in) h1[static_cast<long long>(s0 + r) * NH + tid] = v;
    if (h1t) h1t[static_cast<long long>(tid) * ldt + s0 + r] = v;
  }
}

// Forward pass, layer 3: out_r = m_r (h2_r . W3 + b3) + head_r, m_r = 0 on linear-only rows.
// One warp per row.
__global__ void forward_l3_kernel(const float* __restrict__ h2, const int* __restrict__ tix, int batch,
                                  const __nv_bfloat16* __restrict__ w, const float* __restrict__ head,
                                  float* __restrict__ out) {
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= batch) return;
  float a = 0.f;
  for (int k = lane; k < NH; k += 32) a += h2[static_cast<long long>(r) * NH + k] * bf(w[OFF_W3 + k]);
  for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (lane == 0) out[r] = (tix[r] < NMLP ? a + bf(w[OFF_B3]) : 0.f) + head[r];
}

// C[m][n] = sum_k A[m][k] Bt[n][k] on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32
// accumulation): A (M x K) and Bt (N x K) row-major BF16, K a multiple of 32 within each split,
// N a multiple of 128.  Block tile 64 x 128 (8 warps of 32 x 32), K steps of 32 through shared
// memory (80-byte rows: conflict-free ldmatrix).  Epilogues: layer 2 forward (bias, ReLU, FP32
// h2), layer 2 backward (the unit's ReLU mask from h1, FP32 g1), weight gradient (FP32 atomics,
// one K split per blockIdx.z).
enum { EPI_FWD = 0, EPI_BWD = 1, EPI_WGRAD = 2 };
struct MmaArgs {
  const __nv_bfloat16* A;
  long long lda;
  const __nv_bfloat16* Bt;
  long long ldb;
  int M, N, K, ksplit;
  float* C;
  long long ldc;
  const __nv_bfloat16* bias;   // EPI_FWD: b2
  const __nv_bfloat16* mask;   // EPI_BWD: h1 (ld = ldc)
};

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int EPI>
__global__ void __launch_bounds__(256) mma_gemm_kernel(const MmaArgs p) {
  __shared__ __align__(16) __nv_bfloat16 sa[64][40];
  __shared__ __align__(16) __nv_bfloat16 sb[128][40];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 128;
  const int kb = blockIdx.z * p.ksplit, ke = min(p.K, kb + p.ksplit);
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
  for (int k0 = kb; k0 < ke; k0 += 32) {
    {
      const int r = tid >> 2, c = (tid & 3) * 8;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (m0 + r < p.M) v = *reinterpret_cast<const uint4*>(p.A + static_cast<long long>(m0 + r) * p.lda + k0 + c);
      *reinterpret_cast<uint4*>(&sa[r][c]) = v;
    }
#pragma unroll
    for (int i = tid; i < 512; i += 256) {
      const int r = i >> 2, c = (i & 3) * 8;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (n0 + r < p.N) v = *reinterpret_cast<const uint4*>(p.Bt + static_cast<long long>(n0 + r) * p.ldb + k0 + c);
      *reinterpret_cast<uint4*>(&sb[r][c]) = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 32; kk += 16) {
      uint32_t af[2][4], bq[2][4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) ldsm_x4(af[mi], &sa[wm + mi * 16 + (lane & 15)][kk + (lane >> 4) * 8]);
#pragma unroll
      for (int nj = 0; nj < 2; ++nj)   // n8 tiles 2 nj and 2 nj + 1: {b0, b1} of each
        ldsm_x4(bq[nj], &sb[wn + nj * 16 + ((lane >> 4) & 1) * 8 + (lane & 7)][kk + ((lane >> 3) & 1) * 8]);
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], af[mi], bq[ni >> 1][(ni & 1) * 2], bq[ni >> 1][(ni & 1) * 2 + 1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int m = m0 + wm + mi * 16 + (lane >> 2) + (e >> 1) * 8;
        const int n = n0 + wn + ni * 8 + (lane & 3) * 2 + (e & 1);
        if (m >= p.M || n >= p.N) continue;
        const float v = acc[mi][ni][e];
        const long long o = static_cast<long long>(m) * p.ldc + n;
        if (EPI == EPI_FWD) p.C[o] = fmaxf(v + bf(p.bias[n]), 0.f);
        else if (EPI == EPI_BWD) p.C[o] = (bf(p.mask[o]) > 0.f) ? v : 0.f;
        else atomicAdd(&p.C[o], v);
      }
}

// w2t[n][k] = W2[k][n] (BF16), the forward GEMM's B operand
__global__ void w2t_kernel(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ w2t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NH * NH) return;
  const int n = i / NH, k = i % NH;
  w2t[i] = w[OFF_W2 + k * NH + n];
}

// db[j] += sum_r G[r][j] (FP32), rows split over blockIdx.y
__global__ void colsum_kernel(const float* __restrict__ G, int batch, int rows_per_block, float* __restrict__ db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= NH) return;
  const int r0 = blockIdx.y * rows_per_block, r1 = min(batch, r0 + rows_per_block);
  float a = 0.f;
  for (int r = r0; r < r1; ++r) a += G[static_cast<long long>(r) * NH + j];
  atomicAdd(&db[j], a);
}

// Backward of L = sum_r w_r (out_r - y_r)^2 / sum_r w_r (w_r = 1 without weights),
// activation part: g2 = dL/dpre2, g1 = dL/dpre1; dW3, db3, dC and the loss
// numerator are reduced here.  One block = 32 samples, thread = hidden unit.
__global__ void __launch_bounds__(256) backward_act_kernel(const float* __restrict__ x, const int* __restrict__ tix,
                                                           const float* __restrict__ y, const float* __restrict__ wt,
                                                           int batch, const __nv_bfloat16* __restrict__ w,
                                                           const float* __restrict__ h2,
                                                           const float* __restrict__ out, float* __restrict__ g2,
                                                           __nv_bfloat16* __restrict__ g2b,
                                                           __nv_bfloat16* __restrict__ g2t, long long ldt,
                                                           float* __restrict__ grad, float* __restrict__ red) {
  __shared__ float sd[32];      // dL/dout for the MLP part (0 on linear-only rows)
  __shared__ float sdh[32];     // dL/dout for the head
  const int s0 = blockIdx.x * 32;
  const int tid = threadIdx.x;
  const float inv_sumw = wt ? 1.f / fmaxf(red[1], 1e-30f) : 1.f / batch;
  if (tid < 32) {
    float d = 0.f;
    int t = -1;
    if (s0 + tid < batch) {
      const float e = out[s0 + tid] - y[s0 + tid];
      const float wr = wt ? wt[s0 + tid] : 1.f;
      d = 2.f * wr * e * inv_sumw;
      atomicAdd(&red[0], wr * e * e);
      t = tix[s0 + tid];
    }
    sdh[tid] = d;
    sd[tid] = (t < NMLP) ? d : 0.f;
  }
  __syncthreads();
  // dC[t][i] += d_r x_r[i]
  for (int e = tid; e < 32 * NIN; e += blockDim.x) {
    const int r = e / NIN, i = e % NIN;
    if (s0 + r < batch && sdh[r] != 0.f) {
      const int t = tix[s0 + r];
      if (t >= 0 && t < NTMAX)
        atomicAdd(&grad[OFF_C + t * NIN + i], sdh[r] * x[static_cast<long long>(s0 + r) * NIN + i]);
    }
  }
  const float w3 = bf(w[OFF_W3 + tid]);
  float gw3 = 0.f;
  for (int r = 0; r < 32; ++r) {
    const bool in = s0 + r < batch;
    const float a2 = in ? h2[static_cast<long long>(s0 + r) * NH + tid] : 0.f;
    gw3 += a2 * sd[r];
    const float gv = (a2 > 0.f) ? sd[r] * w3 : 0.f;
    const __nv_bfloat16 gb = __float2bfloat16_rn(gv);
    if (in) {
      g2[static_cast<long long>(s0 + r) * NH + tid] = gv;
      g2b[static_cast<long long>(s0 + r) * NH + tid] = gb;
    }
    g2t[static_cast<long long>(tid) * ldt + s0 + r] = gb;   // zero beyond the batch
  }
  atomicAdd(&grad[OFF_W3 + tid], gw3);
  if (tid == 0) {
    float gb3 = 0.f;
    for (int r = 0; r < 32; ++r) gb3 += sd[r];
    atomicAdd(&grad[OFF_B3], gb3);
  }
}

// dW[k][j] += sum_r A[r][k] G[r][j] over a chunk of rows, db[j] += sum_r G[r][j]
// (k-tile 0 only).  A: (batch x K), G: (batch x NH); block = 32 x 32 tile.
__global__ void __launch_bounds__(256) wgrad_kernel(const float* __restrict__ A, int K, const float* __restrict__ G,
                                                    int batch, int rows_per_block, float* __restrict__ dW,
                                                    float* __restrict__ db) {
  __shared__ float sa[64][33];
  __shared__ float sgm[64][33];
  const int k0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const int r_begin = blockIdx.z * rows_per_block;
  const int r_end = min(batch, r_begin + rows_per_block);
  const int tid = threadIdx.x;
  const int tk = tid >> 3, tj = (tid & 7) * 4;   // each thread: 1 k x 4 j
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  float bacc = 0.f;
  for (int r0 = r_begin; r0 < r_end; r0 += 64) {
    for (int e = tid; e < 64 * 32; e += 256) {
      const int rr = e >> 5, c = e & 31;
      const int r = r0 + rr;
      sa[rr][c] = (r < r_end && k0 + c < K) ? A[static_cast<long long>(r) * K + k0 + c] : 0.f;
      sgm[rr][c] = (r < r_end) ? G[static_cast<long long>(r) * NH + j0 + c] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < 64; ++rr) {
      const float a = sa[rr][tk];
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] += a * sgm[rr][tj + u];
    }
    if (blockIdx.x == 0 && tid < 32) {
      for (int rr = 0; rr < 64; ++rr) bacc += sgm[rr][tid];
    }
    __syncthreads();
  }
  if (k0 + tk < K) {
#pragma unroll
    for (int u = 0; u < 4; ++u) atomicAdd(&dW[(k0 + tk) * NH + j0 + tj + u], acc[u]);
  }
  if (blockIdx.x == 0 && tid < 32) atomicAdd(&db[j0 + tid], bacc);
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m1,
                            float* __restrict__ m2, __nv_bfloat16* __restrict__ w, float lr, float b1, float b2,
                            float c1, float c2, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  const float gi = gr[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = v;
  const float np_ = p[i] - lr * (a / c1) / (sqrtf(v / c2) + eps);
  p[i] = np_;
  w[i] = __float2bfloat16_rn(np_);
}

// Random mini-batch: sample i of step `step` is row mix64(seed, step, i) mod n.
__global__ void gather_batch_kernel(const float* __restrict__ x, const int* __restrict__ tix,
                                    const float* __restrict__ y, const float* __restrict__ wt, long long n, int batch,
                                    unsigned long long seed, int step, float* __restrict__ xb, int* __restrict__ tb,
                                    float* __restrict__ yb, float* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= batch) return;
  const unsigned long long h = mix64(seed ^ mix64(0x632BE59BD9B4E019ULL * (static_cast<unsigned long long>(step) + 1) +
                                                  static_cast<unsigned long long>(i)));
  const long long r = static_cast<long long>(h % static_cast<unsigned long long>(n));
#pragma unroll
  for (int c = 0; c < NIN; ++c) xb[static_cast<long long>(i) * NIN + c] = x[r * NIN + c];
  tb[i] = tix[r];
  yb[i] = y[r];
  wb[i] = wt ? wt[r] : 1.f;
}

// Block of W_c: proj[slot][2 (i + nb j) + c] = component c of W[slot](ridx[i], cidx[j]);
// W slots are ld x ld column-major complex, slot stride ld*ld.
__global__ void project_kernel(const double2* __restrict__ wc, int ld, int nslot, const int* __restrict__ ridx,
                               const int* __restrict__ cidx, int nb, float* __restrict__ proj) {
  const long long tot = static_cast<long long>(nslot) * nb * nb;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % nb);
    const long long r = e / nb;
    const int j = static_cast<int>(r % nb);
    const int sl = static_cast<int>(r / nb);
    const double2 v = wc[static_cast<long long>(sl) * ld * ld + ridx[i] + static_cast<long long>(ld) * cidx[j]];
    proj[2 * e] = static_cast<float>(v.x);
    proj[2 * e + 1] = static_cast<float>(v.y);
  }
}

// Element features after the anchors, x_t and 1 (slots na+2 .. na+5): ftab of the
// element's row and column index (log10 of the Coulomb eigenvalue / 3), the
// channel (0 = re, 1 = im) and 1 on the diagonal.  Zero when ftab is null.
__device__ __forceinline__ void element_features(float* xs, int na, const float* __restrict__ ftab, int row, int col,
                                                 int c) {
  if (!ftab) return;
  xs[na + 2] = ftab[row];
  xs[na + 3] = ftab[col];
  xs[na + 4] = static_cast<float>(c);
  xs[na + 5] = (row == col) ? 1.f : 0.f;
}

// Samples (target fastest, then channel, then q): x, tix, y = v(target)/s, wgt = s^2, scale = s.
// proj: (nq, nw, ne) float, ne = 2 nb nb real channels per frequency, channel
// 2 (i + nb j) + c of the block (rid[i], cid[j]).
__global__ void features_kernel(const float* __restrict__ proj, int nq, int nw, int ne,
                                const int* __restrict__ anchors, int na, const int* __restrict__ targets,
                                const int* __restrict__ tslot, int nt, const float* __restrict__ xcoord,
                                const int* __restrict__ rid, const int* __restrict__ cid, int nb,
                                const float* __restrict__ ftab, float* __restrict__ x, int* __restrict__ tix,
                                float* __restrict__ y, float* __restrict__ wgt, float* __restrict__ scale) {
  const long long tot = static_cast<long long>(nq) * ne * nt;
  for (long long sidx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; sidx < tot;
       sidx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int ti = static_cast<int>(sidx % nt);
    const long long r = sidx / nt;
    const int e = static_cast<int>(r % ne);
    const int q = static_cast<int>(r / ne);
    const float* base = proj + static_cast<long long>(q) * nw * ne + e;
    float s = 1e-30f;
    for (int a = 0; a < na; ++a) s = fmaxf(s, fabsf(base[static_cast<long long>(anchors[a]) * ne]));
    float* xs = x + sidx * NIN;
    for (int a = 0; a < NIN; ++a) xs[a] = 0.f;
    for (int a = 0; a < na; ++a) xs[a] = base[static_cast<long long>(anchors[a]) * ne] / s;
    xs[na] = xcoord[targets[ti]];
    xs[na + 1] = 1.f;
    if (ftab) {
      const int el = e >> 1;
      element_features(xs, na, ftab, rid[el % nb], cid[el / nb], e & 1);
    }
    tix[sidx] = tslot[ti];
    if (y) y[sidx] = base[static_cast<long long>(targets[ti]) * ne] / s;
    if (wgt) wgt[sidx] = s * s;
    if (scale) scale[sidx] = s;
  }
}

// Linear head on the full matrix: for every real channel of W (ld x ld complex per slot),
// W[tslot_out[t]] = s * sum_i C[thead[t]][i] x_i with x built from the anchor slots as in
// features_kernel (ftab over all n indices, or null).  Anchor and target slots are distinct.
__global__ void head_full_kernel(double2* __restrict__ wc, int n, int ld, const int* __restrict__ aslot, int na,
                                 const int* __restrict__ tslot_out, const int* __restrict__ thead,
                                 const float* __restrict__ txc, int nt, const float* __restrict__ ftab,
                                 const float* __restrict__ master) {
  const long long tot = static_cast<long long>(n) * n * 2;
  const long long ss = static_cast<long long>(ld) * ld;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(e & 1);
    const long long el = e >> 1;
    const int i = static_cast<int>(el % n), j = static_cast<int>(el / n);
    const long long off = i + static_cast<long long>(ld) * j;
    const double* w = reinterpret_cast<const double*>(wc);
    float xs[NIN];
    float s = 1e-30f;
    for (int a = 0; a < NIN; ++a) xs[a] = 0.f;
    for (int a = 0; a < na; ++a) {
      xs[a] = static_cast<float>(w[2 * (aslot[a] * ss + off) + c]);
      s = fmaxf(s, fabsf(xs[a]));
    }
    for (int a = 0; a < na; ++a) xs[a] = xs[a] / s;
    xs[na + 1] = 1.f;
    element_features(xs, na, ftab, i, j, c);
    for (int t = 0; t < nt; ++t) {
      const float* C = master + OFF_C + thead[t] * NIN;
      xs[na] = txc[t];
      float acc = 0.f;
#pragma unroll
      for (int a = 0; a < NIN; ++a) acc += C[a] * xs[a];
      reinterpret_cast<double*>(wc)[2 * (tslot_out[t] * ss + off) + c] = static_cast<double>(acc * s);
    }
  }
}

// Network predictions (normalised; samples in the features order, one q) back into the
// dominant block of the target slots: W[tslot_out[t]](idx[i], idx[j]).c = pred * scale.
__global__ void scatter_block_kernel(double2* __restrict__ wc, int ld, const int* __restrict__ idx, int nb,
                                     const int* __restrict__ tslot_out, int nt, const float* __restrict__ pred,
                                     const float* __restrict__ scale) {
  const long long tot = static_cast<long long>(2) * nb * nb * nt;
  const long long ss = static_cast<long long>(ld) * ld;
  for (long long sidx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; sidx < tot;
       sidx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int ti = static_cast<int>(sidx % nt);
    const long long ch = sidx / nt;
    const int c = static_cast<int>(ch & 1);
    const long long el = ch >> 1;
    const int i = static_cast<int>(el % nb), j = static_cast<int>(el / nb);
    const long long off = tslot_out[ti] * ss + idx[i] + static_cast<long long>(ld) * idx[j];
    reinterpret_cast<double*>(wc)[2 * off + c] = static_cast<double>(pred[sidx] * scale[sidx]);
  }
}

// Normal equations of the linear head rows: G[h] += sum_r w_r x_r x_r^T,
// H[h] += sum_r w_r x_r y_r over the samples s = k nt + ti of target ti
// (features order, target fastest), h = thead[ti].  Block (chunk, ti),
// thread (i, j) of the 16 x 16 Gram matrix, FP64 sums (FP32 sums leave the
// Gram matrix indefinite at the 1e-7 level, below any useful ridge).
__global__ void __launch_bounds__(256) lsq_accumulate_kernel(const float* __restrict__ x, const float* __restrict__ y,
                                                             const float* __restrict__ w, long long n, int nt,
                                                             const int* __restrict__ thead, long long per_block,
                                                             double* __restrict__ G, double* __restrict__ H) {
  __shared__ float sx[64][NIN + 1];
  __shared__ float sy[64], sw[64];
  const int ti = blockIdx.y;
  const int h = thead[ti];
  const int tid = threadIdx.x, i = tid >> 4, j = tid & 15;
  const long long nk = (n - ti + nt - 1) / nt;
  const long long k0 = blockIdx.x * per_block;
  const long long k1 = (k0 + per_block < nk) ? k0 + per_block : nk;
  double g = 0.0, hh = 0.0;
  for (long long kb = k0; kb < k1; kb += 64) {
    for (int e = tid; e < 64 * NIN; e += 256) {
      const int r = e / NIN, c = e % NIN;
      const long long k = kb + r;
      sx[r][c] = (k < k1) ? x[(k * nt + ti) * NIN + c] : 0.f;
    }
    if (tid < 64) {
      const long long k = kb + tid;
      sy[tid] = (k < k1) ? y[k * nt + ti] : 0.f;
      sw[tid] = (k < k1) ? (w ? w[k * nt + ti] : 1.f) : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int r = 0; r < 64; ++r) {
      const double wx = static_cast<double>(sw[r]) * sx[r][i];
      g += wx * sx[r][j];
      hh += wx * sy[r];
    }
    __syncthreads();
  }
  atomicAdd(&G[h * NIN * NIN + tid], g);
  if (j == 0) atomicAdd(&H[h * NIN + i], hh);
}

// Cholesky solve of the SPD system a x = b (n <= NIN), a overwritten; false if not SPD.
static bool chol_solve(double* a, double* b, int n) {
  for (int j = 0; j < n; ++j) {
    double d = a[j * n + j];
    for (int k = 0; k < j; ++k) d -= a[j * n + k] * a[j * n + k];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    a[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double v = a[i * n + j];
      for (int k = 0; k < j; ++k) v -= a[i * n + k] * a[j * n + k];
      a[i * n + j] = v / d;
    }
  }
  for (int i = 0; i < n; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= a[i * n + k] * b[k];
    b[i] = v / a[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double v = b[i];
    for (int k = i + 1; k < n; ++k) v -= a[k * n + i] * b[k];
    b[i] = v / a[i * n + i];
  }
  return true;
}

static void free_batch() {
  cudaFree(g.h1); cudaFree(g.h1t); cudaFree(g.h2); cudaFree(g.g1); cudaFree(g.g2); cudaFree(g.g2b);
  cudaFree(g.g2t); cudaFree(g.head); cudaFree(g.out);
  cudaFree(g.xb); cudaFree(g.yb); cudaFree(g.wb); cudaFree(g.tb);
  g.h2 = g.g1 = g.g2 = g.head = g.out = g.xb = g.yb = g.wb = nullptr;
  g.h1 = g.h1t = g.g2b = g.g2t = nullptr;
  g.tb = nullptr;
  g.cap = 0;
}

// rows of the transposed activation buffers (the batch capacity rounded up to the 32-row blocks)
static long long ldt() { return (static_cast<long long>(g.cap) + 31) / 32 * 32; }

static int ensure_cap(int batch) {
  if (batch <= g.cap) return QSGW_OK;
  if (g.cap) {
    QSGW_CUDA(cudaStreamSynchronize(ctx().stream));
    free_batch();
  }
  const size_t b = static_cast<size_t>(batch);
  const size_t b32 = (b + 31) / 32 * 32;
  QSGW_CUDA(cudaMalloc(&g.h1, b * NH * sizeof(__nv_bfloat16)));
  QSGW_CUDA(cudaMalloc(&g.h1t, b32 * NH * sizeof(__nv_bfloat16)));
  QSGW_CUDA(cudaMalloc(&g.h2, b * NH * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.g1, b * NH * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.g2, b * NH * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.g2b, b * NH * sizeof(__nv_bfloat16)));
  QSGW_CUDA(cudaMalloc(&g.g2t, b32 * NH * sizeof(__nv_bfloat16)));
  QSGW_CUDA(cudaMalloc(&g.head, b * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.out, b * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.xb, b * NIN * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.yb, b * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.wb, b * sizeof(float)));
  QSGW_CUDA(cudaMalloc(&g.tb, b * sizeof(int)));
  g.cap = batch;
  return QSGW_OK;
}

static int grid_for(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 32LL * ctx().sm_count)));
}

// the 256 x 256 layer on the tensor cores: C = A Bt^T with one of the epilogues
template <int EPI>
static void mma_gemm(const __nv_bfloat16* A, long long lda, const __nv_bfloat16* Bt, long long ldb, int M, int K,
                     int ksplit, float* C, const __nv_bfloat16* bias, const __nv_bfloat16* mask, cudaStream_t s) {
  MmaArgs p{A, lda, Bt, ldb, M, NH, K, ksplit, C, NH, bias, mask};
  const dim3 grid(static_cast<unsigned>((M + 63) / 64), NH / 128, static_cast<unsigned>((K + ksplit - 1) / ksplit));
  mma_gemm_kernel<EPI><<<grid, 256, 0, s>>>(p);
  count_launch();
}

// forward pass of `batch` rows into g.out (training: also the transposed h1 for the weight gradient)
static void forward_pass(const float* x, const int* tix, int batch, bool train, const float* wt, cudaStream_t s) {
  const int nb = (batch + 31) / 32;
  forward_l1_kernel<<<nb, NH, 0, s>>>(x, tix, batch, g.w16, g.master, g.h1, train ? g.h1t : nullptr, ldt(), g.head,
                                      wt, train ? g.red + 1 : nullptr);
  mma_gemm<EPI_FWD>(g.h1, NH, g.w2t, NH, batch, NH, NH, g.h2, g.w16 + OFF_B2, nullptr, s);
  forward_l3_kernel<<<(batch + 7) / 8, 256, 0, s>>>(g.h2, tix, batch, g.w16, g.head, g.out);
  count_launch(2);
}

// forward + backward on (x, tix, y, wt) rows already on the device; gradient in g.grad, loss terms in g.red
static int grad_pass(const float* x, const int* tix, const float* y, const float* wt, int batch, cudaStream_t s) {
  QSGW_CUDA(cudaMemsetAsync(g.grad, 0, NPARAM * sizeof(float), s));
  QSGW_CUDA(cudaMemsetAsync(g.red, 0, 2 * sizeof(float), s));
  const int nb = (batch + 31) / 32;
  forward_pass(x, tix, batch, true, wt, s);
  backward_act_kernel<<<nb, NH, 0, s>>>(x, tix, y, wt, batch, g.w16, g.h2, g.out, g.g2, g.g2b, g.g2t, ldt(), g.grad,
                                        g.red);
  count_launch();
  // g1 = relu'(h1) (g2 W2^T): Bt = W2 itself ([k][j], k the output unit)
  mma_gemm<EPI_BWD>(g.g2b, NH, g.w16 + OFF_W2, NH, batch, NH, NH, g.g1, nullptr, g.h1, s);
  // dW2 = h1^T g2 over the batch (rows split in ranges of 1024)
  const int kpad = nb * 32;
  mma_gemm<EPI_WGRAD>(g.h1t, ldt(), g.g2t, ldt(), NH, kpad, 1024, g.grad + OFF_W2, nullptr, nullptr, s);
  const int rpb = 1024;
  const int nz = (batch + rpb - 1) / rpb;
  colsum_kernel<<<dim3(1, nz), NH, 0, s>>>(g.g2, batch, rpb, g.grad + OFF_B2);
  wgrad_kernel<<<dim3(1, NH / 32, (batch + 4095) / 4096), 256, 0, s>>>(x, NIN, g.g1, batch, 4096, g.grad + OFF_W1,
                                                                      g.grad + OFF_B1);
  count_launch(2);
  QSGW_LAUNCH_CHECK("wsurr gradient");
  return QSGW_OK;
}

// the BF16 weights and the transposed W2 from the FP32 master parameters
static void refresh_bf16(cudaStream_t s) {
  to_bf16_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(g.master, g.w16);
  w2t_kernel<<<(NH * NH + 255) / 256, 256, 0, s>>>(g.w16, g.w2t);
  count_launch(2);
}

static int adam_step(float lr, cudaStream_t s) {
  g.step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, static_cast<float>(g.step));
  const float c2 = 1.f - std::pow(b2, static_cast<float>(g.step));
  adam_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(g.master, g.grad, g.m1, g.m2, g.w16, lr, b1, b2, c1, c2, 1e-8f);
  w2t_kernel<<<(NH * NH + 255) / 256, 256, 0, s>>>(g.w16, g.w2t);
  count_launch(2);
  QSGW_LAUNCH_CHECK("wsurr adam");
  return QSGW_OK;
}

// host loss = sum w e^2 / sum w (or mean e^2 without weights)
static int read_loss(float* loss_host, int batch, bool weighted, cudaStream_t s) {
  float red[2];
  QSGW_CUDA(cudaMemcpyAsync(red, g.red, sizeof(red), cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  *loss_host = weighted ? red[0] / std::max(red[1], 1e-30f) : red[0] / batch;
  return QSGW_OK;
}

static int device_table(DevBuf& buf, const std::vector<int>& ints, const std::vector<float>& floats, int** di,
                        float** df, cudaStream_t s) {
  const size_t bi = ints.size() * sizeof(int), bfl = floats.size() * sizeof(float);
  int rc = buf.ensure(bi + bfl + 16);
  if (rc) return rc;
  *di = buf.as<int>();
  *df = reinterpret_cast<float*>(buf.as<char>() + ((bi + 15) / 16) * 16);
  if (bi) QSGW_CUDA(cudaMemcpyAsync(*di, ints.data(), bi, cudaMemcpyHostToDevice, s));
  if (bfl) QSGW_CUDA(cudaMemcpyAsync(*df, floats.data(), bfl, cudaMemcpyHostToDevice, s));
  // the host vectors die on return: make the copies complete first
  QSGW_CUDA(cudaStreamSynchronize(s));
  return QSGW_OK;
}

}  // namespace ws
}  // namespace qsgw

using namespace qsgw;
using namespace qsgw::ws;

extern "C" int qsgw_wsurr_init(unsigned long long seed) {
  int rc = require_init();
  if (rc) return rc;
  if (!g.ready) {
    QSGW_CUDA(cudaMalloc(&g.master, NPARAM * sizeof(float)));
    QSGW_CUDA(cudaMalloc(&g.w16, NPARAM * sizeof(__nv_bfloat16)));
    QSGW_CUDA(cudaMalloc(&g.w2t, NH * NH * sizeof(__nv_bfloat16)));
    QSGW_CUDA(cudaMalloc(&g.grad, NPARAM * sizeof(float)));
    QSGW_CUDA(cudaMalloc(&g.m1, NPARAM * sizeof(float)));
    QSGW_CUDA(cudaMalloc(&g.m2, NPARAM * sizeof(float)));
    QSGW_CUDA(cudaMalloc(&g.red, 2 * sizeof(float)));
    QSGW_CUDA(cudaMalloc(&g.lsq, NTMAX * (NIN * NIN + NIN) * sizeof(double)));
    g.ready = true;
  }
  QSGW_CUDA(cudaMemsetAsync(g.lsq, 0, NTMAX * (NIN * NIN + NIN) * sizeof(double), ctx().stream));
  cudaStream_t s = ctx().stream;
  init_params_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(g.master, seed);
  count_launch();
  refresh_bf16(s);
  QSGW_CUDA(cudaMemsetAsync(g.m1, 0, NPARAM * sizeof(float), s));
  QSGW_CUDA(cudaMemsetAsync(g.m2, 0, NPARAM * sizeof(float), s));
  g.step = 0;
  QSGW_LAUNCH_CHECK("wsurr init");
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_nparam(void) { return NPARAM; }

extern "C" int qsgw_wsurr_params(float* host, int set) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(g.ready && host, "wsurr: call qsgw_wsurr_init first");
  cudaStream_t s = ctx().stream;
  if (set) {
    QSGW_CUDA(cudaMemcpyAsync(g.master, host, NPARAM * sizeof(float), cudaMemcpyHostToDevice, s));
    refresh_bf16(s);
    QSGW_LAUNCH_CHECK("wsurr params");
  } else {
    QSGW_CUDA(cudaMemcpyAsync(host, g.master, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  QSGW_CUDA(cudaStreamSynchronize(s));
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_project_d(const double* wc_d, int ld, int nslot, const int* ridx, const int* cidx, int nb,
                                    float* proj_d) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(wc_d && ridx && proj_d && nb >= 1 && nslot >= 1, "wsurr_project: bad arguments");
  if (!cidx) cidx = ridx;
  for (int i = 0; i < nb; ++i)
    QSGW_ARG(ridx[i] >= 0 && ridx[i] < ld && cidx[i] >= 0 && cidx[i] < ld, "wsurr_project: index %d out of range", i);
  cudaStream_t s = ctx().stream;
  static DevBuf tab;
  int* di;
  float* df;
  std::vector<int> ints(ridx, ridx + nb);
  ints.insert(ints.end(), cidx, cidx + nb);
  rc = device_table(tab, ints, {}, &di, &df, s);
  if (rc) return rc;
  project_kernel<<<grid_for(static_cast<long long>(nslot) * nb * nb), 256, 0, s>>>(
      reinterpret_cast<const double2*>(wc_d), ld, nslot, di, di + nb, nb, proj_d);
  count_launch();
  QSGW_LAUNCH_CHECK("wsurr project");
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_features_d(const float* proj_d, int nq, int nw, int ne, const int* anchors, int na,
                                     const int* targets, const int* thead, int nt, const float* xcoord,
                                     const int* rid, const int* cid, int nb, const float* ftab, int nftab,
                                     float* x_d, int* tix_d, float* y_d, float* wgt_d, float* scale_d) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(proj_d && anchors && targets && thead && xcoord && x_d && tix_d && nq >= 1 && ne >= 1 && na >= 1 &&
               na + 6 <= NIN && nt >= 1,
           "wsurr_features: bad arguments (1 <= na <= %d)", NIN - 6);
  if (ftab) {
    QSGW_ARG(rid && cid && nb >= 1 && ne == 2 * nb * nb, "wsurr_features: element features need rid, cid and "
             "ne = 2 nb^2 (ne=%d nb=%d)", ne, nb);
    for (int i = 0; i < nb; ++i)
      QSGW_ARG(rid[i] >= 0 && rid[i] < nftab && cid[i] >= 0 && cid[i] < nftab, "wsurr_features: index %d", i);
  }
  for (int i = 0; i < na; ++i) QSGW_ARG(anchors[i] >= 0 && anchors[i] < nw, "wsurr_features: anchor %d", anchors[i]);
  for (int i = 0; i < nt; ++i) {
    QSGW_ARG(targets[i] >= 0 && targets[i] < nw, "wsurr_features: target %d", targets[i]);
    QSGW_ARG(thead[i] >= 0 && thead[i] < NTMAX, "wsurr_features: head slot %d (max %d)", thead[i], NTMAX);
  }
  cudaStream_t s = ctx().stream;
  std::vector<int> ints(anchors, anchors + na);
  ints.insert(ints.end(), targets, targets + nt);
  ints.insert(ints.end(), thead, thead + nt);
  std::vector<float> floats(xcoord, xcoord + nw);
  if (ftab) {
    ints.insert(ints.end(), rid, rid + nb);
    ints.insert(ints.end(), cid, cid + nb);
    floats.insert(floats.end(), ftab, ftab + nftab);
  }
  static DevBuf tab;
  int* di;
  float* df;
  rc = device_table(tab, ints, floats, &di, &df, s);
  if (rc) return rc;
  const int* drid = ftab ? di + na + 2 * nt : nullptr;
  features_kernel<<<grid_for(static_cast<long long>(nq) * ne * nt), 256, 0, s>>>(
      proj_d, nq, nw, ne, di, na, di + na, di + na + nt, nt, df, drid, ftab ? drid + nb : nullptr, nb,
      ftab ? df + nw : nullptr, x_d, tix_d, y_d, wgt_d, scale_d);
  count_launch();
  QSGW_LAUNCH_CHECK("wsurr features");
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_forward_d(const float* x_d, const int* tix_d, float* y_d, int batch) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(g.ready && x_d && tix_d && y_d && batch >= 0, "wsurr_forward: bad arguments");
  if (batch == 0) return QSGW_OK;
  cudaStream_t s = ctx().stream;
  // chunks of at most 2^16 rows through the activation buffers
  rc = ensure_cap(std::max(g.cap, std::min(batch, 1 << 16)));
  if (rc) return rc;
  const int chunk = g.cap;
  for (int b0 = 0; b0 < batch; b0 += chunk) {
    const int nb = std::min(chunk, batch - b0);
    forward_pass(x_d + static_cast<long long>(b0) * NIN, tix_d + b0, nb, false, nullptr, s);
    QSGW_CUDA(cudaMemcpyAsync(y_d + b0, g.out, nb * sizeof(float), cudaMemcpyDeviceToDevice, s));
  }
  QSGW_LAUNCH_CHECK("wsurr forward");
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_grad_d(const float* x_d, const int* tix_d, const float* y_d, const float* wgt_d, int batch,
                                 float* loss_host, float* grad_host) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(g.ready && x_d && tix_d && y_d && batch >= 1, "wsurr_grad: bad arguments");
  rc = ensure_cap(batch);
  if (rc) return rc;
  cudaStream_t s = ctx().stream;
  rc = grad_pass(x_d, tix_d, y_d, wgt_d, batch, s);
  if (rc) return rc;
  if (grad_host) QSGW_CUDA(cudaMemcpyAsync(grad_host, g.grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (loss_host) return read_loss(loss_host, batch, wgt_d != nullptr, s);
  QSGW_CUDA(cudaStreamSynchronize(s));
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_train_d(const float* x_d, const int* tix_d, const float* y_d, const float* wgt_d,
                                  long long n, int batch, int nsteps, float lr, unsigned long long seed,
                                  float* loss_host) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(g.ready && x_d && tix_d && y_d && n >= 1 && batch >= 1 && nsteps >= 0 && lr > 0.f,
           "wsurr_train: bad arguments");
  rc = ensure_cap(batch);
  if (rc) return rc;
  cudaStream_t s = ctx().stream;
  for (int it = 0; it < nsteps; ++it) {
    gather_batch_kernel<<<(batch + 255) / 256, 256, 0, s>>>(x_d, tix_d, y_d, wgt_d, n, batch, seed, g.step, g.xb,
                                                           g.tb, g.yb, g.wb);
    count_launch();
    rc = grad_pass(g.xb, g.tb, g.yb, g.wb, batch, s);
    if (rc) return rc;
    rc = adam_step(lr, s);
    if (rc) return rc;
  }
  if (loss_host) {
    if (nsteps == 0) {
      *loss_host = 0.f;
      return QSGW_OK;
    }
    return read_loss(loss_host, batch, true, s);
  }
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_head_full_d(double* wc_d, int n, int ld, int nslot, const int* aslot, int na,
                                      const int* tslot, const int* thead, const float* txc, int nt,
                                      const float* ftab) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(g.ready && wc_d && aslot && tslot && thead && txc && n >= 1 && ld >= n && na >= 1 && na + 6 <= NIN &&
               nt >= 1,
           "wsurr_head_full: bad arguments");
  for (int a = 0; a < na; ++a) QSGW_ARG(aslot[a] >= 0 && aslot[a] < nslot, "wsurr_head_full: anchor slot %d", aslot[a]);
  for (int i = 0; i < nt; ++i) {
    QSGW_ARG(tslot[i] >= 0 && tslot[i] < nslot, "wsurr_head_full: target slot %d", tslot[i]);
    QSGW_ARG(thead[i] >= 0 && thead[i] < NTMAX, "wsurr_head_full: head slot %d", thead[i]);
    for (int a = 0; a < na; ++a) QSGW_ARG(tslot[i] != aslot[a], "wsurr_head_full: target slot %d is an anchor", tslot[i]);
  }
  cudaStream_t s = ctx().stream;
  std::vector<int> ints(aslot, aslot + na);
  ints.insert(ints.end(), tslot, tslot + nt);
  ints.insert(ints.end(), thead, thead + nt);
  static DevBuf tab;
  int* di;
  float* df;
  std::vector<float> floats(txc, txc + nt);
  if (ftab) floats.insert(floats.end(), ftab, ftab + n);
  rc = device_table(tab, ints, floats, &di, &df, s);
  if (rc) return rc;
  head_full_kernel<<<grid_for(2LL * n * n), 256, 0, s>>>(reinterpret_cast<double2*>(wc_d), n, ld, di, na, di + na,
                                                         di + na + nt, df, nt, ftab ? df + nt : nullptr, g.master);
  count_launch();
  QSGW_LAUNCH_CHECK("wsurr head_full");
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_scatter_d(double* wc_d, int ld, int nslot, const int* idx, int nb, const int* tslot,
                                    int nt, const float* pred_d, const float* scale_d) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(wc_d && idx && tslot && pred_d && scale_d && nb >= 1 && ld >= nb && nt >= 1, "wsurr_scatter: bad arguments");
  for (int i = 0; i < nb; ++i) QSGW_ARG(idx[i] >= 0 && idx[i] < ld, "wsurr_scatter: idx[%d]=%d", i, idx[i]);
  for (int i = 0; i < nt; ++i) QSGW_ARG(tslot[i] >= 0 && tslot[i] < nslot, "wsurr_scatter: target slot %d", tslot[i]);
  cudaStream_t s = ctx().stream;
  std::vector<int> ints(idx, idx + nb);
  ints.insert(ints.end(), tslot, tslot + nt);
  static DevBuf tab;
  int* di;
  float* df;
  rc = device_table(tab, ints, {}, &di, &df, s);
  if (rc) return rc;
  scatter_block_kernel<<<grid_for(2LL * nb * nb * nt), 256, 0, s>>>(reinterpret_cast<double2*>(wc_d), ld, di, nb,
                                                                    di + nb, nt, pred_d, scale_d);
  count_launch();
  QSGW_LAUNCH_CHECK("wsurr scatter");
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_lsq_accumulate_d(const float* x_d, const float* y_d, const float* wgt_d, long long n, int nt,
                                           const int* thead) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(g.ready && x_d && y_d && thead && n >= 1 && nt >= 1 && nt <= 65535, "wsurr_lsq_accumulate: bad arguments");
  for (int i = 0; i < nt; ++i)
    QSGW_ARG(thead[i] >= 0 && thead[i] < NTMAX, "wsurr_lsq_accumulate: head row %d", thead[i]);
  cudaStream_t s = ctx().stream;
  static DevBuf tab;
  int* di;
  float* df;
  rc = device_table(tab, std::vector<int>(thead, thead + nt), {}, &di, &df, s);
  if (rc) return rc;
  const long long per_target = (n + nt - 1) / nt;
  const long long per_block = 4096;
  const long long nbx = (per_target + per_block - 1) / per_block;
  QSGW_ARG(nbx <= 2147483647LL, "wsurr_lsq_accumulate: too many samples");
  lsq_accumulate_kernel<<<dim3(static_cast<unsigned>(nbx), nt), 256, 0, s>>>(x_d, y_d, wgt_d, n, nt, di, per_block,
                                                                            g.lsq, g.lsq + NTMAX * NIN * NIN);
  count_launch();
  QSGW_LAUNCH_CHECK("wsurr lsq_accumulate");
  return QSGW_OK;
}

extern "C" int qsgw_wsurr_lsq_solve(double ridge, int* rows_solved) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(g.ready && ridge >= 0.0, "wsurr_lsq_solve: bad arguments");
  cudaStream_t s = ctx().stream;
  std::vector<double> eq(NTMAX * (NIN * NIN + NIN));
  std::vector<float> p(NPARAM);
  QSGW_CUDA(cudaMemcpyAsync(eq.data(), g.lsq, eq.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaMemcpyAsync(p.data(), g.master, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  int solved = 0;
  for (int h = 0; h < NTMAX; ++h) {
    double* G = eq.data() + h * NIN * NIN;
    double* H = eq.data() + NTMAX * NIN * NIN + h * NIN;
    double tr = 0.0;
    for (int i = 0; i < NIN; ++i) tr += G[i * NIN + i];
    if (!(tr > 0.0)) continue;
    const double lam = ridge * tr / NIN;
    for (int i = 0; i < NIN; ++i) G[i * NIN + i] += (G[i * NIN + i] > 0.0) ? lam : 1.0;   // unused features -> 0
    if (!chol_solve(G, H, NIN)) continue;
    for (int i = 0; i < NIN; ++i) p[OFF_C + h * NIN + i] = static_cast<float>(H[i]);
    ++solved;
  }
  QSGW_CUDA(cudaMemcpyAsync(g.master, p.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice, s));
  refresh_bf16(s);
  QSGW_CUDA(cudaMemsetAsync(g.lsq, 0, eq.size() * sizeof(double), s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  QSGW_LAUNCH_CHECK("wsurr lsq_solve");
  if (rows_solved) *rows_solved = solved;
  return QSGW_OK;
}
