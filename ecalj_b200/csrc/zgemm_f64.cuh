// Complex FP64 GEMM engine on the FP64 tensor pipe (mma.sync m16n8k8 f64,
// "DMMA"), shared by chi0 (x0gemm), W (basis changes, Gauss-Jordan updates)
// and Sigma_c.  One CTA computes a 64x64 complex tile with 4 warps (each
// 32x32 = 2x4 m16n8 fragments, re and im accumulators); operands stream
// through a 3-stage cp.async pipeline in shared memory laid out [k][row]
// with a pitch of 66 complex (conflict-free fragment loads).  The m16n8k8
// shape does 4x the work of the m8n8k4 one per instruction with the same
// shared-memory reads per multiply-add.
//
// Three problem modes share the main loop:
//   ZM_GEMM  C = alpha op(A) op(B) + beta C, batched, optional split-K.
//   ZM_CHI0  per (jpm, iw) bin: C += sum_pairs conj(z) * w * z^T with the K
//            dimension gathered from a pair -> zmel-column list and the
//            weight applied while the B fragment is loaded (x0gemm.f90:72-89
//            without materialising zw / wzw); optional Hermitian tiling.
//   ZM_SEG   C(:, col) = sum_seg sum_k op(A_seg)(:, k) * s_seg(col) * Z(k, col)
//            over a gathered column list: the whole imaginary-axis sum of
//            Sigma_c (m_sxcf_gemm.f90:463-493) and the pole bins
//            (:556-590) in one launch, weights applied per column in the
//            B-fragment load.
#pragma once
#include "common.cuh"

namespace qsgw {

constexpr int ZG_BM = 64, ZG_BN = 64, ZG_BK = 16, ZG_STAGES = 3, ZG_THREADS = 128;
constexpr int ZG_PA = ZG_BM + 2, ZG_PB = ZG_BN + 2;

enum ZMode { ZM_GEMM = 0, ZM_CHI0 = 1, ZM_SEG = 2 };

struct ZSeg {
  const double2* mat;      // A operand of this segment
  const double* scale;     // per-column scale: scale[col * scale_cs]
  int scale_cs;
  int pad;
};

struct ZParams {
  int M, N, K;             // rows, cols, K (GEMM); K per segment (SEG)
  // A element (m, k) at A[m*a_rs + k*a_ks], B element (k, n) at B[n*b_rs + k*b_ks]
  const double2* A; long long a_rs, a_ks, a_bs; int a_conj;
  const double2* B; long long b_rs, b_ks, b_bs; int b_conj;
  double2* C; long long ldc, c_bs;
  double2 alpha, beta;
  int beta_zero;           // do not read C
  int splitk, kch_per_split;
  int ntm, ntn;            // tile counts
  // CHI0
  const int* bin_cnt; const long long* bin_coff; const long long* bin_woff;
  const int* bin_slab; const int* colidx; const double* wts; int herm;
  // SEG
  const int* tile_group; const int* tile_cols; const int* group_seg_off;
  const int* group_nseg; const ZSeg* segs;
};

struct ZSmem {
  double2 a[ZG_STAGES][ZG_BK][ZG_PA];
  double2 b[ZG_STAGES][ZG_BK][ZG_PB];
  double sk[ZG_STAGES][ZG_BK];
  double sn[ZG_STAGES][ZG_BN];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// D(16x8) += A(16x8) B(8x8), FP64.  Lane (g = lane / 4, t = lane % 4) holds A(g, t), A(g+8, t),
// A(g, t+4), A(g+8, t+4); B(t, g), B(t+4, g); D(g, 2t), D(g, 2t+1), D(g+8, 2t), D(g+8, 2t+1).
__device__ __forceinline__ void dmma16(double (&d)[4], const double (&a)[4], double b0, double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
}

// Decode the t-th lower-triangle tile (tm >= tn).
__device__ __forceinline__ void tri_decode(int t, int& tm, int& tn) {
  int r = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  while (r * (r + 1) / 2 > t) --r;
  tm = r;
  tn = t - r * (r + 1) / 2;
}

template <int MODE, bool A_RC, bool B_RC>
__global__ void __launch_bounds__(ZG_THREADS, 2) zgemm_f64_kernel(const ZParams p) {
  extern __shared__ __align__(16) unsigned char zg_smem_raw[];
  ZSmem& sm = *reinterpret_cast<ZSmem*>(zg_smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp & 1, wn = warp >> 1;

  // ---- per-CTA problem setup ----
  int tm = 0, tn = 0, batch = 0, split = 0, nchunk = 0, ch0 = 0, ch1 = 0;
  const double2* Ab = p.A;
  const double2* Bb = p.B;
  double2* Cb = p.C;
  const int* kcol = nullptr;      // CHI0: pair -> column
  const double* kw = nullptr;     // CHI0: pair weights
  int Kbin = 0;
  int group = 0, nseg = 0, seg0 = 0;
  int Mrows = p.M;
  if (MODE == ZM_GEMM) {
    tm = blockIdx.x % p.ntm; tn = blockIdx.x / p.ntm;
    batch = blockIdx.y; split = blockIdx.z;
    Ab += batch * p.a_bs; Bb += batch * p.b_bs; Cb += batch * p.c_bs;
    nchunk = (p.K + ZG_BK - 1) / ZG_BK;
  } else if (MODE == ZM_CHI0) {
    if (p.herm) tri_decode(blockIdx.x, tm, tn);
    else { tm = blockIdx.x % p.ntm; tn = blockIdx.x / p.ntm; }
    const int bin = blockIdx.y; split = blockIdx.z;
    Kbin = p.bin_cnt[bin];
    kcol = p.colidx + p.bin_coff[bin];
    kw = p.wts + p.bin_woff[bin];
    Cb += static_cast<long long>(p.bin_slab[bin]) * p.c_bs;
    nchunk = (Kbin + ZG_BK - 1) / ZG_BK;
  } else {
    tm = blockIdx.x; tn = blockIdx.y;
    group = p.tile_group[tn];
    nseg = p.group_nseg[group];
    seg0 = p.group_seg_off[group];
    nchunk = nseg * ((p.K + ZG_BK - 1) / ZG_BK);
  }
  ch0 = split * p.kch_per_split;
  ch1 = min(nchunk, ch0 + p.kch_per_split);
  if (MODE == ZM_SEG) { ch0 = 0; ch1 = nchunk; }
  const int m0 = tm * ZG_BM, n0 = tn * ZG_BN;
  const int kch_seg = (p.K + ZG_BK - 1) / ZG_BK;

  auto load_chunk = [&](int c, int st) {
    int kbase;
    const double2* Aseg = Ab;
    const double* sscale = nullptr;
    int scs = 0;
    if (MODE == ZM_SEG) {
      const int s = c / kch_seg;
      kbase = (c - s * kch_seg) * ZG_BK;
      const ZSeg sg = p.segs[seg0 + s];
      Aseg = sg.mat; sscale = sg.scale; scs = sg.scale_cs;
    } else {
      kbase = c * ZG_BK;
    }
    const int Klim = (MODE == ZM_CHI0) ? Kbin : p.K;
    // A operand: BK x BM elements, 8 per thread
#pragma unroll
    for (int i = 0; i < (ZG_BK * ZG_BM) / ZG_THREADS; ++i) {
      const int e = tid + i * ZG_THREADS;
      int r, kk;
      if (A_RC) { r = e % ZG_BM; kk = e / ZG_BM; } else { kk = e % ZG_BK; r = e / ZG_BK; }
      const int k = kbase + kk, m = m0 + r;
      bool ok = (k < Klim) && (m < Mrows);
      const double2* src = Aseg;
      if (ok) {
        long long kk_off;
        if (MODE == ZM_CHI0) kk_off = static_cast<long long>(__ldg(kcol + k));
        else kk_off = k;
        src = Aseg + m * p.a_rs + kk_off * p.a_ks;
      }
      cp_async16(&sm.a[st][kk][r], src, ok);
    }
    // B operand
#pragma unroll
    for (int i = 0; i < (ZG_BK * ZG_BN) / ZG_THREADS; ++i) {
      const int e = tid + i * ZG_THREADS;
      int r, kk;
      if (B_RC) { r = e % ZG_BN; kk = e / ZG_BN; } else { kk = e % ZG_BK; r = e / ZG_BK; }
      const int k = kbase + kk;
      bool ok = (k < Klim);
      const double2* src = Bb;
      if (MODE == ZM_SEG) {
        const int col = p.tile_cols[tn * ZG_BN + r];
        ok = ok && (col >= 0);
        if (ok) src = Bb + static_cast<long long>(col) * p.b_rs + static_cast<long long>(k) * p.b_ks;
      } else {
        const int n = n0 + r;
        ok = ok && (n < p.N);
        if (ok) {
          long long kk_off = (MODE == ZM_CHI0) ? static_cast<long long>(__ldg(kcol + k)) : k;
          src = Bb + n * p.b_rs + kk_off * p.b_ks;
        }
      }
      cp_async16(&sm.b[st][kk][r], src, ok);
    }
    if (MODE == ZM_CHI0) {
      if (tid < ZG_BK) {
        const int k = kbase + tid;
        sm.sk[st][tid] = (k < Kbin) ? __ldg(kw + k) : 0.0;
      }
    }
    if (MODE == ZM_SEG) {
      if (tid < ZG_BN) {
        const int col = p.tile_cols[tn * ZG_BN + tid];
        sm.sn[st][tid] = (col >= 0) ? __ldg(sscale + static_cast<long long>(col) * scs) : 0.0;
      }
    }
  };

  double accr[2][4][4], acci[2][4][4];       // [m16 block][n8 block][fragment element]
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) accr[i][j][e] = acci[i][j][e] = 0.0;

  const int nloc = ch1 - ch0;
#pragma unroll
  for (int s = 0; s < ZG_STAGES - 1; ++s) {
    if (s < nloc) load_chunk(ch0 + s, s);
    cp_async_commit();
  }
  for (int c = 0; c < nloc; ++c) {
    cp_async_wait<ZG_STAGES - 2>();
    __syncthreads();
    const int st = c % ZG_STAGES;
#pragma unroll
    for (int k8 = 0; k8 < ZG_BK / 8; ++k8) {
      const int ka = k8 * 8 + t, kb = ka + 4;       // the lane's two k of the step
      double ar[2][4], ai[2][4], nai[2][4], br[4][2], bi[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r0 = wm * 32 + i * 16 + g;
        const double2 v[4] = {sm.a[st][ka][r0], sm.a[st][ka][r0 + 8], sm.a[st][kb][r0], sm.a[st][kb][r0 + 8]};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          ar[i][e] = v[e].x;
          ai[i][e] = p.a_conj ? -v[e].y : v[e].y;
          nai[i][e] = -ai[i][e];
        }
      }
      double ska = 1.0, skb = 1.0;
      if (MODE == ZM_CHI0) { ska = sm.sk[st][ka]; skb = sm.sk[st][kb]; }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int nn = wn * 32 + j * 8 + g;
        const double2 va = sm.b[st][ka][nn], vb = sm.b[st][kb][nn];
        double sa = ska, sb = skb;
        if (MODE == ZM_SEG) sa = sb = sm.sn[st][nn];
        br[j][0] = va.x * sa;
        br[j][1] = vb.x * sb;
        bi[j][0] = (p.b_conj ? -va.y : va.y) * sa;
        bi[j][1] = (p.b_conj ? -vb.y : vb.y) * sb;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma16(accr[i][j], ar[i], br[j][0], br[j][1]);
          dmma16(accr[i][j], nai[i], bi[j][0], bi[j][1]);
          dmma16(acci[i][j], ar[i], bi[j][0], bi[j][1]);
          dmma16(acci[i][j], ai[i], br[j][0], br[j][1]);
        }
    }
    const int cn = c + ZG_STAGES - 1;
    if (cn < nloc) load_chunk(ch0 + cn, cn % ZG_STAGES);
    cp_async_commit();
  }
  cp_async_wait<0>();
  if (nloc <= 0 && (MODE != ZM_GEMM || p.splitk > 1) && MODE != ZM_SEG) return;

  // ---- epilogue ----
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
    const int row = m0 + wm * 32 + i * 16 + h * 8 + g;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int cl = wn * 32 + j * 8 + 2 * t + e;
        double vr = accr[i][j][2 * h + e], vi = acci[i][j][2 * h + e];
        if (MODE == ZM_GEMM) {
          const int col = n0 + cl;
          if (row >= p.M || col >= p.N) continue;
          double2* dst = Cb + row + col * p.ldc;
          const double r2 = p.alpha.x * vr - p.alpha.y * vi;
          const double i2 = p.alpha.x * vi + p.alpha.y * vr;
          if (p.splitk > 1) {
            atomicAdd(&dst->x, r2);
            atomicAdd(&dst->y, i2);
          } else if (p.beta_zero) {
            *dst = make_double2(r2, i2);
          } else {
            const double2 o = *dst;
            *dst = make_double2(r2 + p.beta.x * o.x - p.beta.y * o.y,
                                i2 + p.beta.x * o.y + p.beta.y * o.x);
          }
        } else if (MODE == ZM_CHI0) {
          const int col = n0 + cl;
          if (row >= p.M || col >= p.N) continue;
          double2* dst = Cb + row + col * p.ldc;
          if (p.splitk > 1) {
            atomicAdd(&dst->x, vr); atomicAdd(&dst->y, vi);
          } else {
            double2 o = *dst; o.x += vr; o.y += vi; *dst = o;
          }
          if (p.herm && tm != tn) {   // rcxq(col,row) += conj(acc(row,col))
            double2* d2 = Cb + col + static_cast<long long>(row) * p.ldc;
            if (p.splitk > 1) {
              atomicAdd(&d2->x, vr); atomicAdd(&d2->y, -vi);
            } else {
              double2 o = *d2; o.x += vr; o.y -= vi; *d2 = o;
            }
          }
        } else {
          const int col = p.tile_cols[tn * ZG_BN + cl];
          if (row >= p.M || col < 0) continue;
          double2* dst = Cb + row + static_cast<long long>(col) * p.ldc;
          if (p.beta_zero) *dst = make_double2(vr, vi);
          else { double2 o = *dst; o.x += vr; o.y += vi; *dst = o; }
        }
      }
  }
}

// Host launch helpers (defined in zgemm_f64.cu).
int zgemm_f64(int opa, int opb, int m, int n, int k, double2 alpha,
              const double2* A, long long lda, long long a_bs,
              const double2* B, long long ldb, long long b_bs, double2 beta,
              double2* C, long long ldc, long long c_bs, int nbatch, cudaStream_t s);
int zgemm_chi0_launch(ZParams p, int nbins, int herm, int splitk, cudaStream_t s);
// C(0:n, 0:n) += A^H B for complex A, B of K x n (column-major), n <= 64, any K (FP64 atomics)
int zgemm_hn_thin(int n, long long K, const double2* A, long long lda, const double2* B, long long ldb, double2* C,
                  long long ldc, cudaStream_t s);
int zgemm_seg_launch(ZParams p, int ncol_tiles, cudaStream_t s);
// Batched inverses (wv.cu: Hermitian positive definite; zminv_piv.cu: general, partial pivoting).
int zminv_hpd_batched(double2* A, int n, long long lda, long long a_bs, int nbatch, cudaStream_t s);
int zminv_general_batched(double2* A, int n, long long lda, long long a_bs, int nbatch, cudaStream_t s);

}  // namespace qsgw
