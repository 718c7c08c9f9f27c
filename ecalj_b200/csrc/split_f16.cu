// Split-FP16 complex contractions on the 5th-generation tensor cores
// (tcgen05.mma kind::f16, FP32 accumulators in TMEM, TMA-fed shared memory).
//
// A complex product C = A B is run as one real GEMM with the M dimension
// doubled and K interleaved (k' = 2k + {re, im}):
//     rows (m, re) of A' = [Re a, -Im a],   rows (m, im) of A' = [Im a, Re a]
//     row n of B'       = [Re b,  Im b]   (K-major)
// so lanes 0..63 of a 128-lane accumulator hold Re C and lanes 64..127 Im C.
// Every FP64 operand is split into two scaled FP16 slices x = hi + lo
// (22 significant bits); the product keeps hi*hi + hi*lo + lo*hi (the lo*lo
// term, ~2^-22 relative, is dropped) and accumulates in FP32.
//
// The weight that differs per frequency (chi0, x0gemm.f90:84) or per
// segment and column (Sigma_c, m_sxcf_gemm.f90:485) multiplies B.  A' and
// the B source are pre-split once into HBM and streamed by TMA.  chi0: eight
// converter warps apply the frequency weight to the B source in shared
// memory and re-split it into B' for every frequency, while one thread issues
// the MMAs.  Sigma_c: S itself is the B operand and the drain applies the
// per-(segment, column) weight to each segment's FP32 sum in FP64.  Warp
// roles (576 threads, one CTA per SM):
//     warp 0        TMA producer
//     warp 1        TMEM owner and MMA issuer
//     warps 2..9    chi0: B' converters (two threads per B' row); Sigma_c: drain
//     warps 10..17  drain: FP32 accumulators -> FP64 sums in TMEM -> output
// Every mbarrier wait is bounded; on time-out the CTA records an error,
// drains its own TMA and MMA work, frees TMEM and exits.
#include <cmath>
#include <cstdlib>
#include <vector>
#include "split_common.cuh"
#include "autotune.cuh"

namespace qsgw {
namespace tc {

// ------------------------------------------------------------------ the kernel
// One CTA = one output tile (64 complex rows x 128 columns) of one frequency
// (chi0) or of the Sigma_c column tile, over its K range.  FP32 accumulation
// in the tensor core truncates, so its error grows with the run length; the
// MMA thread therefore alternates two TMEM accumulators every DRAIN_PERIOD
// chunks (Sigma_c: every segment) while the drain warps fold the finished one
// into FP64 sums kept in
// TMEM (columns 256..511, two 32-bit words per value).
template <int MODE>
__global__ void __launch_bounds__(NTHREADS, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapS,
                      const Params p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  using L = Cfg<MODE>;
  constexpr int NST = L::NST;
  constexpr bool SEG = MODE == MODE_SEG;
  unsigned char* sA = sm + L::OFF_A;
  unsigned char* sS = sm + L::OFF_S;
  unsigned char* sB = sm + L::OFF_B;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::OFF_BAR);
  uint64_t* full = bar;                  // [NST] TMA -> MMA, converters
  uint64_t* empty = bar + NST;        // [NST] MMA -> TMA
  uint64_t* bfull = bar + 2 * NST;    // [NBUF] converters -> MMA
  uint64_t* bempty = bfull + NBUF;       // [NBUF] MMA -> converters
  uint64_t* accfull = bempty + NBUF;     // [2] MMA -> drain
  uint64_t* accempty = accfull + 2;      // [2] drain -> MMA
  uint64_t* done = accempty + 2;         // [1] every MMA of the CTA retired
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::OFF_MISC);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::OFF_MISC + 8);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // ---- work unit
  const int tileid = blockIdx.x;
  const int mt = tileid % p.ntm, nt = tileid / p.ntm;
  const int jw = blockIdx.y;                       // chi0: frequency index
  const int split = blockIdx.z;
  if (!SEG && p.herm && mt * BMC + BMC - 1 < nt * NC) return;   // strictly upper tile
  const int c0 = split * p.kch_per_split;
  const int c1 = min(p.kch_total, c0 + p.kch_per_split);
  int seg0 = 0, nseg = 0;
  if (SEG) {
    const int group = p.tile_group[nt];
    nseg = p.group_nseg[group];
    seg0 = p.group_seg_off[group];
  }
  const int nchunk = SEG ? nseg * p.cps : max(0, c1 - c0);
  const int cbeg = SEG ? 0 : c0;
  // accumulation periods of DRAIN_PERIOD chunks; Sigma_c periods never straddle a segment,
  // because the drain applies the segment's per-column weight to the period's sum
  // Sigma_c: one period per segment (its K is short: 2 ngb), so the drain has a whole
  // segment of MMA time to fold the previous one in
  const int sdp = SEG ? p.cps : DRAIN_PERIOD;                    // chunks per period
  const int pps = (p.cps + sdp - 1) / sdp;                       // periods per segment
  const int nper = SEG ? nseg * pps : (nchunk + DRAIN_PERIOD - 1) / DRAIN_PERIOD;

  if (tid == 0) {
    for (int i = 0; i < NST; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); }
    for (int i = 0; i < NBUF; ++i) { mbar_init(&bfull[i], NCONV); mbar_init(&bempty[i], 1); }
    // Sigma_c has no converters: their warps drain too (twice the drain warps)
    const int ndrain = SEG ? 2 * NDRAIN_WARPS : NDRAIN_WARPS;
    for (int i = 0; i < 2; ++i) { mbar_init(&accfull[i], 1); mbar_init(&accempty[i], ndrain); }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (nchunk > 0) {
    if (warp == 0 && lane == 0) {
      // ---------------- TMA producer
      const uint32_t bytes = 2 * SLICE_A + 2 * SLICE_S;
      int issued = 0;
      // Sigma_c: segment and chunk-in-segment advanced by counting (this thread is on the
      // critical path of every chunk: no divisions, one table load per segment)
      int sg = 0, cin = 0;
      int t = (SEG && nseg > 0) ? p.seg_slot[seg0] * p.tiles_per_slot + mt : 0;
      for (int c = 0; c < nchunk; ++c) {
        const int st = c % NST;
        if (c >= NST && !mbar_wait(&empty[st], ((c / NST) - 1) & 1, abort_flag)) break;
        issued = c + 1;
        mbar_expect_tx(&full[st], bytes);
        unsigned char* a = sA + st * 2 * SLICE_A;
        unsigned char* s = sS + st * 2 * SLICE_S;
        if (!SEG) {
          const int x = (cbeg + c) * KC;
          tma_load_4d(a, &mapA, &full[st], x, 0, 0, mt);
          tma_load_4d(a + SLICE_A, &mapA, &full[st], x, 0, 0, p.lo_tile_off + mt);
          tma_load_4d(s, &mapS, &full[st], x, 0, 0, 2 * nt);
          tma_load_4d(s + SLICE_S, &mapS, &full[st], x, 0, 0, p.lo_row_off + 2 * nt);
        } else {
          const int x = cin * KC;
          tma_load_4d(a, &mapA, &full[st], x, 0, 0, t);
          tma_load_4d(a + SLICE_A, &mapA, &full[st], x, 0, 0, p.lo_tile_off + t);
          tma_load_2d(s, &mapS, &full[st], x, nt * NC);
          tma_load_2d(s + SLICE_S, &mapS, &full[st], x, p.lo_row_off + nt * NC);
          if (++cin == p.cps) {
            cin = 0;
            if (++sg < nseg) t = p.seg_slot[seg0 + sg] * p.tiles_per_slot + mt;
          }
        }
      }
      for (int c = max(0, issued - NST); c < issued; ++c) mbar_drain(&full[c % NST], (c / NST) & 1);
    } else if (warp == 1 && lane == 0) {
      // ---------------- MMA issuer
      constexpr bool seg_mode = SEG;
      // counters instead of divisions, and descriptors built once: this thread's issue latency
      // paces the tensor pipe.  A descriptor's address field is the shared address / 16, so the
      // descriptor of (stage, slice, K step) is the base descriptor plus that offset / 16.
      const uint64_t dA0 = sw128_desc(smem_u32(sA));
      const uint64_t dB0 = seg_mode ? sw128_desc(smem_u32(sS)) : sw128_desc(smem_u32(sB));
      constexpr uint32_t A_ST = (2 * SLICE_A) >> 4, A_LO = SLICE_A >> 4;
      constexpr uint32_t B_ST = (2 * (seg_mode ? SLICE_S : SLICE_B)) >> 4, B_LO = (seg_mode ? SLICE_S : SLICE_B) >> 4;
      int per = 0, cin = 0, cin_p = 0, b = 0, bph = 0;
      for (int c = 0; c < nchunk && !*abort_flag; ++c) {
        const int st = c % NST;
        const int ab = per & 1;                      // accumulator of this period
        const bool first_of_period = cin_p == 0;
        const bool last_of_period = cin_p == sdp - 1 || c == nchunk - 1 || (seg_mode && cin == p.cps - 1);
        if (first_of_period && per >= 2 && !mbar_wait(&accempty[ab], ((per >> 1) - 1) & 1, abort_flag)) break;
        if (!mbar_wait(&full[st], (c / NST) & 1, abort_flag)) break;
        // chi0: B' = weight x S rebuilt by the converters; Sigma_c: B = S itself (its per-column
        // weight is applied to the FP32 period sums by the drain warps)
        if (!seg_mode && !mbar_wait(&bfull[b], bph, abort_flag)) break;
        tc_fence_after();
        const uint64_t a_hi = dA0 + static_cast<uint32_t>(st) * A_ST, a_lo = a_hi + A_LO;
        const uint64_t b_hi = dB0 + static_cast<uint32_t>(seg_mode ? st : b) * B_ST, b_lo = b_hi + B_LO;
        const uint32_t d = tmem + static_cast<uint32_t>(ab * NC);
#pragma unroll
        for (int kk = 0; kk < KC / 16; ++kk) {
          const uint32_t ko = kk * 2;                // 16 FP16 = 32 B along K = 2 descriptor units
          const uint32_t acc0 = (first_of_period && kk == 0) ? 0u : 1u;
          umma_f16(d, a_hi + ko, b_hi + ko, acc0);
          umma_f16(d, a_hi + ko, b_lo + ko, 1u);
          umma_f16(d, a_lo + ko, b_hi + ko, 1u);
        }
        if (!seg_mode) umma_commit(&bempty[b]);
        umma_commit(&empty[st]);
        if (last_of_period) umma_commit(&accfull[ab]);
        // advance: B' buffer, chunk in period / segment, period
        if (++b == NBUF) { b = 0; bph ^= 1; }
        ++cin_p;
        if (seg_mode && ++cin == p.cps) { cin = 0; cin_p = 0; ++per; }
        else if (cin_p == sdp) { cin_p = 0; ++per; }
      }
      // everything issued has retired before TMEM may be freed
      umma_commit(done);
      mbar_drain(done, 0);
    } else if (warp >= CONV_W0 && warp < DRAIN_W0 && !SEG) {
      // ---------------- converters (chi0): B' = weight * (S_hi + S_lo), re-split to FP16 hi/lo
      const int ctid = tid - 32 * CONV_W0;     // 0..255
      const int ct = ctid >> 1;                // row n of the tile
      const int h = ctid & 1;                  // which four of the eight 16-byte chunks
      float4 wn[4];                            // chi0: this thread's 16 weights of the next chunk
      auto load_w = [&](int c, float4 (&wv)[4]) {
        const long long k0 = static_cast<long long>(cbeg + c) * 32 + h * 16;
        const float4* src = reinterpret_cast<const float4*>(p.w32 + static_cast<long long>(jw) * p.w32_ld + k0);
#pragma unroll
        for (int i = 0; i < 4; ++i) wv[i] = __ldg(src + i);
      };
      load_w(0, wn);
      for (int c = 0; c < nchunk; ++c) {
        const int st = c % NST;
        float4 wc[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) wc[i] = wn[i];
        if (c + 1 < nchunk) load_w(c + 1, wn);      // prefetch while this chunk converts
        if (!mbar_wait_warp(&full[st], (c / NST) & 1, abort_flag)) break;
        const int b = c % NBUF;
        if (c >= NBUF && !mbar_wait_warp(&bempty[b], ((c / NBUF) - 1) & 1, abort_flag)) break;
        const unsigned char* s_hi = sS + st * 2 * SLICE_S;
        const unsigned char* s_lo = s_hi + SLICE_S;
        unsigned char* d_hi = sB + b * 2 * SLICE_B;
        unsigned char* d_lo = d_hi + SLICE_B;
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const int ch = h * 4 + cc;
          const int off = sw128_off(ct, ch);
          const uint4 vh = *reinterpret_cast<const uint4*>(s_hi + off);
          const uint4 vl = *reinterpret_cast<const uint4*>(s_lo + off);
          const __half2* h2 = reinterpret_cast<const __half2*>(&vh);
          const __half2* l2 = reinterpret_cast<const __half2*>(&vl);
          uint4 oh, ol;
          __half2* oh2 = reinterpret_cast<__half2*>(&oh);
          __half2* ol2 = reinterpret_cast<__half2*>(&ol);
          const float wq[4] = {wc[cc].x, wc[cc].y, wc[cc].z, wc[cc].w};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            // the pair (re, im) of complex k = 4*ch + q
            // (S_hi + S_lo) w, then its FP16 hi and the FP16 of the remainder; the packed
            // FP32x2 operations round exactly as their scalar pairs
            const float2 f2 = make_float2(wq[q], wq[q]);
            const float2 v = __fmul2_rn(__fadd2_rn(__half22float2(h2[q]), __half22float2(l2[q])), f2);
            const __half2 hi = __float22half2_rn(v);
            const float2 fb = __half22float2(hi);
            oh2[q] = hi;
            ol2[q] = __float22half2_rn(__fadd2_rn(v, make_float2(-fb.x, -fb.y)));
          }
          *reinterpret_cast<uint4*>(d_hi + off) = oh;
          *reinterpret_cast<uint4*>(d_lo + off) = ol;
        }
        fence_async_smem();
        mbar_arrive(&bfull[b]);
      }
    } else if (warp >= DRAIN_W0 || (SEG && warp >= CONV_W0)) {
      // ---------------- drain: FP32 accumulator -> FP64 sums in TMEM, then the output.
      // chi0: warps 10..17, 64 columns each; Sigma_c: warps 2..17, 32 columns each.
      constexpr bool seg_mode = SEG;
      const int d = warp - (seg_mode ? CONV_W0 : DRAIN_W0);
      const int quad = warp & 3;                          // TMEM lanes 32*quad .. +31 (warp id mod 4)
      const int ncolw = seg_mode ? NC / 4 : NC / 2;       // columns of this warp
      const int c_lo = (d >> 2) * ncolw;                  // first column
      const uint32_t lane_base = static_cast<uint32_t>(quad * 32) << 16;
      bool ok = true;
      // Sigma_c: the segment's weights of this warp's columns, in the (then unused) B' area
      double* wsm = reinterpret_cast<double*>(sB + d * 64 * sizeof(double));
      int wseg = -1;
      for (int per = 0; per < nper; ++per) {
        const int ab = per & 1;
        if (seg_mode && per / pps != wseg) {              // a new segment: its per-column weights
          wseg = per / pps;
          const ZSeg zs = p.segs[seg0 + wseg];
          __syncwarp();                                   // the previous segment's reads are done
          for (int j = lane; j < ncolw; j += 32) {
            const int col = p.tile_cols[nt * NC + c_lo + j];
            wsm[j] = (col >= 0) ? zs.scale[static_cast<long long>(col) * zs.scale_cs] : 0.0;
          }
          __syncwarp();
        }
        if (!mbar_wait_warp(&accfull[ab], (per >> 1) & 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
#pragma unroll 1
        for (int cp = 0; cp < ncolw / 32; ++cp) {         // pairs of 16-column blocks
          uint32_t f32a[16], f32b[16], f64w[32];
          const int c0b = c_lo + cp * 32;
          tmem_ld16(tmem + lane_base + static_cast<uint32_t>(ab * NC + c0b), f32a);
          tmem_ld16(tmem + lane_base + static_cast<uint32_t>(ab * NC + c0b + 16), f32b);
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const uint32_t fcol = FP64_COL + static_cast<uint32_t>(2 * c0b + 32 * half);
            if (per > 0) tmem_ld32w(tmem + lane_base + fcol, f64w);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              double a0 = (per > 0) ? __hiloint2double(static_cast<int>(f64w[2 * i + 1]), static_cast<int>(f64w[2 * i])) : 0.0;
              const double v = static_cast<double>(__uint_as_float(half ? f32b[i] : f32a[i]));
              if (seg_mode) {                             // column cp*32 + half*16 + i of this warp's
                a0 = fma(v, wsm[cp * 32 + half * 16 + i], a0);
              } else {
                a0 += v;
              }
              f64w[2 * i] = static_cast<uint32_t>(__double2loint(a0));
              f64w[2 * i + 1] = static_cast<uint32_t>(__double2hiint(a0));
            }
            tmem_st32(tmem + lane_base + fcol, f64w);
          }
        }
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&accempty[ab]);
      }
      if (ok && !*abort_flag) {
        tc_fence_after();
        const int row = quad * 32 + lane;         // accumulator row: 0..63 re, 64..127 im
        const int m = mt * BMC + (row & 63);
        const bool im_part = row >= 64;
        double inv = 1.0 / (p.scales[0] * p.scales[1]);
        double2* Cj = p.C;
        if (!SEG) {
          inv /= p.scales[2 + jw];
          Cj = p.C + static_cast<long long>(jw) * p.c_bs;
        }                                           // Sigma_c: weights applied in FP64 above, no sigma_B
#pragma unroll 1
        for (int cb = 0; cb < ncolw / 16; ++cb) {
          uint32_t f64[32];
          const int cbase = c_lo + cb * 16;
          tmem_ld32w(tmem + lane_base + FP64_COL + static_cast<uint32_t>(2 * cbase), f64);
          tmem_wait_ld();
          if (m >= p.M) continue;
#pragma unroll 4
          for (int i = 0; i < 16; ++i) {
            const double v = __hiloint2double(static_cast<int>(f64[2 * i + 1]), static_cast<int>(f64[2 * i])) * inv;
            const int nloc = cbase + i;
            if (!SEG) {
              const int n = nt * NC + nloc;
              if (n >= p.N) continue;
              if (p.herm && m < n) continue;                // upper part comes from the mirror
              atomicAdd(reinterpret_cast<double*>(Cj + m + static_cast<long long>(n) * p.ldc) + (im_part ? 1 : 0), v);
              if (p.herm && m > n)                         // chi0(n, m) = conj(chi0(m, n))
                atomicAdd(reinterpret_cast<double*>(Cj + n + static_cast<long long>(m) * p.ldc) + (im_part ? 1 : 0),
                          im_part ? -v : v);
            } else {
              const long long col = p.tile_cols[nt * NC + nloc];
              if (col < 0) continue;
              atomicAdd(reinterpret_cast<double*>(Cj + m + col * p.ldc) + (im_part ? 1 : 0), v);
            }
          }
        }
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (*abort_flag && tid == 0) atomicExch(p.err, 2);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ------------------------------------------------------------------ pre-split kernels
__device__ __forceinline__ void split2(double x, double sig, __half& hi, __half& lo) {
  const double v = x * sig;
  hi = __double2half(v);
  lo = __double2half(v - static_cast<double>(__half2float(hi)));
}

// max |re|, |im| over a strided complex set -> atomicMax on the bit pattern
// max |Re|, |Im| over a (rows x cols, column stride ld): columns by block (x), a column's rows by
// thread, split over blockIdx.y when there are few columns; one atomic per block (256 threads)
__global__ void absmax_c128_kernel(const double2* __restrict__ a, long long rows, long long cols, long long ld,
                                   unsigned long long* out) {
  __shared__ double red[8];
  double m = 0.0;
  const long long rchunk = (rows + gridDim.y - 1) / gridDim.y;
  const long long r0 = blockIdx.y * rchunk, r1 = min(rows, r0 + rchunk);
  for (long long c = blockIdx.x; c < cols; c += gridDim.x) {
    const double2* col = a + c * ld;
    for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const double2 v = col[r];
      m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) m = fmax(m, red[w]);
    atomicMax(out, __double_as_longlong(m));
  }
}
static dim3 absmax_grid(long long rows, long long cols, int sms) {
  const long long gx = std::max<long long>(1, std::min<long long>(cols, 8LL * sms));
  const long long gy = std::max<long long>(1, std::min<long long>((rows + 1023) / 1024, (8LL * sms + gx - 1) / gx));
  return dim3(static_cast<unsigned>(gx), static_cast<unsigned>(std::min<long long>(gy, 65535)), 1);
}
__global__ void absmax_f64_rows_kernel(const double* __restrict__ a, long long n, long long stride, int nrow,
                                       unsigned long long* out) {
  // out[r] = max_i |a[r*stride + i]| for i < n
  const int r = blockIdx.y;
  double m = 0.0;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    m = fmax(m, fabs(a[r * stride + i]));
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && r < nrow) atomicMax(out + r, __double_as_longlong(m));
}
// power-of-two scales: sigma = 2^(target - ceil(log2(max)))
__global__ void make_scales_kernel(const unsigned long long* mx, double* scales, int n, int target0, int target_rest) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double m = __longlong_as_double(static_cast<long long>(mx[i]));
  const int t = (i < 2) ? target0 : target_rest;
  int e = 0;
  if (m > 0.0 && isfinite(m)) { frexp(m, &e); }      // m = f * 2^e, f in [0.5, 1)
  scales[i] = ldexp(1.0, t - e);
}

// A' of the M-doubled real GEMM from a complex getter, into
// [slice][slot*T + t][half][64][Kp] FP16 (slice 0 = hi, 1 = lo).
// getter 0 (chi0): a(m, k) = conj(Z[m + k*ld]);  getter 1 (Sigma_c): a(m, k) = conj(W_slot[k + m*ld]).
// Block (32, 8); the tile (slot, t) runs over blockIdx.y (grid-stride), (mm, k) over the block
// and blockIdx.x: getter 0 puts mm on threadIdx.x (Z columns are contiguous in m), getter 1 puts
// k on threadIdx.x (W rows are contiguous in k), so the loads coalesce.
template <int GET>
__global__ void presplit_a_kernel(__half* __restrict__ out, const double2* __restrict__ src, long long ld,
                                  long long slot_stride, int M, long long K, int T, int nslot, long long Kp,
                                  const double* __restrict__ scales, long long slice_elems, int slot_out0 = 0) {
  const double sig = scales[0];
  const long long KH = Kp / 2;
  for (long long st = blockIdx.y; st < static_cast<long long>(nslot) * T; st += gridDim.y) {
  const int t = static_cast<int>(st % T);
  const int slot = static_cast<int>(st / T);
  for (int it = 0; it < (GET == 0 ? 2 : 8); ++it) {
    int mm;
    long long k;
    if (GET == 0) { mm = threadIdx.x + 32 * it; k = blockIdx.x * 8LL + threadIdx.y; }
    else { mm = threadIdx.y + 8 * it; k = blockIdx.x * 32LL + threadIdx.x; }
    if (k >= KH) continue;
    const int m = t * 64 + mm;
    double ar = 0.0, ai = 0.0;
    if (m < M && k < K) {
      double2 v;
      if (GET == 0) v = src[m + k * ld];
      else v = src[slot * slot_stride + k + static_cast<long long>(m) * ld];
      ar = v.x; ai = -v.y;     // a = conj(v)
    }
    const long long row0 = ((static_cast<long long>(slot + slot_out0) * T + t) * 2 + 0) * 64 + mm;
    const long long row1 = row0 + 64;
    // half 0: [Re a, -Im a]; half 1: [Im a, Re a]; each pair is one 4-byte store per slice
    __half h0, l0, h1, l1;
    split2(ar, sig, h0, l0);
    split2(-ai, sig, h1, l1);
    *reinterpret_cast<__half2*>(out + row0 * Kp + 2 * k) = __halves2half2(h0, h1);
    *reinterpret_cast<__half2*>(out + slice_elems + row0 * Kp + 2 * k) = __halves2half2(l0, l1);
    split2(ai, sig, h0, l0);
    split2(ar, sig, h1, l1);
    *reinterpret_cast<__half2*>(out + row1 * Kp + 2 * k) = __halves2half2(h0, h1);
    *reinterpret_cast<__half2*>(out + slice_elems + row1 * Kp + 2 * k) = __halves2half2(l0, l1);
  }
  }
}
// chi0 A' from Z (getter 0 of presplit_a_kernel, one slot): block (32, 8) converts one 64-row tile t
// and 32 consecutive k.  The loads run along m (Z's columns are contiguous in m); the four half2 words
// of each element (row0 / row1 x hi / lo slice) are staged in shared memory, and the stores run
// along k, so a warp writes 128 contiguous bytes of one output row instead of 32 words 2 Kp bytes
// apart.  Writes the same halves as presplit_a_kernel<0>.
__global__ void presplit_z_kernel(__half* __restrict__ out, const double2* __restrict__ src, long long ld, int M,
                                  long long K, int T, long long Kp, const double* __restrict__ scales,
                                  long long slice_elems) {
  __shared__ __half2 st[4][64][33];          // [row0 hi, row0 lo, row1 hi, row1 lo][mm][k - k0]
  const double sig = scales[0];
  const long long KH = Kp / 2;
  const long long k0 = static_cast<long long>(blockIdx.x) * 32;
  for (int t = blockIdx.y; t < T; t += gridDim.y) {
    for (int j = 0; j < 4; ++j) {
      const int kk = threadIdx.y + 8 * j;
      const long long k = k0 + kk;
      for (int it = 0; it < 2; ++it) {
        const int mm = threadIdx.x + 32 * it;
        const int m = t * 64 + mm;
        double ar = 0.0, ai = 0.0;
        if (m < M && k < K) {
          const double2 v = src[m + k * ld];
          ar = v.x; ai = -v.y;     // a = conj(v)
        }
        // row0: [Re a, -Im a]; row1: [Im a, Re a]
        __half h0, l0, h1, l1;
        split2(ar, sig, h0, l0);
        split2(-ai, sig, h1, l1);
        st[0][mm][kk] = __halves2half2(h0, h1);
        st[1][mm][kk] = __halves2half2(l0, l1);
        split2(ai, sig, h0, l0);
        split2(ar, sig, h1, l1);
        st[2][mm][kk] = __halves2half2(h0, h1);
        st[3][mm][kk] = __halves2half2(l0, l1);
      }
    }
    __syncthreads();
    const long long k = k0 + threadIdx.x;
    if (k < KH) {
      for (int r = threadIdx.y; r < 64; r += 8) {
        const long long row0 = static_cast<long long>(t) * 128 + r, row1 = row0 + 64;
        *reinterpret_cast<__half2*>(out + row0 * Kp + 2 * k) = st[0][r][threadIdx.x];
        *reinterpret_cast<__half2*>(out + slice_elems + row0 * Kp + 2 * k) = st[1][r][threadIdx.x];
        *reinterpret_cast<__half2*>(out + row1 * Kp + 2 * k) = st[2][r][threadIdx.x];
        *reinterpret_cast<__half2*>(out + slice_elems + row1 * Kp + 2 * k) = st[3][r][threadIdx.x];
      }
    }
    __syncthreads();
  }
}

template <int GET>
static dim3 presplit_a_grid(long long Kp, long long tiles) {
  const long long KH = Kp / 2;
  const long long gx = (GET == 0) ? (KH + 7) / 8 : (KH + 31) / 32;
  return dim3(static_cast<unsigned>(gx), static_cast<unsigned>(std::min<long long>(tiles, 65535)), 1);
}

// B source rows (K-major): row r = column cols[r] of Z (k contiguous), [Re b, Im b] per k,
// into [slice][rows_pad][Kp]; cols == nullptr means row r = column r.
__global__ void presplit_s_kernel(__half* __restrict__ out, const double2* __restrict__ z, long long ld, long long K,
                                  const int* __restrict__ cols, long long nrows, long long ncols_valid, long long Kp,
                                  const double* __restrict__ scales, long long slice_elems) {
  // block (32, 8): k on threadIdx.x (z columns are contiguous in k), rows over threadIdx.y and
  // blockIdx.y (grid-stride)
  const double sig = scales[1];
  const long long k = blockIdx.x * 32LL + threadIdx.x;
  if (k >= Kp / 2) return;
  for (long long r = blockIdx.y * 8LL + threadIdx.y; r < nrows; r += 8LL * gridDim.y) {
    const long long c = cols ? cols[r] : (r < ncols_valid ? r : -1);
    double br = 0.0, bi = 0.0;
    if (c >= 0 && k < K) {
      const double2 v = z[k + c * ld];
      br = v.x; bi = v.y;
    }
    __half h0, l0, h1, l1;
    split2(br, sig, h0, l0);
    split2(bi, sig, h1, l1);
    *reinterpret_cast<__half2*>(out + r * Kp + 2 * k) = __halves2half2(h0, h1);
    *reinterpret_cast<__half2*>(out + slice_elems + r * Kp + 2 * k) = __halves2half2(l0, l1);
  }
}

// w32[iw][p] = w[iw*npair + p] * sigma_B(iw) (FP32), zero beyond npair
__global__ void scale_weights_kernel(float* __restrict__ w32, const double* __restrict__ w, long long npair,
                                     long long ld, int niw, const double* __restrict__ scales) {
  const long long tot = ld * niw;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long pr = e % ld;
    const int iw = static_cast<int>(e / ld);
    w32[e] = (pr < npair) ? static_cast<float>(w[iw * npair + pr] * scales[2 + iw]) : 0.f;
  }
}

// ------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}

int make_tensor_map(CUtensorMap* map, CUtensorMapDataType dtype, void* base, int rank, const cuuint64_t* dims,
                    const cuuint64_t* strides_bytes, const cuuint32_t* box, CUtensorMapSwizzle swz) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return QSGW_ERR_CUDA;
  }
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) {
    set_error("tensor map base is not 16-byte aligned");
    return QSGW_ERR_ARG;
  }
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = fn(map, dtype, rank, base, dims, strides_bytes, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", static_cast<int>(r));
    return QSGW_ERR_CUDA;
  }
  return QSGW_OK;
}

static int make_map(CUtensorMap* map, void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides_bytes,
                    const cuuint32_t* box, CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B) {
  return make_tensor_map(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, base, rank, dims, strides_bytes, box, swz);
}

static DevBuf g_a, g_s, g_mx, g_sc, g_tabs, g_w32;

template <int MODE>
static int launch_mode(const CUtensorMap& ma, const CUtensorMap& ms, const Params& p, dim3 grid, cudaStream_t s) {
  static uint64_t attr = 0;                       // one bit per device
  int rc = smem_limit_once(reinterpret_cast<const void*>(split_gemm_kernel<MODE>), Cfg<MODE>::SMEM_BYTES, attr);
  if (rc) return rc;
  split_gemm_kernel<MODE><<<grid, NTHREADS, Cfg<MODE>::SMEM_BYTES, s>>>(ma, ms, p);
  return QSGW_OK;
}

// Sigma_c kernel: 0 = one CTA per 64 x 128 tile, 1 = CTA pairs over 128-column tiles, 2 = one
// CTA per 64 x 256 tile (default, the fastest on B200).  QSGW_SIGC_KERNEL=<n> at load time or
// qsgw_set_sigc_kernel fixes it; otherwise the autotuner may pick it per shape (sigc_kind_use).
static int g_sigc_kind = -1;
static bool g_sigc_fixed = false;
static int sigc_kind() {
  if (g_sigc_kind < 0) {
    const char* e = std::getenv("QSGW_SIGC_KERNEL");
    g_sigc_fixed = e && (e[0] == '0' || e[0] == '1' || e[0] == '2') && e[1] == '\0';
    g_sigc_kind = g_sigc_fixed ? e[0] - '0' : 2;
  }
  return g_sigc_kind;
}

static int launch_split(const CUtensorMap& ma, const CUtensorMap& ms, const Params& p, dim3 grid, cudaStream_t s,
                        const char* tag) {
  const int pi = prof_begin(tag, s);
  const int rc = (p.mode == MODE_SEG) ? launch_mode<MODE_SEG>(ma, ms, p, grid, s) : launch_mode<MODE_CHI0>(ma, ms, p, grid, s);
  if (rc) return rc;
  prof_end(pi, s);
  count_launch();
  QSGW_LAUNCH_CHECK("split_gemm_kernel");
  return QSGW_OK;
}

static int grid1(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 32LL * ctx().sm_count)));
}

}  // namespace tc

using namespace tc;

int chi0_split_f16(double2* chi0, int npr, int niw, const double2* zcols, int ldz, long long npair, const double* w,
                   cudaStream_t s) {
  const int T = (npr + BMC - 1) / BMC;             // 64-row tiles of the basis
  const int Tn = (npr + NC - 1) / NC;              // 128-column tiles
  const long long Kp = ((2 * npair + KC - 1) / KC) * KC;
  // the S view reads pairs of A' tiles, so give A' an even tile count covering Tn*2
  const int Ta = std::max(T, 2 * Tn);
  const long long slice_elems = static_cast<long long>(Ta) * 128 * Kp;
  int rc = g_a.ensure(2 * slice_elems * sizeof(__half));
  if (rc) return rc;
  rc = g_mx.ensure((2 + niw) * sizeof(unsigned long long));
  if (rc) return rc;
  rc = g_sc.ensure((2 + niw) * sizeof(double));
  if (rc) return rc;
  unsigned long long* mx = g_mx.as<unsigned long long>();
  QSGW_CUDA(cudaMemsetAsync(mx, 0, (2 + niw) * sizeof(unsigned long long), s));
  absmax_c128_kernel<<<absmax_grid(npr, npair, ctx().sm_count), 256, 0, s>>>(zcols, npr, npair, ldz, mx);
  count_launch();
  QSGW_LAUNCH_CHECK("absmax_c128_kernel");
  QSGW_CUDA(cudaMemcpyAsync(mx + 1, mx, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s));
  absmax_f64_rows_kernel<<<dim3(64, niw), 256, 0, s>>>(w, npair, npair, niw, mx + 2);
  count_launch();
  QSGW_LAUNCH_CHECK("absmax_f64_rows_kernel");
  // A', S magnitudes <= 2^14; B' = S * w * sigma_B <= 2^15
  make_scales_kernel<<<(2 + niw + 63) / 64, 64, 0, s>>>(mx, g_sc.as<double>(), 2 + niw, 14, 1);
  count_launch();
  QSGW_LAUNCH_CHECK("make_scales_kernel");
  const long long w32_ld = Kp / 2;
  rc = g_w32.ensure(static_cast<size_t>(w32_ld) * niw * sizeof(float));
  if (rc) return rc;
  scale_weights_kernel<<<grid1(w32_ld * niw), 256, 0, s>>>(g_w32.as<float>(), w, npair, w32_ld, niw,
                                                           g_sc.as<double>());
  count_launch();
  QSGW_LAUNCH_CHECK("scale_weights_kernel");
  __half* a = g_a.as<__half>();
  QSGW_CUDA(cudaMemsetAsync(a, 0, 2 * slice_elems * sizeof(__half), s));
  presplit_z_kernel<<<dim3(static_cast<unsigned>((Kp / 2 + 31) / 32), static_cast<unsigned>(std::min(T, 65535))),
                      dim3(32, 8), 0, s>>>(a, zcols, ldz, npr, npair, T, Kp, g_sc.as<double>(), slice_elems);
  count_launch();
  QSGW_LAUNCH_CHECK("presplit_z_kernel");
  // maps: A' [Kp, 64, 2, 2*Ta] (hi tiles 0..Ta-1, lo tiles Ta..2Ta-1) box {64,64,2,1};
  //       S  same memory, half 0 of two consecutive tiles: box {64,64,1,2}
  CUtensorMap ma, ms;
  const cuuint64_t dims[4] = {static_cast<cuuint64_t>(Kp), 64, 2, static_cast<cuuint64_t>(2 * Ta)};
  const cuuint64_t str[3] = {static_cast<cuuint64_t>(Kp * 2), static_cast<cuuint64_t>(Kp * 2 * 64),
                             static_cast<cuuint64_t>(Kp * 2 * 128)};
  const cuuint32_t boxa[4] = {KC, 64, 2, 1};
  const cuuint32_t boxs[4] = {KC, 64, 1, 2};
  rc = make_map(&ma, a, 4, dims, str, boxa);
  if (rc) return rc;
  rc = make_map(&ms, a, 4, dims, str, boxs);
  if (rc) return rc;
  Params p{};
  p.mode = MODE_CHI0;
  p.M = npr; p.N = npr;
  p.ntm = T; p.ntn = Tn;
  p.tiles_per_slot = Ta;
  p.lo_tile_off = Ta;                       // lo slice = tiles Ta..2Ta-1 of the same map
  p.lo_row_off = Ta;
  p.herm = 1;                               // chi0(iw) is Hermitian: lower tiles + mirror
  p.kch_total = static_cast<int>(Kp / KC);
  p.w = w; p.npair = npair; p.niw = niw;
  p.w32 = g_w32.as<float>(); p.w32_ld = w32_ld;
  p.C = chi0; p.ldc = npr; p.c_bs = static_cast<long long>(npr) * npr;
  p.scales = g_sc.as<double>();
  p.err = ctx().d_flags + 1;
  // one frequency per CTA; split K only when the tiles alone cannot fill the GPU
  long long units = 0;
  for (int nt = 0; nt < Tn; ++nt)
    for (int mt = 0; mt < T; ++mt)
      if (mt * BMC + BMC - 1 >= nt * NC) ++units;
  units *= niw;
  const long long slots = 2LL * ctx().sm_count;
  const int maxsplit = std::max(1, p.kch_total / 8);
  int heur = static_cast<int>(std::max<long long>(1, (slots + units - 1) / units));
  heur = std::min(heur, maxsplit);
  // split K: the autotuner times 1..4 (and the heuristic) on this shape; each trial clears chi0
  auto run = [&](int splitk, bool clear) -> int {   // trials clear chi0; the caller cleared it or accumulates
    Params q = p;
    q.kch_per_split = (q.kch_total + splitk - 1) / splitk;
    const int sk = (q.kch_total + q.kch_per_split - 1) / q.kch_per_split;
    if (clear) QSGW_CUDA(cudaMemsetAsync(chi0, 0, static_cast<size_t>(npr) * npr * niw * sizeof(double2), s));
    return launch_split(ma, ms, q, dim3(static_cast<unsigned>(T * Tn), niw, sk), s, "chi0_tc");
  };
  std::vector<int> cands;
  for (int c = 1; c <= std::min(4, maxsplit); ++c) cands.push_back(c);
  if (heur > 4) cands.push_back(heur);
  char key[160];
  // pair counts within ~9% share a choice (they differ from q to q)
  std::snprintf(key, sizeof(key), "chi0_split_f16 npr=%d npair~2^%.3f niw=%d", npr,
                std::round(8.0 * std::log2(static_cast<double>(npair))) / 8.0, niw);
  int splitk = heur;
  bool tried = false;
  rc = tuned_choice(key, cands, heur, [&](int c) { return run(c, true); }, s, &splitk, &tried);
  if (rc) return rc;
  return run(splitk, tried);
}

int sigc_split_f16(const SigcSplitArgs& a, cudaStream_t s) {
  const int ngb = a.ngb;
  const int T = (ngb + BMC - 1) / BMC;
  const long long Kp = ((2LL * ngb + KC - 1) / KC) * KC;
  const int nslot = a.nimag + a.nreal;
  const int ntiles = static_cast<int>(a.tile_group.size());
  const int kind = sigc_kind();
  const int tw = (kind == 2) ? NW : NC;                   // columns per tile (as the tables were cut)
  QSGW_ARG(a.tile_cols.size() == static_cast<size_t>(ntiles) * tw, "sigc split: %zu tile columns for %d tiles of %d",
           a.tile_cols.size(), ntiles, tw);
  const long long nrows = static_cast<long long>(ntiles) * tw;
  const long long slice_a = static_cast<long long>(nslot) * T * 128 * Kp;
  const long long slice_s = nrows * Kp;
  int rc = g_a.ensure(2 * slice_a * sizeof(__half));
  if (rc) return rc;
  rc = g_s.ensure(2 * slice_s * sizeof(__half));
  if (rc) return rc;
  rc = g_mx.ensure(3 * sizeof(unsigned long long));
  if (rc) return rc;
  rc = g_sc.ensure(3 * sizeof(double));
  if (rc) return rc;
  unsigned long long* mx = g_mx.as<unsigned long long>();
  QSGW_CUDA(cudaMemsetAsync(mx, 0, 3 * sizeof(unsigned long long), s));
  // magnitudes: W stack (sigma_A), zmel (sigma_S), every weight (sigma_B)
  absmax_c128_kernel<<<absmax_grid(ngb, static_cast<long long>(ngb) * a.nimag, ctx().sm_count), 256, 0, s>>>(
      a.wi, ngb, static_cast<long long>(ngb) * a.nimag, a.ldw, mx);
  count_launch();
  if (a.nreal > 0) {
    absmax_c128_kernel<<<absmax_grid(ngb, static_cast<long long>(ngb) * a.nreal, ctx().sm_count), 256, 0, s>>>(
        a.wr, ngb, static_cast<long long>(ngb) * a.nreal, a.ldw, mx);
    count_launch();
  }
  absmax_c128_kernel<<<absmax_grid(ngb, a.ncol, ctx().sm_count), 256, 0, s>>>(a.zmel, ngb, a.ncol, ngb, mx + 1);
  count_launch();
  absmax_f64_rows_kernel<<<dim3(64, 1), 256, 0, s>>>(a.wgt, a.nwgt, 0, 1, mx + 2);
  count_launch();
  if (a.nw3 > 0) {
    absmax_f64_rows_kernel<<<dim3(16, 1), 256, 0, s>>>(a.w3, a.nw3, 0, 1, mx + 2);
    count_launch();
  }
  make_scales_kernel<<<1, 64, 0, s>>>(mx, g_sc.as<double>(), 3, 14, 1);
  count_launch();
  QSGW_LAUNCH_CHECK("sigc split scales");
  // pre-split A' slots: imag W first, then the symmetrised real-axis records
  __half* A = g_a.as<__half>();
  presplit_a_kernel<1><<<presplit_a_grid<1>(Kp, static_cast<long long>(a.nimag) * T), dim3(32, 8), 0, s>>>(
      A, a.wi, a.ldw, a.ldw * a.ldw, ngb, ngb, T, a.nimag, Kp, g_sc.as<double>(), slice_a, 0);
  count_launch();
  if (a.nreal > 0) {
    presplit_a_kernel<1><<<presplit_a_grid<1>(Kp, static_cast<long long>(a.nreal) * T), dim3(32, 8), 0, s>>>(
        A, a.wr, a.ldw, a.ldw * a.ldw, ngb, ngb, T, a.nreal, Kp, g_sc.as<double>(), slice_a, a.nimag);
    count_launch();
  }
  // B source rows in tile order (tile_cols, -1 = zero row)
  rc = g_tabs.ensure((a.tile_cols.size() + a.tile_group.size() + a.group_seg_off.size() + a.group_nseg.size() +
                      a.seg_slot.size() + 16) * sizeof(int) + a.segs.size() * sizeof(ZSeg) + 256);
  if (rc) return rc;
  unsigned char* tb = g_tabs.as<unsigned char>();
  size_t off = 0;
  int cprc = 0;
  auto put = [&](const void* src, size_t n) -> const void* {
    void* dst = tb + off;
    if (!cprc && n) cprc = h2d(dst, src, n, s);
    off += (n + 15) & ~size_t(15);
    return dst;
  };
  const ZSeg* d_segs = reinterpret_cast<const ZSeg*>(put(a.segs.data(), a.segs.size() * sizeof(ZSeg)));
  const int* d_cols = reinterpret_cast<const int*>(put(a.tile_cols.data(), a.tile_cols.size() * sizeof(int)));
  const int* d_tg = reinterpret_cast<const int*>(put(a.tile_group.data(), a.tile_group.size() * sizeof(int)));
  const int* d_gso = reinterpret_cast<const int*>(put(a.group_seg_off.data(), a.group_seg_off.size() * sizeof(int)));
  const int* d_gns = reinterpret_cast<const int*>(put(a.group_nseg.data(), a.group_nseg.size() * sizeof(int)));
  const int* d_slot = reinterpret_cast<const int*>(put(a.seg_slot.data(), a.seg_slot.size() * sizeof(int)));
  if (cprc) return cprc;
  __half* S = g_s.as<__half>();
  presplit_s_kernel<<<dim3(static_cast<unsigned>((Kp / 2 + 31) / 32),
                          static_cast<unsigned>(std::min<long long>((nrows + 7) / 8, 65535))),
                      dim3(32, 8), 0, s>>>(S, a.zmel, ngb, ngb, d_cols, nrows, 0, Kp,
                                                            g_sc.as<double>(), slice_s);
  count_launch();
  QSGW_LAUNCH_CHECK("sigc presplit");
  CUtensorMap ma, ms;
  const cuuint64_t dima[4] = {static_cast<cuuint64_t>(Kp), 64, 2, static_cast<cuuint64_t>(2LL * nslot * T)};
  const cuuint64_t stra[3] = {static_cast<cuuint64_t>(Kp * 2), static_cast<cuuint64_t>(Kp * 2 * 64),
                              static_cast<cuuint64_t>(Kp * 2 * 128)};
  // 64 x 256 tiles: 32-element K chunks in 64-byte swizzled rows; the others: 64 in 128-byte rows
  const int kch = (kind == 2) ? KCW : KC;
  const CUtensorMapSwizzle swz = (kind == 2) ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
  const cuuint32_t boxa[4] = {static_cast<cuuint32_t>(kch), 64, 2, 1};
  rc = make_map(&ma, A, 4, dima, stra, boxa, swz);
  if (rc) return rc;
  const cuuint64_t dims_[2] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(2 * nrows)};
  const cuuint64_t strs[1] = {static_cast<cuuint64_t>(Kp * 2)};
  // a CTA loads its whole S tile; a pair CTA half of it
  const cuuint32_t boxs[2] = {static_cast<cuuint32_t>(kch), static_cast<cuuint32_t>(kind == 1 ? NC / 2 : tw)};
  rc = make_map(&ms, S, 2, dims_, strs, boxs, swz);
  if (rc) return rc;
  Params p{};
  p.mode = MODE_SEG;
  p.M = ngb; p.N = 0;
  p.ntm = T; p.ntn = ntiles;
  p.cps = static_cast<int>(Kp / kch);
  p.kch_total = 0; p.kch_per_split = 0;
  p.tile_group = d_tg; p.tile_cols = d_cols; p.group_seg_off = d_gso; p.group_nseg = d_gns;
  p.seg_slot = d_slot; p.segs = d_segs;
  p.tiles_per_slot = T;
  p.lo_tile_off = nslot * T;
  p.lo_row_off = static_cast<int>(nrows);
  p.C = a.out; p.ldc = ngb; p.c_bs = 0;
  p.scales = g_sc.as<double>();
  p.err = ctx().d_flags + 1;
  QSGW_CUDA(cudaMemsetAsync(a.out, 0, static_cast<size_t>(ngb) * a.ncol * sizeof(double2), s));
  if (kind == 1) return launch_sigc_pair(ma, ms, p, dim3(static_cast<unsigned>(2 * ((T + 1) / 2) * ntiles), 1, 1), s, "sigc_seg_tc");
  dim3 grid(static_cast<unsigned>(T * ntiles), 1, 1);
  if (kind == 2) return launch_sigc_wide(ma, ms, p, grid, s, "sigc_seg_tc");
  return launch_split(ma, ms, p, grid, s, "sigc_seg_tc");
}

int sigc_split_tile_width() { return sigc_kind() == 2 ? NW : NC; }
bool sigc_kind_fixed() {
  sigc_kind();
  return g_sigc_fixed;
}
void sigc_kind_use(int kind) {
  sigc_kind();
  g_sigc_kind = kind;
}

}  // namespace qsgw

extern "C" int qsgw_set_sigc_kernel(int kind) {
  if (kind < 0 || kind > 2) {
    qsgw::set_error("qsgw_set_sigc_kernel: %d (0 = 64 x 128 tiles, 1 = CTA pairs, 2 = 64 x 256 tiles)", kind);
    return QSGW_ERR_ARG;
  }
  qsgw::tc::sigc_kind();
  qsgw::tc::g_sigc_kind = kind;
  qsgw::tc::g_sigc_fixed = true;
  return QSGW_OK;
}
