// Variants of the split-FP16 Sigma_c contraction (qsgw_set_sigc_kernel): 64 x
// 256 tiles (N = 256 MMAs with the FP64 period sums in a global scratch tile;
// the default) and CTA pairs (tcgen05 cta_group::2, opt-in).  Both compute the
// sums of the 64 x 128 kernel of split_f16.cu.
#include "split_common.cuh"

namespace qsgw {
namespace tc {

// ------------------------------------------------------------------ Sigma_c on 256-column tiles
// The Sigma_c contraction with N = 256 MMAs (64 complex rows x 256 columns per
// CTA): twice the work per instruction, four 48 KB stages of 32-element K
// chunks (64-byte swizzled rows).  The default Sigma_c kernel: measured on
// B200 (8 tasks of 600 x 600 at 1965 MHz) 29.05 ms against 30.5 ms for the
// 64 x 128 kernel, whose single MMA-issuing thread cannot keep up with
// 128 x 128 x 16 MMAs (about 80 clocks of issue per 64 clocks of math).  The
// drain loads the 16 previous sums of a column block before updating them (one
// L2 round trip instead of one per column).  The two FP32
// accumulators (one per segment, alternating) fill TMEM's 512 columns, so the
// FP64 sums over segments live in a per-CTA scratch tile in global memory
// (L2-resident while the CTA runs, [column][TMEM lane], coalesced per warp):
// the drain warps add weight x period sum into it in FP64 (the same fma order
// as the TMEM sums of the 128-column kernel) and the epilogue adds the tile
// into the output.
constexpr int WIDE_NST = 4;                      // four 48 KB stages
constexpr int SLICE_AW = BM2 * KCW * 2;          // 8 KB: one A' slice of a stage
constexpr int SLICE_SW = NW * KCW * 2;           // 16 KB: one S slice of a stage
struct WideCfg {
  static constexpr int OFF_A = 0;
  static constexpr int OFF_S = OFF_A + WIDE_NST * 2 * SLICE_AW;
  static constexpr int OFF_W = OFF_S + WIDE_NST * 2 * SLICE_SW;      // drain weights, 16 warps x 64 doubles
  static constexpr int OFF_BAR = OFF_W + 2 * NDRAIN_WARPS * 64 * 8;
  static constexpr int NBAR = 2 * WIDE_NST + 2 + 2 + 1;
  static constexpr int OFF_MISC = OFF_BAR + NBAR * 8;
  static constexpr int SMEM_BYTES = OFF_MISC + 64 + 1024;
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
};
// kind::f16, A = B = F16, D = F32, both K-major, M = 128, N = 256
constexpr uint32_t IDESC_W = (1u << 4) | (static_cast<uint32_t>(NW >> 3) << 17) | (static_cast<uint32_t>(BM2 >> 4) << 24);

__device__ __forceinline__ void umma_f16_w(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(IDESC_W), "r"(accumulate));
}

__global__ void __launch_bounds__(NTHREADS, 1)
    sigc_wide_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapS,
                     const Params p) {
  using L = WideCfg;
  constexpr int NST = WIDE_NST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = sm + L::OFF_A;
  unsigned char* sS = sm + L::OFF_S;
  unsigned char* sW = sm + L::OFF_W;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::OFF_BAR);
  uint64_t* full = bar;                  // [NST] TMA -> MMA
  uint64_t* empty = bar + NST;           // [NST] MMA -> TMA
  uint64_t* accfull = bar + 2 * NST;     // [2] MMA -> drain
  uint64_t* accempty = accfull + 2;      // [2] drain -> MMA
  uint64_t* done = accempty + 2;         // [1] every MMA of the CTA retired
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::OFF_MISC);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::OFF_MISC + 8);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int mt = blockIdx.x % p.ntm, nt = blockIdx.x / p.ntm;
  const int group = p.tile_group[nt];
  const int nseg = p.group_nseg[group];
  const int seg0 = p.group_seg_off[group];
  const int nchunk = nseg * p.cps;
  double* scr = p.scratch + static_cast<size_t>(blockIdx.x) * NW * BM2;   // [column][TMEM lane]

  if (tid == 0) {
    for (int i = 0; i < NST; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); }
    for (int i = 0; i < 2; ++i) { mbar_init(&accfull[i], 1); mbar_init(&accempty[i], 2 * NDRAIN_WARPS); }
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
      // ---------------- TMA producer: A' (hi, lo) of the segment's slot, S (hi, lo) of the tile
      constexpr uint32_t bytes = 2 * SLICE_AW + 2 * SLICE_SW;
      int issued = 0, sg = 0, cin = 0, st = 0, ph = 0;
      int t = p.seg_slot[seg0] * p.tiles_per_slot + mt;
      for (int c = 0; c < nchunk; ++c) {
        if (c >= NST && !mbar_wait(&empty[st], ph ^ 1, abort_flag)) break;
        issued = c + 1;
        mbar_expect_tx(&full[st], bytes);
        unsigned char* a = sA + st * 2 * SLICE_AW;
        unsigned char* s = sS + st * 2 * SLICE_SW;
        const int x = cin * KCW;
        tma_load_4d(a, &mapA, &full[st], x, 0, 0, t);
        tma_load_4d(a + SLICE_AW, &mapA, &full[st], x, 0, 0, p.lo_tile_off + t);
        tma_load_2d(s, &mapS, &full[st], x, nt * NW);
        tma_load_2d(s + SLICE_SW, &mapS, &full[st], x, p.lo_row_off + nt * NW);
        if (++cin == p.cps) {
          cin = 0;
          if (++sg < nseg) t = p.seg_slot[seg0 + sg] * p.tiles_per_slot + mt;
        }
        if (++st == NST) { st = 0; ph ^= 1; }
      }
      for (int c = max(0, issued - NST); c < issued; ++c) mbar_drain(&full[c % NST], (c / NST) & 1);
    } else if (warp == 1 && lane == 0) {
      // ---------------- MMA issuer: one accumulator per segment, alternating
      int seg = 0, cin = 0, st = 0, ph = 0;
      for (int c = 0; c < nchunk && !*abort_flag; ++c) {
        const int ab = seg & 1;
        const bool first = cin == 0, last = cin == p.cps - 1;
        if (first && seg >= 2 && !mbar_wait(&accempty[ab], ((seg >> 1) - 1) & 1, abort_flag)) break;
        if (!mbar_wait(&full[st], ph, abort_flag)) break;
        tc_fence_after();
        const uint32_t a_hi = smem_u32(sA + st * 2 * SLICE_AW), a_lo = a_hi + SLICE_AW;
        const uint32_t b_hi = smem_u32(sS + st * 2 * SLICE_SW), b_lo = b_hi + SLICE_SW;
        const uint32_t d = tmem + static_cast<uint32_t>(ab * NW);
#pragma unroll
        for (int kk = 0; kk < KCW / 16; ++kk) {
          const uint32_t ko = kk * 32;
          umma_f16_w(d, sw64_desc(a_hi + ko), sw64_desc(b_hi + ko), (first && kk == 0) ? 0u : 1u);
          umma_f16_w(d, sw64_desc(a_hi + ko), sw64_desc(b_lo + ko), 1u);
          umma_f16_w(d, sw64_desc(a_lo + ko), sw64_desc(b_hi + ko), 1u);
        }
        umma_commit(&empty[st]);
        if (last) umma_commit(&accfull[ab]);
        if (++st == NST) { st = 0; ph ^= 1; }
        if (++cin == p.cps) { cin = 0; ++seg; }
      }
      umma_commit(done);
      mbar_drain(done, 0);
    } else if (warp >= CONV_W0) {
      // ---------------- drain (warps 2..17): TMEM lanes 32 (warp mod 4) .. +31, 64 columns a warp
      const int dw = warp - CONV_W0;
      const int quad = warp & 3;
      const int c_lo = (dw >> 2) * 64;
      const int row = quad * 32 + lane;                   // accumulator row: 0..63 re, 64..127 im
      const uint32_t lane_base = static_cast<uint32_t>(quad * 32) << 16;
      double* wsm = reinterpret_cast<double*>(sW + dw * 64 * sizeof(double));
      bool ok = true;
      for (int seg = 0; seg < nseg; ++seg) {
        const int ab = seg & 1;
        const ZSeg zs = p.segs[seg0 + seg];
        __syncwarp();                                     // the previous segment's reads of wsm are done
        for (int j = lane; j < 64; j += 32) {
          const int col = p.tile_cols[nt * NW + c_lo + j];
          wsm[j] = (col >= 0) ? zs.scale[static_cast<long long>(col) * zs.scale_cs] : 0.0;
        }
        __syncwarp();
        if (!mbar_wait_warp(&accfull[ab], (seg >> 1) & 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
#pragma unroll 1
        for (int cb = 0; cb < 64; cb += 16) {
          // the 16 previous sums are loaded together (one L2 round trip), then updated
          uint32_t fa[16];
          double prev[16];
          tmem_ld16(tmem + lane_base + static_cast<uint32_t>(ab * NW + c_lo + cb), fa);
          double* q = scr + static_cast<size_t>(c_lo + cb) * BM2 + row;
          if (seg > 0) {
#pragma unroll
            for (int i = 0; i < 16; ++i) prev[i] = q[static_cast<size_t>(i) * BM2];
          }
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const double v = static_cast<double>(__uint_as_float(fa[i]));
            q[static_cast<size_t>(i) * BM2] = (seg == 0) ? v * wsm[cb + i] : fma(v, wsm[cb + i], prev[i]);
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&accempty[ab]);
      }
      if (ok && !*abort_flag) {
        const int m = mt * BMC + (row & 63);
        const bool im_part = row >= 64;
        const double inv = 1.0 / (p.scales[0] * p.scales[1]);
        if (m < p.M) {
#pragma unroll 4
          for (int j = 0; j < 64; ++j) {
            const long long col = p.tile_cols[nt * NW + c_lo + j];
            if (col < 0) continue;
            const double v = scr[static_cast<size_t>(c_lo + j) * BM2 + row] * inv;
            atomicAdd(reinterpret_cast<double*>(p.C + m + col * p.ldc) + (im_part ? 1 : 0), v);
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

// ------------------------------------------------------------------ Sigma_c on CTA pairs
// The same Sigma_c contraction on pairs of SMs (a cluster of two CTAs) with
// tcgen05.mma.cta_group::2: one MMA of M = 256 real rows (two 64-complex-row
// tiles, one per CTA) x N = 128 columns, each CTA holding its own A' rows and
// HALF of the B = S tile (64 columns) in shared memory.  Each SM thus loads
// 48 KB per K chunk instead of 64 KB for the same tensor work, and four stages
// fit.  Each CTA's TMA signals its own barrier; the follower's (idle) MMA warp
// forwards every landed stage to a second barrier of the leader, so each CTA
// can always wait for its own copies in flight.  The leader's MMA thread commits to the
// barriers of both CTAs; both CTAs' drain warps fold their own TMEM rows and
// arrive on the leader's accumulator-free barrier.  Measured on B200 (8 tasks
// of 600 x 600, 1965 MHz): 40.0 ms against 31.0 ms for one CTA per tile (35.2
// ms with the follower's TMA signalling the leader's barrier directly, which
// leaves the follower unable to wait for its own copies when a wait times
// out): the contraction is bound by the TMA -> MMA latency, not by L2 bytes,
// and the pair couples two SMs' pipelines.  So it is the opt-in variant.
constexpr int PAIR_NST = 4;
constexpr int SLICE_SH = (NC / 2) * KC * 2;       // 8 KB: this CTA's half of an S slice
struct PairCfg {
  static constexpr int OFF_A = 0;
  static constexpr int OFF_S = OFF_A + PAIR_NST * 2 * SLICE_A;
  static constexpr int OFF_W = OFF_S + PAIR_NST * 2 * SLICE_SH;      // drain weights, 16 warps x 64 doubles
  static constexpr int OFF_BAR = OFF_W + 2 * 8 * 64 * 8;
  static constexpr int NBAR = 3 * PAIR_NST + 2 + 2 + 1;
  static constexpr int OFF_MISC = OFF_BAR + NBAR * 8;
  static constexpr int SMEM_BYTES = OFF_MISC + 64 + 1024;
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
};
// kind::f16, A = B = F16, D = F32, both K-major, M = 256 (the pair), N = NC
constexpr uint32_t IDESC_PAIR = (1u << 4) | (static_cast<uint32_t>(NC >> 3) << 17) | (static_cast<uint32_t>(256 >> 4) << 24);

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// shared::cluster address of the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
  return a;
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_bar) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait with cluster-scope acquire (the arrivals come from the other CTA too)
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    if (mbar_try_cluster(b, parity)) return true;
    if (*abort_flag) return false;
    if (i > 64) __nanosleep(64);
  }
  *abort_flag = 1;
  return false;
}
__device__ __forceinline__ void mbar_drain_cluster(uint64_t* b, uint32_t parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    if (mbar_try_cluster(b, parity)) return;
    if (i > 64) __nanosleep(64);
  }
}
__device__ __forceinline__ bool mbar_wait_warp_cluster(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  int ok = 0;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait_cluster(b, parity, abort_flag) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void umma_f16_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(IDESC_PAIR), "r"(accumulate));
}
// arrive (when every MMA issued so far has completed) on a barrier of either CTA of the pair
__device__ __forceinline__ void umma_commit_pair(uint32_t cluster_bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(cluster_bar)
               : "memory");
}

__global__ void __launch_bounds__(NTHREADS, 1)
    split_pair_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapS,
                      const Params p) {
  using L = PairCfg;
  constexpr int NST = PAIR_NST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = sm + L::OFF_A;
  unsigned char* sS = sm + L::OFF_S;
  unsigned char* sW = sm + L::OFF_W;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::OFF_BAR);
  uint64_t* full = bar;                  // [NST] this CTA's TMA -> MMA (leader) / forwarder (follower)
  uint64_t* empty = bar + NST;           // [NST] MMA -> TMA, in both CTAs
  uint64_t* fwd = bar + 2 * NST;         // [NST] the follower's landed stages -> MMA (leader's)
  uint64_t* accfull = bar + 3 * NST;     // [2] MMA -> drain, in both CTAs
  uint64_t* accempty = accfull + 2;      // [2] drain warps of both CTAs -> MMA (the leader's)
  uint64_t* done = accempty + 2;         // [1] every MMA of the pair retired, in both CTAs
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::OFF_MISC);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::OFF_MISC + 8);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  // work unit: the pair covers row tiles 2 mp and 2 mp + 1 of column tile nt
  const int ntp = (p.ntm + 1) >> 1;
  const int pair = blockIdx.x >> 1;
  const int mt = 2 * (pair % ntp) + static_cast<int>(rank), nt = pair / ntp;
  const int group = p.tile_group[nt];
  const int nseg = p.group_nseg[group];
  const int seg0 = p.group_seg_off[group];
  const int nchunk = nseg * p.cps;

  if (tid == 0) {
    for (int i = 0; i < NST; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); mbar_init(&fwd[i], 1); }
    for (int i = 0; i < 2; ++i) { mbar_init(&accfull[i], 1); mbar_init(&accempty[i], 4 * NDRAIN_WARPS); }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {                       // one warp in each CTA of the pair, same offset
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  cluster_sync_all();                    // barriers of both CTAs initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (nchunk > 0) {
    if (warp == 0 && lane == 0) {
      // ---------------- TMA producer (both CTAs): own A' tile, own half of the S tile
      constexpr uint32_t bytes = 2 * SLICE_A + 2 * SLICE_SH;
      int issued = 0, sg = 0, cin = 0;
      int t = p.seg_slot[seg0] * p.tiles_per_slot + mt;
      const int srow = nt * NC + static_cast<int>(rank) * (NC / 2);
      for (int c = 0; c < nchunk; ++c) {
        const int st = c % NST;
        if (c >= NST && !mbar_wait_cluster(&empty[st], ((c / NST) - 1) & 1, abort_flag)) break;
        issued = c + 1;
        mbar_expect_tx(&full[st], bytes);
        unsigned char* a = sA + st * 2 * SLICE_A;
        unsigned char* s = sS + st * 2 * SLICE_SH;
        const int x = cin * KC;
        tma_load_4d(a, &mapA, &full[st], x, 0, 0, t);
        tma_load_4d(a + SLICE_A, &mapA, &full[st], x, 0, 0, p.lo_tile_off + t);
        tma_load_2d(s, &mapS, &full[st], x, srow);
        tma_load_2d(s + SLICE_SH, &mapS, &full[st], x, p.lo_row_off + srow);
        if (++cin == p.cps) {
          cin = 0;
          if (++sg < nseg) t = p.seg_slot[seg0 + sg] * p.tiles_per_slot + mt;
        }
      }
      for (int c = max(0, issued - NST); c < issued; ++c) mbar_drain(&full[c % NST], (c / NST) & 1);
    } else if (warp == 1 && lane == 0 && leader) {
      // ---------------- MMA issuer (leader): 256 x 128 x 16 per instruction over both CTAs
      uint32_t empty_c[2][NST], accfull_c[2][2], done_c[2];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
#pragma unroll
        for (int i = 0; i < NST; ++i) empty_c[r][i] = cluster_addr(&empty[i], r);
        accfull_c[r][0] = cluster_addr(&accfull[0], r);
        accfull_c[r][1] = cluster_addr(&accfull[1], r);
        done_c[r] = cluster_addr(done, r);
      }
      int per = 0, cin = 0, st = 0, sph = 0;
      for (int c = 0; c < nchunk && !*abort_flag; ++c) {
        const int ab = per & 1;
        const bool first = cin == 0;
        const bool last = cin == p.cps - 1;
        if (first && per >= 2 && !mbar_wait_cluster(&accempty[ab], ((per >> 1) - 1) & 1, abort_flag)) break;
        if (!mbar_wait(&full[st], sph, abort_flag)) break;               // this CTA's stage
        if (!mbar_wait_cluster(&fwd[st], sph, abort_flag)) break;        // the follower's stage
        tc_fence_after();
        const uint32_t a_hi = smem_u32(sA + st * 2 * SLICE_A), a_lo = a_hi + SLICE_A;
        const uint32_t b_hi = smem_u32(sS + st * 2 * SLICE_SH), b_lo = b_hi + SLICE_SH;
        const uint32_t d = tmem + static_cast<uint32_t>(ab * NC);
#pragma unroll
        for (int kk = 0; kk < KC / 16; ++kk) {
          const uint32_t ko = kk * 32;
          const uint32_t acc0 = (first && kk == 0) ? 0u : 1u;
          umma_f16_pair(d, sw128_desc(a_hi + ko), sw128_desc(b_hi + ko), acc0);
          umma_f16_pair(d, sw128_desc(a_hi + ko), sw128_desc(b_lo + ko), 1u);
          umma_f16_pair(d, sw128_desc(a_lo + ko), sw128_desc(b_hi + ko), 1u);
        }
        umma_commit_pair(empty_c[0][st]);
        umma_commit_pair(empty_c[1][st]);
        if (last) {
          umma_commit_pair(accfull_c[0][ab]);
          umma_commit_pair(accfull_c[1][ab]);
        }
        if (++st == NST) { st = 0; sph ^= 1; }
        if (++cin == p.cps) { cin = 0; ++per; }
      }
      umma_commit_pair(done_c[0]);
      umma_commit_pair(done_c[1]);
      mbar_drain_cluster(done, 0);
    } else if (warp == 1 && lane == 0) {
      // ---------------- forwarder (follower): each landed stage -> the leader's full barrier
      int st = 0, sph = 0;
      for (int c = 0; c < nchunk; ++c) {
        if (!mbar_wait(&full[st], sph, abort_flag)) break;
        mbar_arrive_cluster(cluster_addr(&fwd[st], 0));
        if (++st == NST) { st = 0; sph ^= 1; }
      }
      mbar_drain_cluster(done, 0);       // the leader's MMAs read this CTA's stages and write its TMEM
    } else if (warp >= CONV_W0) {
      // ---------------- drain (warps 2..17 of both CTAs): this CTA's 128 TMEM lanes, 32 columns a warp
      const int d = warp - CONV_W0;
      const int quad = warp & 3;
      constexpr int ncolw = NC / 4;
      const int c_lo = (d >> 2) * ncolw;
      const uint32_t lane_base = static_cast<uint32_t>(quad * 32) << 16;
      const uint32_t accempty_c0 = cluster_addr(&accempty[0], 0), accempty_c1 = cluster_addr(&accempty[1], 0);
      bool ok = true;
      double* wsm = reinterpret_cast<double*>(sW + d * 64 * sizeof(double));
      for (int per = 0; per < nseg; ++per) {
        const int ab = per & 1;
        {
          const ZSeg zs = p.segs[seg0 + per];
          __syncwarp();
          for (int j = lane; j < ncolw; j += 32) {
            const int col = p.tile_cols[nt * NC + c_lo + j];
            wsm[j] = (col >= 0) ? zs.scale[static_cast<long long>(col) * zs.scale_cs] : 0.0;
          }
          __syncwarp();
        }
        if (!mbar_wait_warp_cluster(&accfull[ab], (per >> 1) & 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        uint32_t f32a[16], f32b[16], f64w[32];
        tmem_ld16(tmem + lane_base + static_cast<uint32_t>(ab * NC + c_lo), f32a);
        tmem_ld16(tmem + lane_base + static_cast<uint32_t>(ab * NC + c_lo + 16), f32b);
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const uint32_t fcol = FP64_COL + static_cast<uint32_t>(2 * c_lo + 32 * half);
          if (per > 0) tmem_ld32w(tmem + lane_base + fcol, f64w);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            double a0 = (per > 0) ? __hiloint2double(static_cast<int>(f64w[2 * i + 1]), static_cast<int>(f64w[2 * i])) : 0.0;
            const double v = static_cast<double>(__uint_as_float(half ? f32b[i] : f32a[i]));
            a0 = fma(v, wsm[half * 16 + i], a0);
            f64w[2 * i] = static_cast<uint32_t>(__double2loint(a0));
            f64w[2 * i + 1] = static_cast<uint32_t>(__double2hiint(a0));
          }
          tmem_st32(tmem + lane_base + fcol, f64w);
        }
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(ab ? accempty_c1 : accempty_c0);
      }
      if (ok && !*abort_flag) {
        tc_fence_after();
        const int row = quad * 32 + lane;
        const int m = mt * BMC + (row & 63);
        const bool im_part = row >= 64;
        const double inv = 1.0 / (p.scales[0] * p.scales[1]);
        uint32_t f64[32];
#pragma unroll 1
        for (int cb = 0; cb < ncolw / 16; ++cb) {
          const int cbase = c_lo + cb * 16;
          tmem_ld32w(tmem + lane_base + FP64_COL + static_cast<uint32_t>(2 * cbase), f64);
          tmem_wait_ld();
          if (m >= p.M) continue;
#pragma unroll 4
          for (int i = 0; i < 16; ++i) {
            const double v = __hiloint2double(static_cast<int>(f64[2 * i + 1]), static_cast<int>(f64[2 * i])) * inv;
            const long long col = p.tile_cols[nt * NC + cbase + i];
            if (col < 0) continue;
            atomicAdd(reinterpret_cast<double*>(p.C + m + col * p.ldc) + (im_part ? 1 : 0), v);
          }
        }
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  cluster_sync_all();                    // no TMEM, shared-memory or barrier traffic of the pair is left
  if (*abort_flag && tid == 0) atomicExch(p.err, 2);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// Sigma_c on CTA pairs (clusters of two): grid.x = 2 * ceil(row tiles / 2) * column tiles
int launch_sigc_pair(const CUtensorMap& ma, const CUtensorMap& ms, const Params& p, dim3 grid, cudaStream_t s,
                     const char* tag) {
  static uint64_t attr = 0;                       // one bit per device
  int rc = smem_limit_once(reinterpret_cast<const void*>(split_pair_kernel), PairCfg::SMEM_BYTES, attr);
  if (rc) return rc;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(NTHREADS, 1, 1);
  cfg.dynamicSmemBytes = PairCfg::SMEM_BYTES;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const int pi = prof_begin(tag, s);
  QSGW_CUDA(cudaLaunchKernelEx(&cfg, split_pair_kernel, ma, ms, p));
  prof_end(pi, s);
  count_launch();
  QSGW_LAUNCH_CHECK("split_pair_kernel");
  return QSGW_OK;
}

static DevBuf g_scr;                      // FP64 sums of the 256-column kernel

int launch_sigc_wide(const CUtensorMap& ma, const CUtensorMap& ms, Params p, dim3 grid, cudaStream_t s,
                     const char* tag) {
  static uint64_t attr = 0;                       // one bit per device
  int rc = smem_limit_once(reinterpret_cast<const void*>(sigc_wide_kernel), WideCfg::SMEM_BYTES, attr);
  if (rc) return rc;
  rc = g_scr.ensure(static_cast<size_t>(grid.x) * NW * BM2 * sizeof(double));
  if (rc) return rc;
  p.scratch = g_scr.as<double>();
  const int pi = prof_begin(tag, s);
  sigc_wide_kernel<<<grid, NTHREADS, WideCfg::SMEM_BYTES, s>>>(ma, ms, p);
  prof_end(pi, s);
  count_launch();
  QSGW_LAUNCH_CHECK("sigc_wide_kernel");
  return QSGW_OK;
}

}  // namespace tc
}  // namespace qsgw
