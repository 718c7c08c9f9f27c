// Ozaki-scheme complex contractions on the 5th-generation tensor cores: int8
// slices, tcgen05.mma kind::i8 with exact INT32 accumulation in TMEM, operands
// streamed by TMA into 64-byte-swizzled shared memory.
//
// Why int8.  The FP32 accumulation of tcgen05 kind::f16 truncates: the split
// FP16 path carries a bias that grows with the accumulation length (about 4e-8
// per K step, 3.7e-6 relative on a Sigma_c segment of K' = 1216) whatever the
// slice count, and a bias in Sigma_c moves every QP energy the same way.
// Integer products accumulate exactly; the only error left is the rounding of
// the operands to NS slices, which is unbiased.
//
// The scheme.  Every row of A and every column of B gets a power-of-two scale
// mu >= max |x| over its K range; with t = 64 x / mu in [-64, 64]
//     s_1 = rint(t), t_1 = 128 (t - s_1), s_2 = rint(t_1), t_2 = 128 (t_1 - s_2), ...
// every s_i lies in [-64, 64] (one int8) and every step is exact in FP64, so
//     x = mu (s_1 2^-6 + s_2 2^-13 + ... + s_NS 2^-(7 NS - 1)) + r,  |r| <= mu 2^-(7 NS).
// The product keeps the slice pairs (p, q) with p + q <= NS + 1 (the dropped
// ones are below the rounding of the last slice), grouped by level
// L = p + q - 2 into one INT32 TMEM accumulator per level (NS accumulators of
// 128 columns); the drain combines the levels exactly in int64,
//     v = sum_L acc_L 2^(7 (NS - 1 - L)),
// and scales v by mu_row nu_col 2^-(12 + 7 (NS - 1)) in FP64.  A level holds at
// most NS products of |s| <= 64 over K' real K, so |acc| < NS 2^12 K', which
// bounds K' between drains (INT32).  These base-128 digits are the chi0
// kernel's: symmetric, so negation commutes with the slicing (rint is
// symmetric) and the slices of -x are the negated slices of x, which the chi0
// kernel uses to build rows in shared memory.
//
// The Sigma_c kernel (also behind the zmel M -> E product) slices every
// operand in HBM, negated parts included, and so uses base-256 digits over the
// whole int8 range [-128, 127] (slice8): V = rint(x U8 / mu), U8 just under
// 2^(8 NS - 1), mu = max |x| of the row (column) itself rather than a power of
// two above it, eight bits a slice instead of seven, v = sum_L acc_L
// 256^(NS - 1 - L) scaled by mu nu 256^(NS - 1) / U8^2.  Three base-256 slices
// hold 23 bits, four base-128 ones 27: six slice products instead of ten for
// an error within the QP-energy target.  |acc| < NS 2^14 K'.
//
// A complex product C = A B is one real GEMM with M doubled and K interleaved
// (k' = 2k + {re, im}): rows (m, re) of A' = [Re a, -Im a], rows (m, im) =
// [Im a, Re a], B' row n = [Re b, Im b]; lanes 0..63 of an accumulator hold
// Re C, 64..127 Im C.
//
// Kernels (576 threads, one CTA per SM):
//     warp 0        TMA producer
//     warp 1        TMEM owner and MMA issuer (one thread)
//     warps 2..17   drain (chi0: they also build the (m, im) rows of A' from
//                   the (m, re) rows in shared memory, a byte shuffle)
// Every mbarrier wait is bounded; on time-out the CTA records an error, waits
// (bounded) for its own TMA and MMA work, frees TMEM and exits.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>
#include "split_common.cuh"
#include "ozaki_i8.cuh"
#include "autotune.cuh"

namespace qsgw {
namespace oz {

using namespace tc;

constexpr int BM = 128;                  // accumulator rows (64 complex rows x {re, im})
constexpr int BN = kOzTileN;             // accumulator columns (UMMA N)
constexpr int K8 = 64;                   // int8 K per chunk: one 64-byte swizzled row
constexpr int THREADS = 576;
constexpr int NDW = 16;                  // drain warps 2..17
constexpr int NCONV = 12;                // chi0: the drain warps that also convert (warp mod 4 != 1)
constexpr int SLA8 = BM * K8;         // 8 KB: one slice of the A' tile of a stage
constexpr int SLB8 = BN * K8;         // 8 KB: one slice of the B tile of a stage
constexpr int STAGE_BUDGET = 192 * 1024;
constexpr uint32_t TMEM8 = 512;

template <int NS>
struct Cfg {
  static constexpr int STAGE = NS * (SLA8 + SLB8);
  static constexpr int NST = STAGE_BUDGET / STAGE;                // 6, 4, 3 stages for NS = 2, 3, 4
  static constexpr int OFF_A = 0;                                 // [NST][NS] A' slices
  static constexpr int OFF_B = OFF_A + NST * NS * SLA8;        // [NST][NS] B slices
  static constexpr int OFF_W = OFF_B + NST * NS * SLB8;        // drain column factors [16][2][32]
  static constexpr int OFF_BAR = OFF_W + NDW * 64 * 8;
  static constexpr int NBAR = 3 * NST + 3;                        // full, cfull, empty [NST]; accfull, accempty, done
  static constexpr int OFF_MISC = OFF_BAR + NBAR * 8;
  static constexpr int SMEM = OFF_MISC + 64 + 1024;               // + slack for the 1024-byte alignment
  // exact INT32 levels: at most NS products of |s| <= 64 per K element
  static constexpr int MAX_PERIOD = static_cast<int>((1LL << 30) / (NS * 4096LL * K8));
  static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
  static_assert(NS * BN <= static_cast<int>(TMEM8), "one TMEM accumulator per level");
};

// The Sigma_c kernel's shared memory: NBUF chunk buffers (NS A' slices and NS B slices of one
// 64-byte K chunk each), grouped into NST stages of CPS consecutive chunks.  A stage is one
// full/empty barrier pair: the producer fills its CPS chunks under one expected byte count and the
// MMA thread waits for it and releases it once, so the fixed cost of a stage (barrier test or
// wait, commit, TMA bookkeeping) is paid once per CPS chunks.  Two chunks a stage up to 3 slices
// (3 stages of 64 KB at 2, 2 stages of 96 KB at 3), one at 4 slices (3 stages of 64 KB).
template <int NS>
struct SegCfg {
  static constexpr int CPS = NS <= 3 ? 2 : 1;
  static constexpr int CHUNK = NS * (SLA8 + SLB8);
  static constexpr int NBUF = STAGE_BUDGET / CHUNK / CPS * CPS;   // 6, 4, 3 chunk buffers for NS = 2, 3, 4
  static constexpr int NST = NBUF / CPS;                          // 3, 2, 3 stages
  static constexpr int OFF_A = 0;                                 // [NBUF][NS] A' slices
  static constexpr int OFF_B = OFF_A + NBUF * NS * SLA8;          // [NBUF][NS] B slices
  static constexpr int OFF_W = OFF_B + NBUF * NS * SLB8;          // drain column factors [16][2][32]
  static constexpr int OFF_BAR = OFF_W + NDW * 64 * 8;
  static constexpr int NBAR = 2 * NST + 3;                        // full, empty [NST]; accfull, accempty, done
  static constexpr int OFF_MISC = OFF_BAR + NBAR * 8;
  static constexpr int SMEM = OFF_MISC + 64 + 1024;
  static_assert(NST >= 2, "a ring of at least two stages");
  static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
  static_assert(NBUF * NS * SLA8 >= 8 * 32 * 32 * 8, "the paired tail's cross-half sums fit in the A' buffers");
};

// kind::i8, A = B = signed 8-bit, D = S32, both K-major, M = 128, N = BN
constexpr uint32_t IDESC_I8 = (2u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(BN >> 3) << 17) |
                              (static_cast<uint32_t>(BM >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(IDESC_I8), "r"(accumulate));
}
// The MMA above preceded by a non-blocking test (mbarrier.test_wait, acquire) of phase `parity` of
// the barrier at shared address `bar`, whose answer (1 = complete) is read only after the MMA has
// been issued.  The issuing thread blocks in every MMA issue until the tensor core takes it, so a
// wait between two K chunks leaves the tensor core idle; the test's latency is spent inside the
// MMA issue instead.
__device__ __forceinline__ uint32_t umma_i8_then_test(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate,
                                                      uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p, q;\n"
      " mbarrier.test_wait.parity.shared::cta.b64 q, [%5], %6;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%1], %2, %3, %7, p;\n"
      " selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(ok)
      : "r"(tmem_d), "l"(da), "l"(db), "r"(accumulate), "r"(bar), "r"(parity), "r"(IDESC_I8)
      : "memory");
  return ok;
}
// The same MMA with the A operand kept in the tensor core's collector buffer: FILL loads it and
// keeps it, USE reads the kept copy (same A descriptor), LAST reads it and releases the buffer.
enum { A_FILL = 0, A_USE = 1, A_LAST = 2 };
template <int MODE>
__device__ __forceinline__ void umma_i8_ca(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  if (MODE == A_FILL)
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8.collector::a::fill [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(IDESC_I8), "r"(accumulate));
  else if (MODE == A_USE)
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8.collector::a::use [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(IDESC_I8), "r"(accumulate));
  else
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8.collector::a::lastuse [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(IDESC_I8), "r"(accumulate));
}

// The slice products of one K step: for each A slice pa (one shared-memory read through the
// collector buffer), the B slices qb with pa + qb < NS into the accumulator of level pa + qb.
// The first product into each level (pa == 0) starts it when `start` is set.  With test_bar != 0
// the last product (pa = NS - 1, no collector) also tests phase test_parity of that barrier
// (umma_i8_then_test); the answer is returned (0 otherwise).
template <int NS>
__device__ __forceinline__ uint32_t slice_products(uint32_t tmem, uint64_t da0, uint64_t db0, uint32_t a_step,
                                                   uint32_t b_step, bool start, uint32_t test_bar = 0,
                                                   uint32_t test_parity = 0) {
  uint32_t ready = 0;
#pragma unroll
  for (int pa = 0; pa < NS; ++pa) {
    const uint64_t da = da0 + pa * a_step;
#pragma unroll
    for (int qb = 0; qb < NS - pa; ++qb) {
      const uint64_t db = db0 + qb * b_step;
      const uint32_t d = tmem + static_cast<uint32_t>((pa + qb) * kOzTileN);
      const uint32_t acc = (start && pa == 0) ? 0u : 1u;
      if (NS - pa == 1) {
        if (test_bar) ready = umma_i8_then_test(d, da, db, acc, test_bar, test_parity);
        else umma_i8(d, da, db, acc);
      }
      else if (qb == 0) umma_i8_ca<A_FILL>(d, da, db, acc);
      else if (qb == NS - pa - 1) umma_i8_ca<A_LAST>(d, da, db, acc);
      else umma_i8_ca<A_USE>(d, da, db, acc);
    }
  }
  return ready;
}

// 32 lanes x 4 consecutive 32-bit TMEM columns
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}

__device__ __forceinline__ unsigned char* align1024(unsigned char* p) {
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// the smallest power of two >= m (1 for m = 0 or not finite)
__host__ __device__ __forceinline__ double pow2_at_least(double m) {
  if (!(m > 0.0) || !isfinite(m)) return 1.0;
  int e = 0;
  frexp(m, &e);                          // m = f 2^e, f in [0.5, 1)
  return ldexp(1.0, e);
}

// 2^(6 + 7 (NS - 1)): x / mu in [-1, 1] times this is the integer of NS base-128 digits
template <int NS>
__host__ __device__ constexpr double slice_unit() { return static_cast<double>(1LL << (6 + 7 * (NS - 1))); }

// NS slices of x / mu, given scale = slice_unit<NS>() / mu (a power of two, so x * scale is exact):
// V = rint(x * scale) (|V| <= 64 * 128^(NS-1) <= 2^27, an int32) written in base 128 from the
// bottom with digits d = sign(V) r, r = |V| mod 128 taken in [-63, 64]; the top digit holds the
// rest.  Every digit lies in [-64, 64] (one int8), negation commutes with the slicing, and the
// digits rebuild x to mu 2^-(7 NS).  One FP64 multiply and round, then 32-bit integer work:
// the rule above is q = v / 128 rounded to nearest with ties toward zero, d = v - 128 q, i.e.
// q = (v + 63 + [v < 0]) >> 7 (arithmetic shift), four operations a digit (these kernels are
// bound by the integer pipe, not by HBM).
template <int NS>
__device__ __forceinline__ void slice(double x, double scale, int (&s)[NS]) {
  static_assert(6 + 7 * (NS - 1) <= 30, "V must fit an int32");
  int v = __double2int_rn(x * scale);
#pragma unroll
  for (int i = NS - 1; i >= 1; --i) {
    const int q = (v + 63 - (v >> 31)) >> 7;
    s[i] = v - (q << 7);
    v = q;
  }
  s[0] = v;
}
// The Sigma_c kernel's digits: base 256, every int8 value.  U8 = 127 256^(NS-1) - 128 (256^(NS-1) - 1)
// / 255, so that x / mu in [-1, 1] times U8 is an integer V with |V| <= U8 whose NS digits, taken
// from the bottom in [-128, 127], leave a top digit in [-128, 127] too (the lower digits sum to at
// most 128 (256^(NS-1) - 1) / 255 in magnitude).  One bit more per slice than the base-128 digits;
// negation does not commute with this slicing, so the kernels that need -x slice it on their own.
template <int NS>
__host__ __device__ constexpr double slice_unit8() {
  return static_cast<double>(127LL * (1LL << (8 * (NS - 1))) - 128LL * (((1LL << (8 * (NS - 1))) - 1) / 255));
}
// NS base-256 slices of x given scale = slice_unit8<NS>() / mu, mu = max |x| of the row or column
// (x * scale rounded once; |x| <= mu keeps |V| <= U8 < 2^31 - 128 after the rounding, as U8 is an
// integer): V = rint(x * scale), digits d = v - 256 q, q = floor((v + 128) / 256) (arithmetic
// shift), three integer operations a digit
template <int NS>
__device__ __forceinline__ void slice8(double x, double scale, int (&s)[NS]) {
  int v = __double2int_rn(x * scale);
#pragma unroll
  for (int i = NS - 1; i >= 1; --i) {
    const int q = (v + 128) >> 8;
    s[i] = v - (q << 8);
    v = q;
  }
  s[0] = v;
}
// the low bytes of a, b, c, d (two's complement int8) as one word, a lowest
__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  const uint32_t ab = __byte_perm(static_cast<uint32_t>(a), static_cast<uint32_t>(b), 0x0040);
  const uint32_t cd = __byte_perm(static_cast<uint32_t>(c), static_cast<uint32_t>(d), 0x0040);
  return __byte_perm(ab, cd, 0x5410);
}
// (re, im) byte pairs -> (-im, re): the (m, im) row of A' from its (m, re) row
__device__ __forceinline__ uint32_t rotate_pairs(uint32_t w) {
  const uint32_t sw = __byte_perm(w, 0, 0x2301);           // [im0, re0, im1, re1]
  return (__vneg4(sw) & 0x00FF00FFu) | (sw & 0xFF00FF00u);
}

// the extent of the chi0 weights of sign `sign` in bin b (0: the pass has nothing to do there)
__device__ __forceinline__ double w_extent(const double* wr, int b, double sign) {
  return sign < 0.0 ? wr[2 * b] : wr[2 * b + 1];
}

// =====================================================================================
// Sigma_c: out(:, col) = sum over the segments of the column's group of W_slot^H (w_seg(col) z_col)
struct SegParams {
  int M;                      // complex rows (ngb)
  int ntm;                    // 64-row tiles
  int cps;                    // chunks per segment
  int nslot, T;               // A' tile coordinate (q nslot + slot) T + mt
  int nrows;                  // B rows per slice (tile-ordered columns)
  const int* tile_group;
  const int* tile_cols;
  const int* group_seg_off;
  const int* group_nseg;
  const int* seg_slot;
  const ZSeg* segs;
  const double* mu_a;         // [slot][T * 64] row scales
  const double* nu_b;         // [nrows] column scales
  double post;                // 256^(NS - 1) / U8^2 (slice_unit8)
  double2* const* tile_out;   // [tile] output of the tile's task: column col at tile_out[t] + col ldc
  long long ldc;
  int tail;                   // 1: M mod 64 <= 32 and the last row tile holds segment pairs (mapT)
  int* err;
};

// Paired tail.  When the last 64-row tile has at most 32 valid rows, its CTAs run the segments two at
// a time: complex rows 0..31 of the A' tile are the tail rows of segment 2i, rows 32..63 those of
// segment 2i + 1 (each half read from the half-height tail slices through mapT), so those CTAs do
// half the MMAs; the drain weights each half with its own segment and adds the halves at the end.
template <int NS, bool PAIRED>
__global__ void __launch_bounds__(THREADS, 1)
    oz_seg_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                  const __grid_constant__ CUtensorMap mapT, const SegParams p) {
  using L = SegCfg<NS>;
  constexpr int NST = L::NST, CPS = L::CPS;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* sm = align1024(smem_raw);
  unsigned char* sA = sm + L::OFF_A;
  unsigned char* sB = sm + L::OFF_B;
  double* sW = reinterpret_cast<double*>(sm + L::OFF_W);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::OFF_BAR);
  uint64_t* full = bar;                  // [NST] TMA -> MMA
  uint64_t* empty = bar + NST;           // [NST] MMA -> TMA
  uint64_t* accfull = bar + 2 * NST;     // MMA -> drain
  uint64_t* accempty = accfull + 1;      // drain -> MMA
  uint64_t* done = accempty + 1;         // every MMA of the CTA retired
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::OFF_MISC);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::OFF_MISC + 8);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // the row tiles of a column tile adjacent; the paired launch covers the last row tile only
  const int mt = PAIRED ? p.T - 1 : blockIdx.x % p.ntm, nt = PAIRED ? blockIdx.x : blockIdx.x / p.ntm;
  const int group = p.tile_group[nt];
  const int nseg = p.group_nseg[group];
  const int seg0 = p.group_seg_off[group];
  constexpr bool paired = PAIRED;
  const int nstep = paired ? (nseg + 1) / 2 : nseg;   // accumulation periods: segments or segment pairs
  const int nchunk = nstep * p.cps;

  if (tid == 0) {
    for (int i = 0; i < NST; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); }
    mbar_init(accfull, 1);
    mbar_init(accempty, NDW);
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM8));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (nchunk > 0) {
    if (warp == 0 && lane == 0) {
      // ---------------- TMA producer: NS slices of the segment's A' tile and of the B tile
      constexpr uint32_t bytes = NS * (SLA8 + SLB8);
      int issued = 0, sg = 0, cin = 0, st = 0, ph = 0, sub = 0;   // issued: stages begun
      // this step's slot (paired: the slots of segments 2 sg and 2 sg + 1, the second repeated when absent)
      auto step_slots = [&](int g, int& s0, int& s1) {
        if (!paired) { s0 = s1 = p.seg_slot[seg0 + g]; return; }
        s0 = p.seg_slot[seg0 + 2 * g];
        s1 = 2 * g + 1 < nseg ? p.seg_slot[seg0 + 2 * g + 1] : s0;
      };
      int slot = 0, slot1 = 0;
      step_slots(0, slot, slot1);
      for (int c = 0; c < nchunk; ++c) {
        if (sub == 0) {                               // a new stage: its CPS chunks (fewer at the end)
          if (issued >= NST && !mbar_wait(&empty[st], ph ^ 1, abort_flag)) break;
          ++issued;
          mbar_expect_tx(&full[st], bytes * static_cast<uint32_t>(min(CPS, nchunk - c)));
        }
        const int buf = st * CPS + sub;
        const int x = cin * K8;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          unsigned char* dA = sA + (buf * NS + q) * SLA8;
          if constexpr (PAIRED) {                     // rows 0-31 / 32-63 re, 64-95 / 96-127 im
            tma_load_4d(dA, &mapT, &full[st], x, 0, 0, q * p.nslot + slot);
            tma_load_4d(dA + SLA8 / 4, &mapT, &full[st], x, 0, 0, q * p.nslot + slot1);
            tma_load_4d(dA + SLA8 / 2, &mapT, &full[st], x, 0, 1, q * p.nslot + slot);
            tma_load_4d(dA + 3 * SLA8 / 4, &mapT, &full[st], x, 0, 1, q * p.nslot + slot1);
          } else {
            tma_load_4d(dA, &mapA, &full[st], x, 0, 0, (q * p.nslot + slot) * p.T + mt);
          }
          tma_load_3d(sB + (buf * NS + q) * SLB8, &mapB, &full[st], x, nt * BN, q);
        }
        if (++cin == p.cps) {
          cin = 0;
          if (++sg < nstep) step_slots(sg, slot, slot1);
        }
        if (++sub == CPS) {
          sub = 0;
          if (++st == NST) { st = 0; ph ^= 1; }
        }
      }
      for (int g = max(0, issued - NST); g < issued; ++g) mbar_drain(&full[g % NST], (g / NST) & 1);
    } else if (warp == 1 && lane == 0) {
      // ---------------- MMA issuer: NS level accumulators, one accumulation period per segment
      const uint64_t dA0 = sw64_desc(smem_u32(sA)), dB0 = sw64_desc(smem_u32(sB));
      int seg = 0, cin = 0, st = 0, ph = 0, sub = 0;
      uint32_t ready = 0;                            // the next stage was seen full by the last test
      for (int c = 0; c < nchunk && !*abort_flag; ++c) {
        const bool first = cin == 0, last = cin == p.cps - 1;
        const bool stage_end = sub == CPS - 1 || c + 1 == nchunk;
        if (first && seg >= 1 && !mbar_wait(accempty, (seg - 1) & 1, abort_flag)) break;
        if (sub == 0 && !ready && !mbar_wait(&full[st], ph, abort_flag)) break;
        tc_fence_after();
        // the next stage is tested during the last MMA of this stage's last chunk
        const uint32_t nbar = stage_end && c + 1 < nchunk ? smem_u32(&full[st + 1 == NST ? 0 : st + 1]) : 0u;
        const uint32_t npar = st + 1 == NST ? (ph ^ 1) : ph;
        const int buf = st * CPS + sub;
#pragma unroll
        for (int kk = 0; kk < K8 / 32; ++kk) {        // 32 int8 = 32 B along K = 2 descriptor units
          const uint32_t r = slice_products<NS>(tmem, dA0 + static_cast<uint32_t>((buf * NS * SLA8) >> 4) + 2 * kk,
                                                dB0 + static_cast<uint32_t>((buf * NS * SLB8) >> 4) + 2 * kk,
                                                SLA8 >> 4, SLB8 >> 4, first && kk == 0,
                                                kk == K8 / 32 - 1 ? nbar : 0u, npar);
          if (kk == K8 / 32 - 1) ready = nbar ? r : 0u;
        }
        if (last) umma_commit(accfull);
        if (stage_end) {
          umma_commit(&empty[st]);
          sub = 0;
          if (++st == NST) { st = 0; ph ^= 1; }
        } else {
          ++sub;
        }
        if (++cin == p.cps) { cin = 0; ++seg; }
      }
      umma_commit(done);
      mbar_drain(done, 0);
    } else if (warp >= 2) {
      // ---------------- drain: TMEM lanes 32 (warp mod 4) .. +31, 32 columns a warp, FP64 sums in registers
      const int dw = warp - 2;
      const int quad = warp & 3;
      const int c_lo = (dw >> 2) * 32;
      const int row = quad * 32 + lane;                 // accumulator row: 0..63 re, 64..127 im
      const int mloc = row & 63;
      // paired tail: rows 32..63 (and 96..127) belong to the second segment of each pair
      const int hb = paired ? (mloc >> 5) : 0;
      const int mrow = paired ? (mloc & 31) : mloc;     // the row within the tile's output rows
      const uint32_t lane_base = static_cast<uint32_t>(quad * 32) << 16;
      double* wsm = sW + dw * 64;                       // [2][32]: the pair's two weight sets
      double acc[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] = 0.0;
      const int rtile = nt * BN + c_lo;
      auto drain = [&]() -> bool {
        for (int seg = 0; seg < nstep; ++seg) {
          // this period's segment(s): one, or a pair (the second absent past the end: weight 0)
          const int sa = PAIRED ? seg0 + 2 * seg : seg0 + seg;
          int slot;
          __syncwarp();                                 // the previous period's reads of wsm are done
          {
            const int col = p.tile_cols[rtile + lane];
            const ZSeg z0 = p.segs[sa];
            wsm[lane] = (col >= 0) ? z0.scale[static_cast<long long>(col) * z0.scale_cs] * p.nu_b[rtile + lane] : 0.0;
            if constexpr (PAIRED) {
              const bool has1 = 2 * seg + 1 < nseg;
              double v1 = 0.0;
              if (has1 && col >= 0) {
                const ZSeg z1 = p.segs[sa + 1];
                v1 = z1.scale[static_cast<long long>(col) * z1.scale_cs] * p.nu_b[rtile + lane];
              }
              wsm[32 + lane] = v1;
              slot = p.seg_slot[hb && has1 ? sa + 1 : sa];
            } else {
              slot = p.seg_slot[sa];
            }
          }
          const double rf = p.mu_a[static_cast<long long>(slot) * p.T * 64 + mt * 64 + mrow] * p.post;
          const double* wuse = PAIRED ? wsm + 32 * hb : wsm;
          __syncwarp();
          if (!mbar_wait_warp(accfull, seg & 1, abort_flag)) return false;
          tc_fence_after();
#pragma unroll
          for (int blk = 0; blk < 8; ++blk) {           // 4 columns at a time (96 registers per thread)
            uint32_t v[NS][4];
#pragma unroll
            for (int lv = 0; lv < NS; ++lv)
              tmem_ld4(tmem + lane_base + static_cast<uint32_t>(lv * BN + c_lo + blk * 4), v[lv]);
            tmem_wait_ld();
            if (blk == 7) {                             // every TMEM read of this segment is done
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(accempty);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              long long comb = static_cast<int>(v[0][j]);
#pragma unroll
              for (int lv = 1; lv < NS; ++lv) comb = comb * 256 + static_cast<int>(v[lv][j]);
              acc[blk * 4 + j] = fma(static_cast<double>(comb) * rf, wuse[blk * 4 + j], acc[blk * 4 + j]);
            }
          }
        }
        return true;
      };
      const bool ok = drain();
      if constexpr (PAIRED) {
        // add the second segments' sums (rows 32..63, 96..127) to the first ones': through the A'
        // stage buffers, free once the last period's MMAs are done (its accfull was seen above)
        double* xb = reinterpret_cast<double*>(sA) + (((dw >> 2) * 2 + (quad >> 1)) * 32) * 32;
        if (hb) {
#pragma unroll
          for (int j = 0; j < 32; ++j) xb[j * 32 + lane] = acc[j];
        }
        asm volatile("bar.sync 1, %0;" ::"r"(NDW * 32) : "memory");
        if (!hb) {
#pragma unroll
          for (int j = 0; j < 32; ++j) acc[j] += xb[j * 32 + lane];
        }
      }
      if (ok && !*abort_flag && !hb) {
        const int m = mt * 64 + mrow;
        const int part = row >= 64 ? 1 : 0;
        double2* const C = p.tile_out[nt];
        if (m < p.M) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = p.tile_cols[rtile + j];
            if (col >= 0) reinterpret_cast<double*>(C + m + static_cast<long long>(col) * p.ldc)[part] = acc[j];
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM8));
  }
}

// =====================================================================================
// chi0: C(:, :, slab_b) += sign sum_{e in bin b} conj(y_e(0:M)) y_e(row_b0 : row_b0 + N)^T,
// y_e = sqrt(sign w_e) z_col(e) sliced in HBM as Y8[slice][row][K'] (the (m, re) rows of A' and
// the rows of B are both rows of Y8; the (m, im) rows are rotated from them in shared memory)
struct HerkParams {
  int M, N;                   // output rows / columns
  int ntm;                    // 64-row tiles
  int herm;
  int row_b0;
  int Rows;                   // rows of Y8 per slice
  const long long* bin_k0;    // first K chunk of bin b in Y8
  const int* bin_nch;         // K chunks of bin b
  const int* bin_slab;
  const double* wrange;       // [bin][2]: largest -w and largest w (0 when none)
  const double* mu;           // [bin][Rows] row scales of y
  double sign;                // -1 or +1: the weight class of this pass
  double post;
  double2* C;
  long long ldc, c_bs;
  int* err;
};

template <int NS>
__global__ void __launch_bounds__(THREADS, 1)
    oz_herk_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                   const HerkParams p) {
  using L = Cfg<NS>;
  constexpr int NST = L::NST;
  constexpr int PER = L::MAX_PERIOD;
  constexpr int HALF = SLA8 / 2;      // the (m, re) half of an A' slice: 64 rows x 64 B
  const int mt = blockIdx.x % p.ntm, nt = blockIdx.x / p.ntm;
  const int bin = blockIdx.y;
  if (p.herm && mt * 64 + 63 < nt * BN) return;              // strictly upper tile: mirrored
  if (!(w_extent(p.wrange, bin, p.sign) > 0.0)) return;       // no weight of this sign in the bin
  const int nch = p.bin_nch[bin];
  const int per_split = (nch + gridDim.z - 1) / gridDim.z;
  const int cbeg = blockIdx.z * per_split;
  const int nchunk = min(nch, cbeg + per_split) - cbeg;
  if (nchunk <= 0) return;
  const int kc0 = static_cast<int>(p.bin_k0[bin] + cbeg);    // first chunk of this CTA in Y8

  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* sm = align1024(smem_raw);
  unsigned char* sA = sm + L::OFF_A;
  unsigned char* sB = sm + L::OFF_B;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::OFF_BAR);
  uint64_t* full = bar;                  // [NST] TMA -> converters
  uint64_t* cfull = bar + NST;           // [NST] converters -> MMA
  uint64_t* empty = bar + 2 * NST;       // [NST] MMA -> TMA
  uint64_t* accfull = bar + 3 * NST;
  uint64_t* accempty = accfull + 1;
  uint64_t* done = accempty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::OFF_MISC);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::OFF_MISC + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nper = (nchunk + PER - 1) / PER;

  if (tid == 0) {
    for (int i = 0; i < NST; ++i) { mbar_init(&full[i], 1); mbar_init(&cfull[i], NCONV); mbar_init(&empty[i], 1); }
    mbar_init(accfull, 1);
    mbar_init(accempty, NDW);
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM8));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer: the (m, re) half of the A' tile and the B tile, NS slices each
    constexpr uint32_t bytes = NS * (HALF + SLB8);
    int issued = 0, st = 0, ph = 0;
    for (int c = 0; c < nchunk; ++c) {
      if (c >= NST && !mbar_wait(&empty[st], ph ^ 1, abort_flag)) break;
      issued = c + 1;
      mbar_expect_tx(&full[st], bytes);
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        tma_load_4d(sA + (st * NS + q) * SLA8, &mapA, &full[st], 0, mt * 64, q, kc0 + c);
        tma_load_4d(sB + (st * NS + q) * SLB8, &mapB, &full[st], 0, p.row_b0 + nt * BN, q, kc0 + c);
      }
      if (++st == NST) { st = 0; ph ^= 1; }
    }
    for (int c = max(0, issued - NST); c < issued; ++c) mbar_drain(&full[c % NST], (c / NST) & 1);
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer: periods of at most PER chunks (exact INT32 levels)
    const uint64_t dA0 = sw64_desc(smem_u32(sA)), dB0 = sw64_desc(smem_u32(sB));
    int st = 0, ph = 0, cin = 0, per = 0;
    uint32_t ready = 0;                              // the chunk's stage was seen converted by the last test
    for (int c = 0; c < nchunk && !*abort_flag; ++c) {
      const bool first = cin == 0;
      const bool last = cin == PER - 1 || c == nchunk - 1;
      if (first && per >= 1 && !mbar_wait(accempty, (per - 1) & 1, abort_flag)) break;
      if (!ready && !mbar_wait(&cfull[st], ph, abort_flag)) break;
      tc_fence_after();
      const uint32_t nbar = c + 1 < nchunk ? smem_u32(&cfull[st + 1 == NST ? 0 : st + 1]) : 0u;
      const uint32_t npar = st + 1 == NST ? (ph ^ 1) : ph;
#pragma unroll
      for (int kk = 0; kk < K8 / 32; ++kk)
        ready = slice_products<NS>(tmem, dA0 + static_cast<uint32_t>((st * NS * SLA8) >> 4) + 2 * kk,
                                   dB0 + static_cast<uint32_t>((st * NS * SLB8) >> 4) + 2 * kk, SLA8 >> 4,
                                   SLB8 >> 4, first && kk == 0, kk == K8 / 32 - 1 ? nbar : 0u, npar);
      umma_commit(&empty[st]);
      if (last) umma_commit(accfull);
      if (++st == NST) { st = 0; ph ^= 1; }
      if (last) { cin = 0; ++per; } else { ++cin; }
    }
    umma_commit(done);
    mbar_drain(done, 0);
  } else if (warp >= 2) {
    // ---------------- converters + drain (warps 2..17)
    // The converters are the 12 warps off the MMA warp's sub-partition (warp mod 4 != 1): the
    // MMA thread blocks in every MMA issue, so issue slots taken from it idle the tensor core.
    // The other four (they own TMEM lanes 32..63) only drain.
    const int dw = warp - 2;
    const bool conv = (warp & 3) != 1;
    const int ct = (dw - (dw + 1) / 4) * 32 + lane;      // 0..383 over the converter warps
    const int quad = warp & 3;
    const int c_lo = (dw >> 2) * 32;
    const int row = quad * 32 + lane;
    const uint32_t lane_base = static_cast<uint32_t>(quad * 32) << 16;
    long long acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0;
    bool ok = true;
    int st = 0, ph = 0, cin = 0, per = 0;
    for (int c = 0; c < nchunk; ++c) {
      if (conv) {
        if (!mbar_wait_warp(&full[st], ph, abort_flag)) { ok = false; break; }
        // the (m, im) rows [-Im y, Re y] from the (m, re) rows [Re y, Im y]: same swizzled offsets
        // (rows r and r + 64 share their 64-byte swizzle pattern)
        for (int i = ct; i < NS * (HALF / 16); i += NCONV * 32) {
          const int q = i / (HALF / 16), j = i % (HALF / 16);
          const uint4 v = *reinterpret_cast<const uint4*>(sA + (st * NS + q) * SLA8 + j * 16);
          uint4 o;
          o.x = rotate_pairs(v.x); o.y = rotate_pairs(v.y); o.z = rotate_pairs(v.z); o.w = rotate_pairs(v.w);
          *reinterpret_cast<uint4*>(sA + (st * NS + q) * SLA8 + HALF + j * 16) = o;
        }
        fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&cfull[st]);
      }
      if (++st == NST) { st = 0; ph ^= 1; }
      const bool last = cin == PER - 1 || c == nchunk - 1;
      if (!last) { ++cin; continue; }
      cin = 0;
      // drain the period: exact int64 sums of the combined levels
      if (!mbar_wait_warp(accfull, per & 1, abort_flag)) { ok = false; break; }
      tc_fence_after();
#pragma unroll
      for (int blk = 0; blk < 8; ++blk) {
        uint32_t v[NS][4];
#pragma unroll
        for (int lv = 0; lv < NS; ++lv)
          tmem_ld4(tmem + lane_base + static_cast<uint32_t>(lv * BN + c_lo + blk * 4), v[lv]);
        tmem_wait_ld();
        if (blk == 7) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(accempty);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          long long comb = static_cast<int>(v[0][j]);
#pragma unroll
          for (int lv = 1; lv < NS; ++lv) comb = comb * 128 + static_cast<int>(v[lv][j]);
          acc[blk * 4 + j] += comb;
        }
      }
      ++per;
    }
    if (ok && per == nper && !*abort_flag) {
      const int m = mt * 64 + (row & 63);
      const int part = row >= 64 ? 1 : 0;
      if (m < p.M) {
        const double* mub = p.mu + static_cast<long long>(bin) * p.Rows;
        const double fm = mub[m] * p.post * p.sign;
        double2* Cb = p.C + static_cast<long long>(p.bin_slab[bin]) * p.c_bs;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int n = nt * BN + c_lo + j;
          // the upper part of a Hermitian output comes from the mirror
          if (n < p.N && !(p.herm && m < n)) {
            const double val = static_cast<double>(acc[j]) * fm * mub[p.row_b0 + n];
            atomicAdd(reinterpret_cast<double*>(Cb + m + static_cast<long long>(n) * p.ldc) + part, val);
            if (p.herm && m > n)                          // C(n, m) = conj(C(m, n))
              atomicAdd(reinterpret_cast<double*>(Cb + n + static_cast<long long>(m) * p.ldc) + part,
                        part ? -val : val);
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM8));
  }
}

// =====================================================================================
// operand preparation (HBM-bound)

// out[slot * ncols_out + j] = scale of column c = colmap[j] (or j) of the complex column-major
// matrix src + slot * slot_stride (leading dimension ld): the max over k < K of max(|Re|, |Im|)
// itself (the base-256 slicing divides by it, so no power of two is needed, and the full
// digit range is used); 1 for absent, zero or non-finite columns.  One warp per column.
__global__ void oz_colscale_kernel(const double2* __restrict__ src, long long ld, long long slot_stride, int K,
                                   int ncols_valid, const int* __restrict__ colmap, int ncols_out,
                                   double* __restrict__ out) {
  const int slot = blockIdx.y;
  const int j = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= ncols_out) return;
  const int c = colmap ? colmap[j] : (j < ncols_valid ? j : -1);
  double m = 0.0;
  if (c >= 0) {
    const double2* col = src + static_cast<long long>(slot) * slot_stride + static_cast<long long>(c) * ld;
    for (int k = lane; k < K; k += 32) {
      const double2 v = col[k];
      m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) out[static_cast<long long>(slot) * ncols_out + j] = (m > 0.0 && isfinite(m)) ? m : 1.0;
}

// Sigma_c A' slices from W (K x M per slot): A(m, k) = conj(W_slot[k + m ld]) into
// [q][slot_out0 + slot][t][half][64][Kp] int8; each thread four consecutive k of one row.
// grid (ceil(Kp/2 / 128), nslot * T), block 256: warp w rows w, w + 8, ..
// TAIL: only the first 32 complex rows of the last row tile t = T - 1 (grid y = slot), into the
// half-height tail layout [q][slot_out0 + slot][half][32][Kp] that the paired tail tiles read.
// Tw: row tiles written per slot (T, or T - 1 when the last one is read from the tail slices).
template <int NS, bool TAIL = false>
__global__ void oz_slice_w_kernel(int8_t* __restrict__ out, const double2* __restrict__ w, long long ld,
                                  long long slot_stride, int M, int K, int T, int Tw, int nslot_total, int slot_out0,
                                  int Kp, const double* __restrict__ mu) {
  const int st = blockIdx.y;                           // slot * Tw + t of this launch (TAIL: slot)
  const int t = TAIL ? T - 1 : st % Tw, slot = TAIL ? st : st / Tw;
  const int k0 = (blockIdx.x * 32 + (threadIdx.x & 31)) * 4;
  if (k0 >= Kp / 2) return;
  const int gslot = slot_out0 + slot;
  constexpr int ROWS = TAIL ? 32 : 64;
  for (int mm = threadIdx.x >> 5; mm < ROWS; mm += 8) {
    const int m = t * 64 + mm;
    const double inv = slice_unit8<NS>() / mu[static_cast<long long>(gslot) * T * 64 + m];
    int sr[4][NS], si[4][NS], sn[4][NS];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int k = k0 + i;
      double2 v = make_double2(0.0, 0.0);
      if (m < M && k < K) v = w[static_cast<long long>(slot) * slot_stride + k + static_cast<long long>(m) * ld];
      slice8<NS>(v.x, inv, sr[i]);                     // Re a
      slice8<NS>(-v.y, inv, si[i]);                    // Im a  (a = conj(W))
      slice8<NS>(v.y, inv, sn[i]);                     // -Im a, sliced on its own (base-256 digits)
    }
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const long long r0 = TAIL ? (static_cast<long long>(q) * nslot_total + gslot) * 64 + mm
                                : ((static_cast<long long>(q) * nslot_total + gslot) * T + t) * 128 + mm;
      uint2 h0, h1;                                    // half 0: [Re a, -Im a]; half 1: [Im a, Re a]
      h0.x = pack4(sr[0][q], sn[0][q], sr[1][q], sn[1][q]);
      h0.y = pack4(sr[2][q], sn[2][q], sr[3][q], sn[3][q]);
      h1.x = pack4(si[0][q], sr[0][q], si[1][q], sr[1][q]);
      h1.y = pack4(si[2][q], sr[2][q], si[3][q], sr[3][q]);
      *reinterpret_cast<uint2*>(out + r0 * Kp + 2 * k0) = h0;
      *reinterpret_cast<uint2*>(out + (r0 + ROWS) * Kp + 2 * k0) = h1;
    }
  }
}

// Sigma_c B slices: row r = zmel column cols[r] (-1: zero row), [Re b, Im b] per k, into
// [q][rs][Kp] (slice q of row r at (q rs + r) Kp; rs >= nrows).
// grid (ceil(Kp/2 / 128), ceil(nrows / 8)), block 256: one row per warp
template <int NS>
__global__ void oz_slice_z_kernel(int8_t* __restrict__ out, const double2* __restrict__ z, long long ld, int K,
                                  const int* __restrict__ cols, int nrows, long long rs, int Kp,
                                  const double* __restrict__ nu) {
  const int r = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int k0 = (blockIdx.x * 32 + (threadIdx.x & 31)) * 4;
  if (r >= nrows || k0 >= Kp / 2) return;
  const int c = cols[r];
  const double inv = slice_unit8<NS>() / nu[r];
  int sr[4][NS], si[4][NS];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int k = k0 + i;
    double2 v = make_double2(0.0, 0.0);
    if (c >= 0 && k < K) v = z[k + static_cast<long long>(c) * ld];
    slice8<NS>(v.x, inv, sr[i]);
    slice8<NS>(v.y, inv, si[i]);
  }
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    uint2 h;
    h.x = pack4(sr[0][q], si[0][q], sr[1][q], si[1][q]);
    h.y = pack4(sr[2][q], si[2][q], sr[3][q], si[3][q]);
    *reinterpret_cast<uint2*>(out + (static_cast<long long>(q) * rs + r) * Kp + 2 * k0) = h;
  }
}

// chi0: per-row max over every column of z (rows < Rows), as the bits of a non-negative double
__global__ void oz_rowmax_kernel(const double2* __restrict__ z, long long ldz, int Rows, long long ncols,
                                 unsigned long long* __restrict__ out) {
  for (int m = threadIdx.x; m < Rows; m += blockDim.x) {
    double mx = 0.0;
    for (long long c = blockIdx.x; c < ncols; c += gridDim.x) {
      const double2 v = z[m + c * ldz];
      mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
    }
    atomicMax(out + m, static_cast<unsigned long long>(__double_as_longlong(mx)));
  }
}

// chi0: the weight extents of every bin, wr[2 b] = max(-w, 0) and wr[2 b + 1] = max(w, 0) over its
// entries, as the bits of non-negative doubles (atomicMax; zeroed by the caller).  grid (x, bins).
__global__ void oz_wrange_kernel(const double* __restrict__ ew, const long long* __restrict__ ebeg,
                                 const int* __restrict__ cnt, unsigned long long* __restrict__ wr) {
  const int b = blockIdx.y;
  double neg = 0.0, pos = 0.0;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < cnt[b];
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double w = ew[ebeg[b] + e];
    neg = fmax(neg, -w);
    pos = fmax(pos, w);
  }
  for (int o = 16; o; o >>= 1) {
    neg = fmax(neg, __shfl_xor_sync(0xffffffffu, neg, o));
    pos = fmax(pos, __shfl_xor_sync(0xffffffffu, pos, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (neg > 0.0) atomicMax(wr + 2 * b, static_cast<unsigned long long>(__double_as_longlong(neg)));
    if (pos > 0.0) atomicMax(wr + 2 * b + 1, static_cast<unsigned long long>(__double_as_longlong(pos)));
  }
}

// chi0: mu[b][m] = 2^e >= sqrt(largest sign * w of bin b) * zmax[m], a bound on |y| over the bin's row m
__global__ void oz_mu_kernel(const unsigned long long* __restrict__ zmax, const double* __restrict__ wr, int Rows,
                             int nbins, double sign, double* __restrict__ mu) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= static_cast<long long>(Rows) * nbins) return;
  const int b = static_cast<int>(i / Rows), m = static_cast<int>(i % Rows);
  mu[i] = pow2_at_least(sqrt(w_extent(wr, b, sign)) * __longlong_as_double(static_cast<long long>(zmax[m])));
}

// chi0: Y8[q][m][k0_b + 2 e' + {0,1}] = slices of (Re, Im) of sqrt(max(sign w_e, 0)) z_col(e)(m).
// blockIdx.y = bin; blockIdx.x strides over (entry block of 32, 64-row tile) items of the bin.
// Thread (row mm, group g) slices the 8 consecutive entries 8 g .. 8 g + 7 of its row (loads
// coalesced along m), the 16 bytes per slice go to a shared tile with 80-byte rows (no bank
// conflicts), and 64 rows x 64 bytes per slice leave coalesced along K.
// the NS slices of the 8 entries (f z) of one row as 16 bytes each: (re, im) int8 pairs in entry order
template <int NS>
__device__ __forceinline__ void y_pack(uint4 (&out)[NS], const double (&f)[8], const double2 (&zv)[8],
                                       double scale) {
  uint32_t w[NS][4];
#pragma unroll
  for (int jp = 0; jp < 4; ++jp) {
    int r0[NS], i0[NS], r1[NS], i1[NS];
    // (f z) scale with scale a power of two is z (f scale), rounded the same way
    const double fs0 = f[2 * jp] * scale, fs1 = f[2 * jp + 1] * scale;
    slice<NS>(zv[2 * jp].x, fs0, r0);
    slice<NS>(zv[2 * jp].y, fs0, i0);
    slice<NS>(zv[2 * jp + 1].x, fs1, r1);
    slice<NS>(zv[2 * jp + 1].y, fs1, i1);
#pragma unroll
    for (int q = 0; q < NS; ++q) w[q][jp] = pack4(r0[q], i0[q], r1[q], i1[q]);
  }
#pragma unroll
  for (int q = 0; q < NS; ++q) out[q] = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
}
template <int NS>
__device__ __forceinline__ void y_tile_pack(int8_t (*tile)[64][80], int mm, int g, const double (&f)[8],
                                            const double2 (&zv)[8], double scale) {
  uint4 out[NS];
  y_pack<NS>(out, f, zv, scale);
#pragma unroll
  for (int q = 0; q < NS; ++q) *reinterpret_cast<uint4*>(&tile[q][mm][g * 16]) = out[q];
}

// Y8 is chunk-major: [chunk][slice][row][64 bytes], so one TMA box (64 or 128 rows of one chunk
// and slice) is one contiguous block of HBM
template <int NS>
__device__ __forceinline__ void y_tile_store(int8_t* __restrict__ y8, const int8_t (*tile)[64][80], int Rows, int rt,
                                             long long chunk) {
  const int row = threadIdx.x >> 2, part = threadIdx.x & 3;
  const int mo = rt * 64 + row;
  if (mo < Rows) {
#pragma unroll
    for (int q = 0; q < NS; ++q)
      *reinterpret_cast<uint4*>(y8 + ((chunk * NS + q) * Rows + mo) * 64 + part * 16) =
          *reinterpret_cast<const uint4*>(&tile[q][row][part * 16]);
  }
}

template <int NS>
__global__ void __launch_bounds__(256)
    oz_slice_y_kernel(int8_t* __restrict__ y8, int Rows, const double2* __restrict__ z, long long ldz,
                      const int* __restrict__ ecol, const double* __restrict__ ew, const long long* __restrict__ ebeg,
                      const int* __restrict__ cnt, const long long* __restrict__ bin_k0,
                      const double* __restrict__ wr, const double* __restrict__ mu, double sign) {
  __shared__ __align__(16) int8_t tile[NS][64][80];
  const int b = blockIdx.y;
  if (!(w_extent(wr, b, sign) > 0.0)) return;
  const int n = cnt[b];
  const int neb = (n + 31) / 32;
  const int nrt = (Rows + 63) / 64;
  const long long e0 = ebeg[b];
  const long long kc = bin_k0[b];
  const double* mub = mu + static_cast<long long>(b) * Rows;
  const int mm = threadIdx.x & 63, g = threadIdx.x >> 6;
  for (long long item = blockIdx.x; item < static_cast<long long>(neb) * nrt; item += gridDim.x) {
    const int eb = static_cast<int>(item % neb), rt = static_cast<int>(item / neb);
    const int m = rt * 64 + mm;
    const double scale = (m < Rows) ? slice_unit<NS>() / mub[m] : 0.0;
    double f[8];
    double2 zv[8];
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      const int e = eb * 32 + g * 8 + jj;
      f[jj] = 0.0;
      zv[jj] = make_double2(0.0, 0.0);
      if (e < n && m < Rows) {
        const long long ge = e0 + e;
        const long long col = ecol ? ecol[ge] : e;
        f[jj] = sqrt(fmax(sign * ew[ge], 0.0));
        zv[jj] = z[m + col * ldz];
      }
    }
    y_tile_pack<NS>(tile, mm, g, f, zv, scale);
    __syncthreads();
    y_tile_store<NS>(y8, tile, Rows, rt, kc + eb);
    __syncthreads();
  }
}

// chi0, every bin over the same columns 0..n-1 in order (bin b's weights at ew[b * n + e]): z is read
// once per (32-column block, 64-row tile) item and sliced for every bin with a weight of this sign.
// Thread (row mm = tid / 4, group g = tid % 4) slices the 8 consecutive entries 8 g .. 8 g + 7 of
// its row; their 16 bytes per slice are one piece of the row's 64-byte chunk, so a warp (8 rows x
// 4 groups) stores 512 contiguous bytes per slice straight from registers and loads 4 x 128
// contiguous bytes of z per entry.  The square roots of the weights of up to kDenseBins bins are
// formed once per item in shared memory: two barriers per item and bin group, none per bin.
constexpr int kDenseBins = 32;
template <int NS>
__global__ void __launch_bounds__(256)
    oz_slice_y_dense_kernel(int8_t* __restrict__ y8, int Rows, const double2* __restrict__ z,
                            long long ldz, int n, int nbins, const double* __restrict__ ew,
                            const long long* __restrict__ bin_k0, const double* __restrict__ wr,
                            const double* __restrict__ mu, double sign) {
  __shared__ double sf[kDenseBins][32];
  const int neb = (n + 31) / 32;
  const int nrt = (Rows + 63) / 64;
  const int mm = threadIdx.x >> 2, g = threadIdx.x & 3;
  for (long long item = blockIdx.x; item < static_cast<long long>(neb) * nrt; item += gridDim.x) {
    const int eb = static_cast<int>(item % neb), rt = static_cast<int>(item / neb);
    const int m = rt * 64 + mm;
    double2 zv[8];
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      const int e = eb * 32 + g * 8 + jj;
      zv[jj] = (e < n && m < Rows) ? z[m + static_cast<long long>(e) * ldz] : make_double2(0.0, 0.0);
    }
    for (int b0 = 0; b0 < nbins; b0 += kDenseBins) {
      const int nb = min(kDenseBins, nbins - b0);
      __syncthreads();                                   // every read of the previous group's sf is done
      for (int i = threadIdx.x; i < nb * 32; i += 256) {
        const int bb = i >> 5, c = i & 31, e = eb * 32 + c;
        sf[bb][c] = (e < n) ? sqrt(fmax(sign * ew[static_cast<long long>(b0 + bb) * n + e], 0.0)) : 0.0;
      }
      __syncthreads();
      if (m >= Rows) continue;
      for (int bb = 0; bb < nb; ++bb) {
        const int b = b0 + bb;
        if (!(w_extent(wr, b, sign) > 0.0)) continue;
        double f[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) f[jj] = sf[bb][g * 8 + jj];
        uint4 out[NS];
        y_pack<NS>(out, f, zv, slice_unit<NS>() / mu[static_cast<long long>(b) * Rows + m]);
        const long long chunk = bin_k0[b] + eb;
#pragma unroll
        for (int q = 0; q < NS; ++q)
          *reinterpret_cast<uint4*>(y8 + ((chunk * NS + q) * Rows + m) * 64 + g * 16) = out[q];
      }
    }
  }
}

// out[0] += sum |a - b|^2, out[1] += sum |b|^2 (one atomic pair per block)
__global__ void oz_diff_norm_kernel(const double2* __restrict__ a, const double2* __restrict__ b, long long n,
                                    double* __restrict__ out) {
  __shared__ double sd[8], sb[8];
  double d = 0.0, r = 0.0;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double2 x = a[i], y = b[i];
    d += (x.x - y.x) * (x.x - y.x) + (x.y - y.y) * (x.y - y.y);
    r += y.x * y.x + y.y * y.y;
  }
  for (int o = 16; o; o >>= 1) {
    d += __shfl_xor_sync(0xffffffffu, d, o);
    r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  if ((threadIdx.x & 31) == 0) { sd[threadIdx.x >> 5] = d; sb[threadIdx.x >> 5] = r; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < static_cast<int>(blockDim.x >> 5); ++i) { d += sd[i]; r += sb[i]; }
    atomicAdd(out, d);
    atomicAdd(out + 1, r);
  }
}

// =====================================================================================
// host side

static DevBuf g_a8, g_b8, g_mu, g_nu, g_tabs;          // Sigma_c
static DevBuf g_y8, g_ymu, g_zmax, g_wr, g_bins;       // chi0

template <int NS, bool PAIRED>
static int launch_seg(const CUtensorMap& ma, const CUtensorMap& mb, const CUtensorMap& mt, const SegParams& p,
                      dim3 grid, cudaStream_t s) {
  static uint64_t attr = 0;                             // one bit per device
  int rc = smem_limit_once(reinterpret_cast<const void*>(oz_seg_kernel<NS, PAIRED>), SegCfg<NS>::SMEM, attr);
  if (rc) return rc;
  const int pi = prof_begin("sigc_seg_tc", s);
  oz_seg_kernel<NS, PAIRED><<<grid, THREADS, SegCfg<NS>::SMEM, s>>>(ma, mb, mt, p);
  prof_end(pi, s);
  count_launch();
  QSGW_LAUNCH_CHECK("oz_seg_kernel");
  return QSGW_OK;
}

template <int NS>
static int launch_herk(const CUtensorMap& ma, const CUtensorMap& mb, const HerkParams& p, dim3 grid,
                       cudaStream_t s) {
  static uint64_t attr = 0;
  int rc = smem_limit_once(reinterpret_cast<const void*>(oz_herk_kernel<NS>), Cfg<NS>::SMEM, attr);
  if (rc) return rc;
  const int pi = prof_begin("chi0_tc", s);
  oz_herk_kernel<NS><<<grid, THREADS, Cfg<NS>::SMEM, s>>>(ma, mb, p);
  prof_end(pi, s);
  count_launch();
  QSGW_LAUNCH_CHECK("oz_herk_kernel");
  return QSGW_OK;
}

static double post_scale(int ns) { return std::ldexp(1.0, -(12 + 7 * (ns - 1))); }
// the Sigma_c kernel's base-256 digits: 256^(ns-1) / U8^2
static double post_scale8(int ns) {
  const double u = ns == 2 ? slice_unit8<2>() : (ns == 3 ? slice_unit8<3>() : slice_unit8<4>());
  return std::ldexp(1.0, 8 * (ns - 1)) / (u * u);
}

}  // namespace oz

using namespace oz;

int rel_diff_fro(const double2* a, const double2* b, long long n, cudaStream_t s, double* rel) {
  static DevBuf acc;
  int rc = acc.ensure(2 * sizeof(double));
  if (rc) return rc;
  QSGW_CUDA(cudaMemsetAsync(acc.p, 0, 2 * sizeof(double), s));
  const int g = static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 8LL * ctx().sm_count)));
  oz_diff_norm_kernel<<<g, 256, 0, s>>>(a, b, n, acc.as<double>());
  count_launch();
  QSGW_LAUNCH_CHECK("oz_diff_norm_kernel");
  double h[2] = {0.0, 0.0};
  QSGW_CUDA(cudaMemcpyAsync(h, acc.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  *rel = h[1] > 0.0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
  return QSGW_OK;
}

static DevBuf g_cols;                                   // Sigma_c column map of every tile of a batch
static DevBuf g_t8;                                     // Sigma_c half-height tail slices (paired tail)

// the last row tile runs segment pairs when it has at most 32 valid rows
static bool paired_tail(int M) { return M % 64 != 0 && M % 64 <= 32; }

size_t OzSigcBatch::bytes_per(int ns, int ngb, int mrows, long long nslot, long long ntiles) {
  const long long T = (mrows + 63) / 64;
  const long long Kp = ((2LL * ngb + K8 - 1) / K8) * K8;
  return static_cast<size_t>(ns) * (nslot * T * 128 + ntiles * BN + (paired_tail(mrows) ? nslot * 64 : 0)) * Kp +
         (nslot * T * 64 + ntiles * BN) * 8 + ntiles * BN * 4;
}

int OzSigcBatch::reserve(int ns, int ngb, int mrows, long long ldc, long long nslot, long long ntiles) {
  QSGW_ARG(ns >= 2 && ns <= 4, "sigc split-i8: %d slices (2..4)", ns);
  QSGW_ARG(ngb >= 1 && mrows >= 1 && nslot >= 1 && ntiles >= 1,
           "sigc split-i8: ngb=%d rows=%d slots=%lld tiles=%lld", ngb, mrows, nslot, ntiles);
  const int T = (mrows + 63) / 64;
  const int Kp = ((2 * ngb + K8 - 1) / K8) * K8;
  // exact INT32 levels over one segment (K' = Kp, at most ns products of |d| <= 128 per level):
  // ns * 16384 * Kp < 2^31; int tile coordinates
  QSGW_ARG(static_cast<long long>(ns) * 16384 * Kp < (1LL << 31), "sigc split-i8: ngb=%d too large", ngb);
  QSGW_ARG(ns * nslot * T < (1LL << 31) && ntiles * BN < (1LL << 31),
           "sigc split-i8: batch of %lld slots, %lld tiles too large", nslot, ntiles);
  ns_ = ns; ngb_ = ngb; M_ = mrows; ldc_ = ldc; T_ = T; Kp_ = Kp;
  cap_slot_ = nslot; cap_tiles_ = ntiles;
  nslot_ = 0; ntiles_ = 0;
  tile_group_.clear(); group_seg_off_.clear(); group_nseg_.clear(); seg_slot_.clear();
  segs_.clear(); tile_out_.clear();
  int rc = g_a8.ensure(static_cast<size_t>(ns) * nslot * T * 128 * Kp);
  if (rc) return rc;
  if ((rc = g_b8.ensure(static_cast<size_t>(ns) * ntiles * BN * Kp))) return rc;
  if ((rc = g_mu.ensure(static_cast<size_t>(nslot) * T * 64 * sizeof(double)))) return rc;
  if ((rc = g_nu.ensure(static_cast<size_t>(ntiles) * BN * sizeof(double)))) return rc;
  if (paired_tail(mrows) && (rc = g_t8.ensure(static_cast<size_t>(ns) * nslot * 64 * Kp))) return rc;
  return g_cols.ensure(static_cast<size_t>(ntiles) * BN * sizeof(int));
}

int OzSigcBatch::add(const SigcSplitArgs& a, cudaStream_t s) {
  const int ngb = a.ngb;                              // K: rows of W and of the B columns
  const int M = a.mrows > 0 ? a.mrows : ngb;          // output rows: columns of W
  const long long ldz = a.ldz > 0 ? a.ldz : ngb;
  const long long ldc = a.ldc > 0 ? a.ldc : M;
  const long long wst = a.wstride > 0 ? a.wstride : a.ldw * a.ldw;   // one W record
  QSGW_ARG(cap_slot_ > 0, "sigc split-i8 batch: add before reserve");
  QSGW_ARG(ngb == ngb_ && M == M_ && ldc == ldc_,
           "sigc split-i8 batch: task ngb=%d rows=%d ldc=%lld in a batch of ngb=%d rows=%d ldc=%lld", ngb, M, ldc,
           ngb_, M_, ldc_);
  const int nslot = a.nimag + a.nreal;
  const int ntiles = static_cast<int>(a.tile_group.size());
  QSGW_ARG(a.tile_cols.size() == static_cast<size_t>(ntiles) * BN, "sigc split-i8: %zu tile columns for %d tiles",
           a.tile_cols.size(), ntiles);
  QSGW_ARG(a.group_seg_off.size() == a.group_nseg.size() && a.seg_slot.size() == a.segs.size(),
           "sigc split-i8: inconsistent segment tables");
  QSGW_ARG(nslot_ + nslot <= cap_slot_ && ntiles_ + ntiles <= cap_tiles_,
           "sigc split-i8 batch: %lld + %d slots, %lld + %d tiles over the reserved %lld, %lld", nslot_, nslot,
           ntiles_, ntiles, cap_slot_, cap_tiles_);
  for (int sl : a.seg_slot) QSGW_ARG(sl >= 0 && sl < nslot, "sigc split-i8: segment slot %d of %d", sl, nslot);
  for (int g : a.tile_group)
    QSGW_ARG(g >= 0 && g < static_cast<int>(a.group_nseg.size()), "sigc split-i8: tile group %d", g);
  for (size_t g = 0; g < a.group_nseg.size(); ++g)
    QSGW_ARG(a.group_seg_off[g] >= 0 && a.group_nseg[g] >= 0 &&
                 a.group_seg_off[g] + a.group_nseg[g] <= static_cast<int>(a.segs.size()),
             "sigc split-i8: group %zu segments %d + %d of %zu", g, a.group_seg_off[g], a.group_nseg[g],
             a.segs.size());
  const int T = T_, Kp = Kp_, ns = ns_;
  const long long slot0 = nslot_, row0 = ntiles_ * BN;
  const int nrows = ntiles * BN;
  // the task's column map: the slicing below reads it now, the contraction at launch()
  int* d_cols = g_cols.as<int>() + row0;
  int rc = h2d(d_cols, a.tile_cols.data(), a.tile_cols.size() * sizeof(int), s);
  if (rc) return rc;
  double* mu = g_mu.as<double>();
  double* nu = g_nu.as<double>() + row0;
  // row scales of A' (= column scales of every W record) and column scales of B
  oz_colscale_kernel<<<dim3((T * 64 + 7) / 8, a.nimag), 256, 0, s>>>(a.wi, a.ldw, wst, ngb, M, nullptr, T * 64,
                                                                    mu + slot0 * T * 64);
  count_launch();
  if (a.nreal > 0) {
    oz_colscale_kernel<<<dim3((T * 64 + 7) / 8, a.nreal), 256, 0, s>>>(a.wr, a.ldw, wst, ngb, M, nullptr, T * 64,
                                                                      mu + (slot0 + a.nimag) * T * 64);
    count_launch();
  }
  oz_colscale_kernel<<<dim3((nrows + 7) / 8, 1), 256, 0, s>>>(a.zmel, ldz, 0, ngb, 0, d_cols, nrows, nu);
  count_launch();
  QSGW_LAUNCH_CHECK("oz_colscale_kernel");
  const int pslice = prof_begin("sigc_slice_i8", s);
  int8_t* A8 = g_a8.as<int8_t>();
  int8_t* B8 = g_b8.as<int8_t>() + row0 * Kp;
  const int nst = static_cast<int>(cap_slot_);
  const long long rs = cap_tiles_ * BN;
  const dim3 gk(static_cast<unsigned>((Kp / 2 + 127) / 128));
  const bool tail = paired_tail(M);
  const int Tw = tail ? T - 1 : T;                     // the last row tile goes to the tail slices instead
  auto slice_w = [&](const double2* w, int n, int gslot0) {
    if (Tw > 0) {
      const dim3 g(gk.x, static_cast<unsigned>(n * Tw));
      if (ns == 2) oz_slice_w_kernel<2><<<g, 256, 0, s>>>(A8, w, a.ldw, wst, M, ngb, T, Tw, nst, gslot0, Kp, mu);
      else if (ns == 3) oz_slice_w_kernel<3><<<g, 256, 0, s>>>(A8, w, a.ldw, wst, M, ngb, T, Tw, nst, gslot0, Kp, mu);
      else oz_slice_w_kernel<4><<<g, 256, 0, s>>>(A8, w, a.ldw, wst, M, ngb, T, Tw, nst, gslot0, Kp, mu);
      count_launch();
    }
    if (tail) {                                        // the last row tile, half height
      int8_t* T8 = g_t8.as<int8_t>();
      const dim3 gt(gk.x, static_cast<unsigned>(n));
      if (ns == 2)
        oz_slice_w_kernel<2, true><<<gt, 256, 0, s>>>(T8, w, a.ldw, wst, M, ngb, T, Tw, nst, gslot0, Kp, mu);
      else if (ns == 3)
        oz_slice_w_kernel<3, true><<<gt, 256, 0, s>>>(T8, w, a.ldw, wst, M, ngb, T, Tw, nst, gslot0, Kp, mu);
      else oz_slice_w_kernel<4, true><<<gt, 256, 0, s>>>(T8, w, a.ldw, wst, M, ngb, T, Tw, nst, gslot0, Kp, mu);
      count_launch();
    }
  };
  slice_w(a.wi, a.nimag, static_cast<int>(slot0));
  if (a.nreal > 0) slice_w(a.wr, a.nreal, static_cast<int>(slot0) + a.nimag);
  {
    const dim3 g(gk.x, static_cast<unsigned>((nrows + 7) / 8));
    if (ns == 2) oz_slice_z_kernel<2><<<g, 256, 0, s>>>(B8, a.zmel, ldz, ngb, d_cols, nrows, rs, Kp, nu);
    else if (ns == 3) oz_slice_z_kernel<3><<<g, 256, 0, s>>>(B8, a.zmel, ldz, ngb, d_cols, nrows, rs, Kp, nu);
    else oz_slice_z_kernel<4><<<g, 256, 0, s>>>(B8, a.zmel, ldz, ngb, d_cols, nrows, rs, Kp, nu);
    count_launch();
  }
  QSGW_LAUNCH_CHECK("Sigma_c int8 slices");
  prof_end(pslice, s);
  // host tables of the contraction, in the batch's numbering
  const int g0 = static_cast<int>(group_nseg_.size());
  const int sg0 = static_cast<int>(segs_.size());
  for (size_t g = 0; g < a.group_nseg.size(); ++g) {
    group_seg_off_.push_back(sg0 + a.group_seg_off[g]);
    group_nseg_.push_back(a.group_nseg[g]);
  }
  for (size_t i = 0; i < a.segs.size(); ++i) {
    segs_.push_back(a.segs[i]);
    seg_slot_.push_back(static_cast<int>(slot0) + a.seg_slot[i]);
  }
  for (int t = 0; t < ntiles; ++t) {
    tile_group_.push_back(g0 + a.tile_group[t]);
    tile_out_.push_back(a.out);
  }
  nslot_ += nslot;
  ntiles_ += ntiles;
  return QSGW_OK;
}

int OzSigcBatch::launch(cudaStream_t s) {
  if (ntiles_ == 0) return QSGW_OK;
  const int T = T_, Kp = Kp_, ns = ns_;
  int rc = g_tabs.ensure((tile_group_.size() + group_seg_off_.size() + group_nseg_.size() + seg_slot_.size() + 16) *
                             sizeof(int) + segs_.size() * sizeof(ZSeg) + tile_out_.size() * sizeof(double2*) + 256);
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
  SegParams p{};
  p.segs = reinterpret_cast<const ZSeg*>(put(segs_.data(), segs_.size() * sizeof(ZSeg)));
  p.tile_out = reinterpret_cast<double2* const*>(put(tile_out_.data(), tile_out_.size() * sizeof(double2*)));
  p.tile_group = reinterpret_cast<const int*>(put(tile_group_.data(), tile_group_.size() * sizeof(int)));
  p.group_seg_off = reinterpret_cast<const int*>(put(group_seg_off_.data(), group_seg_off_.size() * sizeof(int)));
  p.group_nseg = reinterpret_cast<const int*>(put(group_nseg_.data(), group_nseg_.size() * sizeof(int)));
  p.seg_slot = reinterpret_cast<const int*>(put(seg_slot_.data(), seg_slot_.size() * sizeof(int)));
  if (cprc) return cprc;
  const long long nrows = cap_tiles_ * BN;
  // maps: A' [Kp, 64, 2, ns * cap_slot * T] box {64, 64, 2, 1}; B [Kp, cap_rows, ns] box {64, 128, 1}
  CUtensorMap ma, mb;
  {
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(Kp), 64, 2, static_cast<cuuint64_t>(ns) * cap_slot_ * T};
    const cuuint64_t str[3] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(Kp) * 64,
                               static_cast<cuuint64_t>(Kp) * 128};
    const cuuint32_t box[4] = {K8, 64, 2, 1};
    rc = make_tensor_map(&ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, g_a8.p, 4, dims, str, box, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc) return rc;
  }
  {
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(nrows),
                                static_cast<cuuint64_t>(ns)};
    const cuuint64_t str[2] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(Kp) * nrows};
    const cuuint32_t box[3] = {K8, BN, 1};
    rc = make_tensor_map(&mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, g_b8.p, 3, dims, str, box, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc) return rc;
  }
  // paired tail: T8 [Kp, 32, 2, ns * cap_slot] box {64, 32, 1, 1} (one half of one slot's tail rows);
  // without it the map is a copy of A's and never read
  CUtensorMap mt = ma;
  const bool tail = paired_tail(M_);
  if (tail) {
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(Kp), 32, 2, static_cast<cuuint64_t>(ns) * cap_slot_};
    const cuuint64_t str[3] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(Kp) * 32,
                               static_cast<cuuint64_t>(Kp) * 64};
    const cuuint32_t box[4] = {K8, 32, 1, 1};
    rc = make_tensor_map(&mt, CU_TENSOR_MAP_DATA_TYPE_UINT8, g_t8.p, 4, dims, str, box, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc) return rc;
  }
  p.tail = tail ? 1 : 0;
  p.M = M_;
  p.ntm = T;
  p.cps = Kp / K8;
  p.nslot = static_cast<int>(cap_slot_);
  p.T = T;
  p.nrows = static_cast<int>(nrows);
  p.tile_cols = g_cols.as<int>();
  p.mu_a = g_mu.as<double>(); p.nu_b = g_nu.as<double>();
  p.post = post_scale8(ns);
  p.ldc = ldc_;
  p.err = ctx().d_flags + 1;
  // the full row tiles in one launch, the paired last row tile (if any) in a second
  const int tmain = tail ? T - 1 : T;
  p.ntm = tmain;
  const long long nt_all = ntiles_;
  nslot_ = 0; ntiles_ = 0; cap_slot_ = 0; cap_tiles_ = 0;      // the next batch starts with reserve()
  auto run = [&](auto nsc) -> int {
    constexpr int NSV = decltype(nsc)::value;
    int r = QSGW_OK;
    if (tmain > 0) r = launch_seg<NSV, false>(ma, mb, mt, p, dim3(static_cast<unsigned>(tmain * nt_all)), s);
    if (!r && tail) r = launch_seg<NSV, true>(ma, mb, mt, p, dim3(static_cast<unsigned>(nt_all)), s);
    return r;
  };
  if (ns == 2) return run(std::integral_constant<int, 2>());
  if (ns == 3) return run(std::integral_constant<int, 3>());
  return run(std::integral_constant<int, 4>());
}

int sigc_split_i8(const SigcSplitArgs& a, int ns, cudaStream_t s) {
  const int M = a.mrows > 0 ? a.mrows : a.ngb;
  const long long ldc = a.ldc > 0 ? a.ldc : M;
  if (a.tile_group.empty()) return QSGW_OK;
  OzSigcBatch b;
  int rc = b.reserve(ns, a.ngb, M, ldc, a.nimag + a.nreal, static_cast<long long>(a.tile_group.size()));
  if (rc) return rc;
  if ((rc = b.add(a, s))) return rc;
  return b.launch(s);
}

int zgemm_ch_i8(double2* C, long long ldc, int M, int N, int K, const double2* W, long long ldw, const double2* B,
                long long ldb, int ns, cudaStream_t s) {
  if (M <= 0 || N <= 0) return QSGW_OK;
  static DevBuf g_one;
  int rc = g_one.ensure(sizeof(double));
  if (rc) return rc;
  const double one = 1.0;
  if ((rc = h2d(g_one.p, &one, sizeof(double), s))) return rc;
  SigcSplitArgs a;
  a.ngb = K; a.mrows = M; a.ldz = ldb; a.ldc = ldc;
  a.ldw = ldw;
  a.wi = W; a.nimag = 1;
  a.wr = nullptr; a.nreal = 0;
  a.zmel = B; a.ncol = N;
  a.wgt = nullptr; a.nwgt = 0; a.w3 = nullptr; a.nw3 = 0;
  const int ntiles = (N + BN - 1) / BN;
  for (int t = 0; t < ntiles; ++t) {
    a.tile_group.push_back(0);
    for (int j = 0; j < BN; ++j) a.tile_cols.push_back(t * BN + j < N ? t * BN + j : -1);
  }
  a.group_seg_off.push_back(0);
  a.group_nseg.push_back(1);
  a.seg_slot.push_back(0);
  a.segs.push_back(ZSeg{W, g_one.as<double>(), 0, 0});        // unit weight for every column
  a.out = C;
  return sigc_split_i8(a, ns, s);
}

int chi0_split_i8(double2* C, long long ldc, long long c_bs, int M, int N, int row_b0, bool herm, const double2* z,
                  long long ldz, long long ncols, const int* ecol_d, const double* ew_d, const OzChi0Bins& bins,
                  int classes, int ns, cudaStream_t s, const char* tune_key) {
  QSGW_ARG(ns >= 2 && ns <= 4, "chi0 split-i8: %d slices (2..4)", ns);
  const int nbins = static_cast<int>(bins.cnt.size());
  if (nbins == 0 || M <= 0 || N <= 0 || (classes & 3) == 0) return QSGW_OK;
  QSGW_ARG(nbins <= 65535, "chi0 split-i8: %d bins exceed the grid limit", nbins);
  const int Rows = std::max(M, row_b0 + N);
  // bin layout in Y8: each bin padded to whole 64-byte chunks (32 entries)
  std::vector<long long> k0(nbins);
  std::vector<int> nch(nbins);
  long long tot = 0;
  int maxch = 0;
  for (int b = 0; b < nbins; ++b) {
    k0[b] = tot;
    nch[b] = (bins.cnt[b] + 31) / 32;
    tot += nch[b];
    maxch = std::max(maxch, nch[b]);
  }
  const long long Ktot = tot * K8;
  QSGW_ARG(tot < (1LL << 31), "chi0 split-i8: %lld K chunks exceed the TMA coordinate range", tot);
  int rc = g_y8.ensure(static_cast<size_t>(ns) * Rows * Ktot);
  if (rc) return rc;
  rc = g_ymu.ensure(static_cast<size_t>(nbins) * Rows * sizeof(double));
  if (rc) return rc;
  rc = g_zmax.ensure(static_cast<size_t>(Rows) * sizeof(unsigned long long));
  if (rc) return rc;
  rc = g_wr.ensure(static_cast<size_t>(2 * nbins) * sizeof(double));
  if (rc) return rc;
  const size_t tb = static_cast<size_t>(nbins) * (2 * sizeof(long long) + 2 * sizeof(int));
  rc = g_bins.ensure(tb + 64);
  if (rc) return rc;
  unsigned char* base = g_bins.as<unsigned char>();
  long long* d_k0 = reinterpret_cast<long long*>(base);
  long long* d_eb = d_k0 + nbins;
  int* d_nch = reinterpret_cast<int*>(d_eb + nbins);
  int* d_cnt = d_nch + nbins;
  int* d_slab = nullptr;
  {
    // the slab table follows in a second small copy (keeps the four arrays 8-byte aligned)
    static DevBuf g_slab;
    rc = g_slab.ensure(static_cast<size_t>(nbins) * sizeof(int));
    if (rc) return rc;
    d_slab = g_slab.as<int>();
    if ((rc = h2d(d_slab, bins.slab.data(), nbins * sizeof(int), s))) return rc;
  }
  if ((rc = h2d(d_k0, k0.data(), nbins * sizeof(long long), s))) return rc;
  if ((rc = h2d(d_eb, bins.ebeg.data(), nbins * sizeof(long long), s))) return rc;
  if ((rc = h2d(d_nch, nch.data(), nbins * sizeof(int), s))) return rc;
  if ((rc = h2d(d_cnt, bins.cnt.data(), nbins * sizeof(int), s))) return rc;
  unsigned long long* zmax = g_zmax.as<unsigned long long>();
  QSGW_CUDA(cudaMemsetAsync(zmax, 0, static_cast<size_t>(Rows) * sizeof(unsigned long long), s));
  {
    const int g = static_cast<int>(std::max<long long>(1, std::min<long long>(ncols, 8LL * ctx().sm_count)));
    oz_rowmax_kernel<<<g, 256, 0, s>>>(z, ldz, Rows, ncols, zmax);
    count_launch();
  }
  QSGW_CUDA(cudaMemsetAsync(g_wr.p, 0, static_cast<size_t>(2 * nbins) * sizeof(double), s));
  {
    const int per = std::max(1, std::min(64, static_cast<int>((maxch * 32LL + 4095) / 4096)));
    oz_wrange_kernel<<<dim3(static_cast<unsigned>(per), static_cast<unsigned>(nbins)), 256, 0, s>>>(
        ew_d, d_eb, d_cnt, reinterpret_cast<unsigned long long*>(g_wr.p));
    count_launch();
  }
  QSGW_LAUNCH_CHECK("chi0 int8 ranges");
  int8_t* Y8 = g_y8.as<int8_t>();
  double* mu = g_ymu.as<double>();
  CUtensorMap ma, mb;
  {
    // [chunk][slice][row][64 B]: rows beyond Rows read as zero, boxes never cross a slice
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(K8), static_cast<cuuint64_t>(Rows),
                                static_cast<cuuint64_t>(ns), static_cast<cuuint64_t>(tot)};
    const cuuint64_t str[3] = {static_cast<cuuint64_t>(K8), static_cast<cuuint64_t>(K8) * Rows,
                               static_cast<cuuint64_t>(K8) * Rows * ns};
    const cuuint32_t boxa[4] = {K8, 64, 1, 1};
    const cuuint32_t boxb[4] = {K8, BN, 1, 1};
    rc = make_tensor_map(&ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, Y8, 4, dims, str, boxa, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc) return rc;
    rc = make_tensor_map(&mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, Y8, 4, dims, str, boxb, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc) return rc;
  }
  const int ntm = (M + 63) / 64, ntn = (N + BN - 1) / BN;
  long long units = 0;
  for (int nt = 0; nt < ntn; ++nt)
    for (int mt = 0; mt < ntm; ++mt)
      if (!herm || mt * 64 + 63 >= nt * BN) ++units;
  units *= nbins;
  // split K so that one wave of CTAs covers whole (bin, K part) units: the tiles of a unit share its
  // rows of Y8 through L2 only while they run together
  const long long tiles_per_bin = units / nbins;
  const int maxsplit = std::max(1, std::min(maxch / 4, 64));
  int heur = static_cast<int>(std::max<long long>(1, (ctx().sm_count + tiles_per_bin / 2) / tiles_per_bin));
  heur = std::min(heur, maxsplit);
  // every bin over the same columns in order, weights at ew[b * n + e]: z is sliced in one pass
  bool dense = ecol_d == nullptr;
  for (int b = 0; b < nbins && dense; ++b) dense = bins.cnt[b] == bins.cnt[0] && bins.ebeg[b] == static_cast<long long>(b) * bins.cnt[0];
  HerkParams p{};
  p.M = M; p.N = N; p.ntm = ntm; p.herm = herm ? 1 : 0; p.row_b0 = row_b0; p.Rows = Rows;
  p.bin_k0 = d_k0; p.bin_nch = d_nch; p.bin_slab = d_slab; p.wrange = g_wr.as<double>(); p.mu = mu;
  p.post = post_scale(ns);
  p.C = C; p.ldc = ldc; p.c_bs = c_bs;
  p.err = ctx().d_flags + 1;
  auto run_class = [&](double sign, int splitk) -> int {
    const int nmu = nbins * Rows;
    oz_mu_kernel<<<(nmu + 255) / 256, 256, 0, s>>>(zmax, g_wr.as<double>(), Rows, nbins, sign, mu);
    count_launch();
    const long long items = static_cast<long long>(maxch) * ((Rows + 63) / 64);   // (32-entry block, 64 rows)
    const int pslice = prof_begin("chi0_slice_i8", s);
    if (dense) {
      const int n = bins.cnt[0];
      const unsigned gd = static_cast<unsigned>(std::max<long long>(1, std::min<long long>(items, 16LL * ctx().sm_count)));
      if (ns == 2) oz_slice_y_dense_kernel<2><<<gd, 256, 0, s>>>(Y8, Rows, z, ldz, n, nbins, ew_d, d_k0,
                                                                 g_wr.as<double>(), mu, sign);
      else if (ns == 3) oz_slice_y_dense_kernel<3><<<gd, 256, 0, s>>>(Y8, Rows, z, ldz, n, nbins, ew_d, d_k0,
                                                                      g_wr.as<double>(), mu, sign);
      else oz_slice_y_dense_kernel<4><<<gd, 256, 0, s>>>(Y8, Rows, z, ldz, n, nbins, ew_d, d_k0,
                                                         g_wr.as<double>(), mu, sign);
      count_launch();
      QSGW_LAUNCH_CHECK("oz_slice_y_dense_kernel");
      prof_end(pslice, s);
      HerkParams q = p;
      q.sign = sign;
      const dim3 grid(static_cast<unsigned>(ntm * ntn), static_cast<unsigned>(nbins), static_cast<unsigned>(splitk));
      if (ns == 2) return launch_herk<2>(ma, mb, q, grid, s);
      if (ns == 3) return launch_herk<3>(ma, mb, q, grid, s);
      return launch_herk<4>(ma, mb, q, grid, s);
    }
    const dim3 gy(static_cast<unsigned>(std::max<long long>(1, std::min<long long>(items, 4LL * ctx().sm_count))),
                  static_cast<unsigned>(nbins));
    if (ns == 2) oz_slice_y_kernel<2><<<gy, 256, 0, s>>>(Y8, Rows, z, ldz, ecol_d, ew_d, d_eb, d_cnt, d_k0,
                                                         g_wr.as<double>(), mu, sign);
    else if (ns == 3) oz_slice_y_kernel<3><<<gy, 256, 0, s>>>(Y8, Rows, z, ldz, ecol_d, ew_d, d_eb, d_cnt, d_k0,
                                                              g_wr.as<double>(), mu, sign);
    else oz_slice_y_kernel<4><<<gy, 256, 0, s>>>(Y8, Rows, z, ldz, ecol_d, ew_d, d_eb, d_cnt, d_k0,
                                                 g_wr.as<double>(), mu, sign);
    count_launch();
    QSGW_LAUNCH_CHECK("oz_slice_y_kernel");
    prof_end(pslice, s);
    HerkParams q = p;
    q.sign = sign;
    const dim3 grid(static_cast<unsigned>(ntm * ntn), static_cast<unsigned>(nbins), static_cast<unsigned>(splitk));
    if (ns == 2) return launch_herk<2>(ma, mb, q, grid, s);
    if (ns == 3) return launch_herk<3>(ma, mb, q, grid, s);
    return launch_herk<4>(ma, mb, q, grid, s);
  };
  auto run = [&](int splitk, bool clear) -> int {
    if (clear) {
      for (int b = 0; b < nbins; ++b) {
        // only the slabs this call writes; the slab tables of the callers are distinct per bin
        QSGW_CUDA(cudaMemsetAsync(C + static_cast<long long>(bins.slab[b]) * c_bs, 0,
                                  static_cast<size_t>(ldc) * N * sizeof(double2), s));
      }
    }
    int r = QSGW_OK;
    if (classes & 1) r = run_class(-1.0, splitk);
    if (!r && (classes & 2)) r = run_class(1.0, splitk);
    return r;
  };
  std::vector<int> cands;
  for (int c : {1, 2, 3, 4, 5, 6, 8})
    if (c <= maxsplit) cands.push_back(c);
  if (heur > 8) cands.push_back(heur);
  char key[200];
  std::snprintf(key, sizeof(key), "%s i8x%d M=%d N=%d bins=%d chunks~2^%.3f", tune_key ? tune_key : "-", ns, M, N, nbins,
                std::round(8.0 * std::log2(static_cast<double>(std::max(1, maxch)))) / 8.0);
  if (!tune_key) return run(heur, false);              // accumulating callers: no trials
  int splitk = heur;
  bool tried = false;
  rc = tuned_choice(key, cands, heur, [&](int c) { return run(c, true); }, s, &splitk, &tried);
  if (rc) return rc;
  return run(splitk, tried);
}

}  // namespace qsgw
