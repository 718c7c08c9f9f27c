// Shared pieces of the split-FP16 tcgen05 kernels (split_f16.cu: the chi0 and
// Sigma_c kernel; split_sigc_variants.cu: the opt-in Sigma_c variants): tile
// constants, launch parameters and the PTX helpers (mbarrier waits bounded by
// an iteration count, TMA loads, swizzled shared-memory descriptors, MMA and
// TMEM access).
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "split_f16.cuh"

namespace qsgw {
namespace tc {

constexpr int BM2 = 128;                 // real accumulator rows (64 complex x {re, im})
constexpr int BMC = 64;                  // complex rows per tile
constexpr int NC = 128;                  // complex columns per tile (UMMA N)
constexpr int KC = 64;                   // FP16 elements per chunk along K' (32 complex k)
constexpr int NTHREADS = 576;            // warp 0 TMA, 1 MMA, 2..9 converters, 10..17 drain
constexpr int NCONV = 256;               // converter threads (warps 2..9), two per B' row
constexpr int CONV_W0 = 2, DRAIN_W0 = 10;
constexpr int NDRAIN_WARPS = 8;          // chi0 drain warps 10..17 (64 columns each); Sigma_c: warps 2..17 (32 each)
constexpr int NBUF = 3;                  // B' buffers
constexpr int DRAIN_PERIOD = 2;          // K chunks per FP32 accumulation run (24 MMAs)
constexpr int SLICE_A = BM2 * KC * 2;    // 16 KB
constexpr int SLICE_S = NC * KC * 2;     // 16 KB
constexpr int SLICE_B = NC * KC * 2;     // 16 KB
constexpr uint32_t TMEM_COLS = 512;                      // acc0 [0,128) acc1 [128,256) FP64 sums [256,512)
constexpr uint32_t FP64_COL = 256;
constexpr long long WAIT_LIMIT = 1LL << 24;              // bounded spin (several seconds)

enum { MODE_CHI0 = 0, MODE_SEG = 1 };

// Shared-memory layout per mode.  chi0: two TMA stages (A' and S, hi and lo
// slices) and three B' buffers.  Sigma_c multiplies by S directly, so the B'
// area only holds the drain warps' per-column weights and a third stage fits.
template <int MODE>
struct Cfg {
  static constexpr int NST = MODE == MODE_SEG ? 3 : 2;            // TMA stages
  static constexpr int BAREA = MODE == MODE_SEG ? 2 * 8 * 64 * 8 : NBUF * 2 * SLICE_B;
  static constexpr int OFF_A = 0;
  static constexpr int OFF_S = OFF_A + NST * 2 * SLICE_A;
  static constexpr int OFF_B = OFF_S + NST * 2 * SLICE_S;
  static constexpr int OFF_BAR = OFF_B + BAREA;
  static constexpr int NBAR = 2 * NST + 2 * NBUF + 2 + 2 + 1;
  static constexpr int OFF_MISC = OFF_BAR + NBAR * 8;
  static constexpr int SMEM_BYTES = OFF_MISC + 64 + 1024;         // + slack for 1024-B alignment
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
};

struct Params {
  int mode;
  int M, N;                 // complex rows / columns of C
  int ntm, ntn;
  int kch_total, kch_per_split, cps;
  // chi0
  const double* w;          // w[iw * npair + p]
  const float* w32;         // w * sigma_B(iw) in FP32, rows of w32_ld (multiple of 32, zero padded)
  long long w32_ld;
  long long npair;
  int niw;
  // seg
  const int* tile_group;
  const int* tile_cols;
  const int* group_seg_off;
  const int* group_nseg;
  const int* seg_slot;      // A' slot of every segment
  const ZSeg* segs;         // scale pointer / column stride of every segment
  int herm;                 // chi0: skip tiles above the diagonal, mirror the lower part
  int tiles_per_slot;       // m-tiles of one A' slot
  int lo_tile_off;          // tile offset of the lo slice in the A' map
  int lo_row_off;           // row (2-D) / tile (4-D) offset of the lo slice in the S map
  // output
  double2* C;
  long long ldc, c_bs;
  const double* scales;     // [0] sigma_A, [1] sigma_S, [2 + j] sigma_B(j)
  int* err;
  double* scratch;          // Sigma_c on 256-column tiles: FP64 sums, 256 x 128 per CTA
};

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and raises the CTA abort flag) on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    if (mbar_try(b, parity)) return true;
    if (*abort_flag) return false;
    if (i > 64) __nanosleep(64);
  }
  *abort_flag = 1;
  return false;
}
// Warp-uniform bounded wait: lane 0 polls, every lane gets the same answer.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  int ok = 0;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(b, parity, abort_flag) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}
// Bounded wait that ignores the abort flag: used only to drain the CTA's own
// in-flight TMA / MMA work before it frees TMEM and exits.
__device__ __forceinline__ void mbar_drain(uint64_t* b, uint32_t parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    if (mbar_try(b, parity)) return;
    if (i > 64) __nanosleep(64);
  }
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2),
        "r"(c3)
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}

// K-major, 128-byte swizzle UMMA shared-memory descriptor: rows of 128 B in
// 8-row atoms (SBO = 1024 B), version 1, layout type SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFF);
  d |= static_cast<uint64_t>(1) << 16;                 // LBO (unused for swizzled K-major)
  d |= static_cast<uint64_t>(1024 >> 4) << 32;         // SBO
  d |= static_cast<uint64_t>(1) << 46;                 // version
  d |= static_cast<uint64_t>(2) << 61;                 // SWIZZLE_128B
  return d;
}
// K-major, 64-byte swizzle: rows of 64 B in 8-row atoms (SBO = 512 B), layout type SWIZZLE_64B
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFF);
  d |= static_cast<uint64_t>(1) << 16;
  d |= static_cast<uint64_t>(512 >> 4) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(4) << 61;
  return d;
}
// kind::f16, A = B = F16, D = F32, both K-major, M = 128, N = NC
constexpr uint32_t IDESC = (1u << 4) | (static_cast<uint32_t>(NC >> 3) << 17) | (static_cast<uint32_t>(BM2 >> 4) << 24);

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(IDESC), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};"
      ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
        "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]),
        "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]),
        "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}
__device__ __forceinline__ void tmem_ld32w(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 8-lane TMEM load: 32 lanes x 8 consecutive 32-bit columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// Tiled tensor map over `base` (host side, split_f16.cu): dims / strides in elements / bytes as
// cuTensorMapEncodeTiled takes them, no interleave, 256-byte L2 promotion, zero fill out of range.
int make_tensor_map(CUtensorMap* map, CUtensorMapDataType dtype, void* base, int rank, const cuuint64_t* dims,
                    const cuuint64_t* strides_bytes, const cuuint32_t* box, CUtensorMapSwizzle swz);

// offset of the 16-byte chunk `c` of row `r` inside a 128B-swizzled tile
__device__ __forceinline__ int sw128_off(int r, int c) { return r * 128 + ((c ^ (r & 7)) << 4); }

// ---- the opt-in Sigma_c variants (split_sigc_variants.cu)
constexpr int NW = 256;                          // complex columns of a 64 x 256 tile (UMMA N)
constexpr int KCW = 32;                          // its FP16 elements per K chunk (64-byte swizzled rows)
// Sigma_c on CTA pairs (clusters of two): grid.x = 2 * ceil(row tiles / 2) * column tiles
int launch_sigc_pair(const CUtensorMap& ma, const CUtensorMap& ms, const Params& p, dim3 grid, cudaStream_t s,
                     const char* tag);
// Sigma_c on 64 x 256 tiles: grid.x = row tiles * column tiles
int launch_sigc_wide(const CUtensorMap& ma, const CUtensorMap& ms, Params p, dim3 grid, cudaStream_t s,
                     const char* tag);

}  // namespace tc
}  // namespace qsgw
