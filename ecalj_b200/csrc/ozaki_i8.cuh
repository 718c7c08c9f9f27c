// Ozaki-scheme int8 complex contractions (tcgen05.mma kind::i8, exact INT32
// accumulation): the Sigma_c segmented product and the binned chi0 rank-k
// update.  ozaki_i8.cu holds the kernels and the scheme.
#pragma once
#include <vector>
#include "split_f16.cuh"

namespace qsgw {

// columns per output tile of the int8 Sigma_c kernel (the column tables are cut to it)
constexpr int kOzTileN = 128;

// The Sigma_c segmented contraction of SigcSplitArgs (tables cut to kOzTileN
// columns per tile) with ns int8 slices per operand (2..4).
int sigc_split_i8(const SigcSplitArgs& a, int ns, cudaStream_t s);

// Several such contractions of one shape (equal ngb, row count and ldc; each task with its own W
// records, zmel, weights and output) in ONE launch of the int8 kernel.  reserve() sizes the slice
// buffers for the whole batch (slots = sum of nimag + nreal, tiles = sum of the tile counts);
// add() slices one task into them on stream s -- its W records and zmel may be overwritten by
// work enqueued after add(), its weight tables (the ZSeg scales) and output must stay valid until
// launch(); launch() runs the tiles of every added task, task after task, and ends the batch.
// The outputs are those of one sigc_split_i8 call per task, bit for bit.  One batch at a time
// (the slice buffers are the library's).
class OzSigcBatch {
 public:
  int reserve(int ns, int ngb, int mrows, long long ldc, long long nslot, long long ntiles);
  int add(const SigcSplitArgs& a, cudaStream_t s);
  int launch(cudaStream_t s);
  // device bytes of the slice buffers for nslot slots and ntiles tiles
  static size_t bytes_per(int ns, int ngb, int mrows, long long nslot, long long ntiles);

 private:
  int ns_ = 0, ngb_ = 0, M_ = 0, T_ = 0, Kp_ = 0;
  long long ldc_ = 0, cap_slot_ = 0, cap_tiles_ = 0, nslot_ = 0, ntiles_ = 0;
  std::vector<int> tile_group_, group_seg_off_, group_nseg_, seg_slot_;
  std::vector<ZSeg> segs_;
  std::vector<double2*> tile_out_;
};

// Binned chi0 rank-k update:
//   C(:, :, slab[b]) += sum_{e in bin b} w_e conj(z_col(e)(0:M)) z_col(e)(row_b0 : row_b0+N)^T
// with bin b's entries e in [ebeg[b], ebeg[b] + cnt[b]); col(e) = ecol_d[e], or e - ebeg[b]
// when ecol_d is null (every bin runs over the columns 0..cnt-1 in order); w_e = ew_d[e].
// herm (row_b0 == 0, N == M): lower tiles only, mirrored.  classes: bit 0 = the bins may hold
// negative weights, bit 1 = positive ones (each present sign is one pass).
struct OzChi0Bins {
  std::vector<long long> ebeg;
  std::vector<int> cnt, slab;
};
int chi0_split_i8(double2* C, long long ldc, long long c_bs, int M, int N, int row_b0, bool herm,
                  const double2* z, long long ldz, long long ncols, const int* ecol_d, const double* ew_d,
                  const OzChi0Bins& bins, int classes, int ns, cudaStream_t s, const char* tune_key);

// C = W^H B (C: M x N, ldc; W: K x M, ldw; B: K x N, ldb) on the int8 path with ns slices,
// C overwritten: the Sigma_c kernel with one segment of unit weight.
int zgemm_ch_i8(double2* C, long long ldc, int M, int N, int K, const double2* W, long long ldw, const double2* B,
                long long ldb, int ns, cudaStream_t s);

// ||a - b||_F / ||b||_F of two complex device arrays of n elements (synchronises s)
int rel_diff_fro(const double2* a, const double2* b, long long n, cudaStream_t s, double* rel);

}  // namespace qsgw
