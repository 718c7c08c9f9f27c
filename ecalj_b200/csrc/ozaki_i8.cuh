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
