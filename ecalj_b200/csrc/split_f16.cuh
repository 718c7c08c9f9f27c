// Split-FP16 (Ozaki-style) complex contractions on the tcgen05 tensor cores.
#pragma once
#include <vector>
#include "zgemm_f64.cuh"

namespace qsgw {

// chi0(:,:,iw) += sum_p w[iw*npair + p] conj(z_p) z_p^T for every iw, where
// z_p is column p of zcols (npr x npair, leading dimension ldz).
int chi0_split_f16(double2* chi0, int npr, int niw, const double2* zcols, int ldz,
                   long long npair, const double* w, cudaStream_t s);

// Sigma_c imaginary-axis + pole contraction (the segmented problem of the
// FP64 ZM_SEG launch) in split FP16:  out(:, col) = sum over the segments of
// the column's group of  W_slot^H (scale_seg(col) z_col).
struct SigcSplitArgs {
  int ngb;
  long long ldw;                       // leading dimension of every W record
  const double2* wi; int nimag;        // imaginary-axis stack (slots 0..nimag-1)
  const double2* wr; int nreal;        // symmetrised real-axis records (slots nimag..)
  const double2* zmel; long long ncol; // zmel columns (ngb each)
  const double* wgt; long long nwgt;   // every imaginary weight (for the scale)
  const double* w3; long long nw3;     // every pole weight
  std::vector<int> tile_cols, tile_group, group_seg_off, group_nseg, seg_slot;  // sigc_split_tile_width() columns
  std::vector<ZSeg> segs;
  double2* out;                        // (ngb, ncol), overwritten
  // int8 path only: a non-square product C = W^H B with W (ngb x mrows), B (ngb x ncol, leading
  // dimension ldz), C (mrows x ncol, leading dimension ldc); 0 = ngb for each
  int mrows = 0;
  long long ldz = 0, ldc = 0;
  long long wstride = 0;               // elements between W records; 0 = ldw * ldw
};
int sigc_split_f16(const SigcSplitArgs& a, cudaStream_t s);
// columns per tile of the selected split Sigma_c kernel (the tables are cut to it)
int sigc_split_tile_width();
// The split-FP16 Sigma_c kernel kind (0, 1, 2 as qsgw_set_sigc_kernel): whether the caller fixed
// it (qsgw_set_sigc_kernel or QSGW_SIGC_KERNEL), and the kind the following calls use (the
// autotuner's choice for their shape otherwise).
bool sigc_kind_fixed();
void sigc_kind_use(int kind);

}  // namespace qsgw
