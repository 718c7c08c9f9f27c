// Split-FP16 (Ozaki-style) complex contractions on the tcgen05 tensor cores.
#pragma once
#include "zgemm_f64.cuh"

namespace qsgw {

// chi0(:,:,iw) += sum_p w[iw*npair + p] conj(z_p) z_p^T for every iw, where
// z_p is column p of zcols (npr x npair, leading dimension ldz).
int chi0_split_f16(double2* chi0, int npr, int niw, const double2* zcols, int ldz,
                   long long npair, const double* w, cudaStream_t s);

// Sigma_c segmented contraction (same problem description as the FP64
// ZM_SEG launch): C(:, col) = sum_seg op(A_seg) * s_seg(col) * Z(:, col).
int sigc_seg_split_f16(const ZParams& p, int ncol_tiles, cudaStream_t s);

}  // namespace qsgw
