// Split-FP16 tcgen05 path (placeholder until the kernel lands).
#include "split_f16.cuh"

namespace qsgw {

int chi0_split_f16(double2*, int, int, const double2*, int, long long, const double*, cudaStream_t) {
  set_error("split-FP16 chi0 is not built yet");
  return QSGW_ERR_UNSUPPORTED;
}

int sigc_seg_split_f16(const ZParams&, int, cudaStream_t) {
  set_error("split-FP16 Sigma_c is not built yet");
  return QSGW_ERR_UNSUPPORTED;
}

}  // namespace qsgw
