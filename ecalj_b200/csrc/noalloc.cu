// Allocation-free variant of the batched Hermitian positive definite inverse
// (qsgw_zminv_hpd_batched_d).  Its Gauss-Jordan panel scratch and status word
// live in one file-scope static device array, so a call performs no
// cudaMalloc / cudaFree and needs no qsgw_init: it is for callers that cannot
// allocate device memory at that point.
#include "zgemm_f64.cuh"

namespace qsgw {

int zminv_hpd_batched_explicit(double2* A, int n, long long lda, long long a_bs, int nbatch, double2* rb,
                               double2* qb, int* flag, cudaStream_t s);

namespace {

constexpr int kPanel = 32;                       // Gauss-Jordan block width
constexpr long long kMaxCols = 16384;            // n * nbatch limit
constexpr long long kPanelElems = kPanel * kMaxCols;
// [0, kPanelElems) R panels, [kPanelElems, 2 kPanelElems) Q panels, then the status word.
// 2 * 32 * 16384 * 16 B = 16 MiB (+256 B) held by every GPU that loads the library.
static __device__ __align__(256) double2 g_gj_scratch[2 * kPanelElems + 16];

constexpr int kMaxDevices = 64;
static double2* g_scratch_ptr[kMaxDevices] = {};

// Device address of the static array for the current device; the host-side
// symbol is only a stand-in, so it is resolved once per device with that
// device current.
int scratch_for_current_device(double2** out) {
  int dev = 0;
  QSGW_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("zminv_hpd_noalloc: device %d beyond the %d supported", dev, kMaxDevices);
    return QSGW_ERR_UNSUPPORTED;
  }
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_gj_scratch);
    if (e != cudaSuccess || p == nullptr) return check_cuda(e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                                                           "cudaGetSymbolAddress(g_gj_scratch)");
    g_scratch_ptr[dev] = static_cast<double2*>(p);
  }
  *out = g_scratch_ptr[dev];
  return QSGW_OK;
}

}  // namespace
}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_zminv_hpd_batched_noalloc_d(double* a, int n, int lda, int nbatch, void* stream) {
  QSGW_ARG(a && n >= 0 && nbatch >= 0 && lda >= (n > 1 ? n : 1),
           "zminv_hpd_noalloc: n=%d lda=%d nbatch=%d", n, lda, nbatch);
  QSGW_ARG((reinterpret_cast<uintptr_t>(a) & 15) == 0, "zminv_hpd_noalloc: array must be 16-byte aligned");
  QSGW_ARG(static_cast<long long>(n) * nbatch <= kMaxCols,
           "zminv_hpd_noalloc: n*nbatch = %lld exceeds the static scratch limit %lld",
           static_cast<long long>(n) * nbatch, kMaxCols);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  QSGW_CUDA(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    set_error("zminv_hpd_noalloc: the call waits for its stream to read the status word, so it cannot be "
              "recorded into a CUDA graph");
    return QSGW_ERR_UNSUPPORTED;
  }
  if (n == 0 || nbatch == 0) return QSGW_OK;
  double2* base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  int* status = reinterpret_cast<int*>(base + 2 * kPanelElems);
  QSGW_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));          // the array keeps the last call's status
  rc = zminv_hpd_batched_explicit(reinterpret_cast<double2*>(a), n, lda, static_cast<long long>(lda) * n, nbatch,
                                  base, base + kPanelElems, status, s);
  if (rc) return rc;
  int h = 0;
  QSGW_CUDA(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  if (h) {
    set_error("zminv_hpd_noalloc: a pivot block was singular or not finite");
    return QSGW_ERR_NUMERIC;
  }
  return QSGW_OK;
}
