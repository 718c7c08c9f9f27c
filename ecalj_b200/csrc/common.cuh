// Shared helpers for libqsgw_b200: error plumbing, the library context and
// its device scratch buffers.  All entry points return 0 or a negative
// qsgw_status code and never abort; qsgw_last_error() returns the text.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "qsgw_b200.h"

namespace qsgw {

struct Context {
  bool initialized = false;
  int device = -1;
  cudaStream_t stream = nullptr;      // stream every entry point launches on
  bool own_stream = false;
  int prec_mode = QSGW_PREC_FP64;     // runtime precision switch
  int nslices = 2;                    // SPLIT_I8: 0 = chosen per contraction by the accuracy targets
  double sigc_qp_tol = 1e-3 / 27.211386245988;   // Hartree: largest |Re Sigma_c,nn| change allowed (1 meV)
  double chi0_rel_tol = 2e-5;         // relative Frobenius error allowed on chi0
  int sm_count = 148;
  int* d_flags = nullptr;             // device-side error/status words
  // CUDA graph of one recorded call sequence (qsgw_graph_*)
  bool capturing = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<void*> graph_host;      // pinned copies of host tables the graph reads
};

Context& ctx();
void set_error(const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what);

// Grows-only device scratch buffer owned by the library.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t n);
  void release();
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

int require_init();
// Host -> device copy of a small host table on stream s.  Outside capture it
// copies from the caller's memory; while a graph is being recorded the data
// is first copied into pinned memory owned by the graph, which the recorded
// copy node reads at every replay.
int h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);
// kernels launched by this library since init (qsgw_launch_count)
void count_launch(int n = 1);

// Optional per-kernel timing with CUDA events on the launch stream
// (qsgw_profile).  prof_begin returns -1 when profiling is off.
int prof_begin(const char* tag, cudaStream_t s);
void prof_end(int idx, cudaStream_t s);

// cudaFuncSetAttribute acts on the current device only, so a kernel's raised
// dynamic shared-memory limit is applied once per device: `done` holds one
// bit per device index (devices beyond 63 set it on every call).
int smem_limit_once(const void* kernel, int bytes, uint64_t& done);

}  // namespace qsgw

#define QSGW_CUDA(call)                                                   \
  do {                                                                    \
    int _rc = ::qsgw::check_cuda((call), #call);                          \
    if (_rc != 0) return _rc;                                             \
  } while (0)

#define QSGW_LAUNCH_CHECK(what)                                           \
  do {                                                                    \
    int _rc = ::qsgw::check_cuda(cudaGetLastError(), what);               \
    if (_rc != 0) return _rc;                                             \
  } while (0)

#define QSGW_ARG(cond, ...)                                               \
  do {                                                                    \
    if (!(cond)) {                                                        \
      ::qsgw::set_error(__VA_ARGS__);                                     \
      return QSGW_ERR_ARG;                                                \
    }                                                                     \
  } while (0)
