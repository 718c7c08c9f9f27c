// Library context: device selection, launch stream, precision switch and
// error text.  Replaces gpu_init (m_gpu.f90:14-68) and the cuBLAS/cuSOLVER
// handle set-up/teardown (m_lapack.f90:230-255) of the reference.
#include <cstdarg>
#include <atomic>
#include "common.cuh"
#include "hoststage.cuh"

namespace qsgw {

static Context g_ctx;
static char g_err[1024] = "";
static std::atomic<long long> g_launches{0};

Context& ctx() { return g_ctx; }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

void count_launch(int n) { g_launches += n; }

int smem_limit_once(const void* kernel, int bytes, uint64_t& done) {
  int dev = 0;
  QSGW_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t{1} << dev) : 0;
  if (bit && (done & bit)) return QSGW_OK;
  QSGW_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done |= bit;
  return QSGW_OK;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return QSGW_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? QSGW_ERR_OOM : QSGW_ERR_CUDA;
}

int DevBuf::ensure(size_t n) {
  if (n <= bytes && p) return QSGW_OK;
  if (g_ctx.capturing) {
    // nodes recorded earlier may point into the old buffer
    set_error("scratch of %zu bytes needed while recording a graph: run the same calls once before "
              "qsgw_graph_begin", n);
    return QSGW_ERR_UNSUPPORTED;
  }
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  size_t want = n < 256 ? 256 : n;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    return check_cuda(e, "cudaMalloc(scratch)");
  }
  bytes = want;
  return QSGW_OK;
}

int h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return QSGW_OK;
  if (!g_ctx.capturing) {
    if (host_async()) return async_table_h2d(dst, src, bytes, s);
    return check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "H2D table");
  }
  void* pin = nullptr;
  int rc = check_cuda(cudaHostAlloc(&pin, bytes, cudaHostAllocDefault), "cudaHostAlloc(graph table)");
  if (rc) return rc;
  std::memcpy(pin, src, bytes);
  g_ctx.graph_host.push_back(pin);
  return check_cuda(cudaMemcpyAsync(dst, pin, bytes, cudaMemcpyHostToDevice, s), "H2D table (graph)");
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

struct ProfRec {
  std::string tag;
  cudaEvent_t a, b;
};
static bool g_prof = false;
static std::vector<ProfRec> g_prof_recs;
static std::vector<cudaEvent_t> g_event_pool;

static cudaEvent_t pool_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

static void prof_reset() {
  for (auto& r : g_prof_recs) {
    g_event_pool.push_back(r.a);
    g_event_pool.push_back(r.b);
  }
  g_prof_recs.clear();
}

// While a graph is recorded the events become external event-record nodes:
// each replay records them again, so the times read afterwards are those of
// the latest replay.
static void prof_record(cudaEvent_t e, cudaStream_t s) {
  if (g_ctx.capturing) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
  else cudaEventRecord(e, s);
}

int prof_begin(const char* tag, cudaStream_t s) {
  if (!g_prof) return -1;
  ProfRec r{tag, pool_event(), pool_event()};
  prof_record(r.a, s);
  g_prof_recs.push_back(r);
  return static_cast<int>(g_prof_recs.size()) - 1;
}

void prof_end(int idx, cudaStream_t s) {
  if (idx < 0 || idx >= static_cast<int>(g_prof_recs.size())) return;
  prof_record(g_prof_recs[idx].b, s);
}

int require_init() {
  if (!g_ctx.initialized) {
    set_error("qsgw_init has not been called");
    return QSGW_ERR_NOTINIT;
  }
  cudaError_t e = cudaSetDevice(g_ctx.device);
  return check_cuda(e, "cudaSetDevice");
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_init(int device) {
  Context& c = ctx();
  if (c.initialized) {
    if (c.device == device) return QSGW_OK;
    set_error("qsgw_init: already initialised on device %d", c.device);
    return QSGW_ERR_ARG;
  }
  int ndev = 0;
  QSGW_CUDA(cudaGetDeviceCount(&ndev));
  QSGW_ARG(device >= 0 && device < ndev, "qsgw_init: device %d out of range (%d devices)", device, ndev);
  QSGW_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  QSGW_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("qsgw_init: device %d is sm_%d%d; this library is built for sm_100a only",
              device, prop.major, prop.minor);
    return QSGW_ERR_UNSUPPORTED;
  }
  c.sm_count = prop.multiProcessorCount;
  QSGW_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  c.own_stream = true;
  QSGW_CUDA(cudaMalloc(&c.d_flags, 64 * sizeof(int)));
  QSGW_CUDA(cudaMemset(c.d_flags, 0, 64 * sizeof(int)));
  c.device = device;
  c.initialized = true;
  g_launches = 0;
  return QSGW_OK;
}

static void graph_free();

extern "C" int qsgw_finalize(void) {
  Context& c = ctx();
  if (!c.initialized) return QSGW_OK;
  cudaSetDevice(c.device);
  if (c.capturing) {                       // abandon an unfinished recording
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(c.stream, &g);
    if (g) cudaGraphDestroy(g);
    c.capturing = false;
  }
  cudaDeviceSynchronize();
  graph_free();
  host_stage_release();
  if (c.d_flags) cudaFree(c.d_flags);
  if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
  c = Context();
  return QSGW_OK;
}

extern "C" int qsgw_set_stream(void* stream) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(!ctx().capturing, "set_stream: a graph is being recorded");
  Context& c = ctx();
  if (stream == nullptr) {
    if (!c.own_stream) {
      QSGW_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
      c.own_stream = true;
    }
    return QSGW_OK;
  }
  if (c.own_stream && c.stream) {
    QSGW_CUDA(cudaStreamSynchronize(c.stream));
    cudaStreamDestroy(c.stream);
  }
  c.stream = reinterpret_cast<cudaStream_t>(stream);
  c.own_stream = false;
  return QSGW_OK;
}

extern "C" int qsgw_synchronize(void) {
  int rc = require_init();
  if (rc) return rc;
  Context& c = ctx();
  QSGW_CUDA(cudaStreamSynchronize(c.stream));
  rc = host_stage_sync();
  if (rc) return rc;
  int flag[2] = {0, 0};
  QSGW_CUDA(cudaMemcpy(flag, c.d_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost));
  if (flag[0]) {
    QSGW_CUDA(cudaMemset(c.d_flags, 0, sizeof(int)));
    set_error("a pivot block of the Hermitian inverse was singular or not finite");
    return QSGW_ERR_NUMERIC;
  }
  if (flag[1]) {   // a tensor-core kernel gave up a bounded wait and skipped its output
    QSGW_CUDA(cudaMemset(c.d_flags + 1, 0, sizeof(int)));
    set_error("a split-precision kernel timed out waiting for its pipeline; its output is incomplete");
    return QSGW_ERR_TIMEOUT;
  }
  return QSGW_OK;
}

extern "C" int qsgw_set_precision(int mode, int nslices) {
  QSGW_ARG(mode == QSGW_PREC_FP64 || mode == QSGW_PREC_SPLIT_F16 || mode == QSGW_PREC_SPLIT_I8,
           "qsgw_set_precision: unknown mode %d", mode);
  QSGW_ARG(mode != QSGW_PREC_SPLIT_F16 || nslices == 2,
           "qsgw_set_precision: SPLIT_F16 is built for 2 slices per operand (got %d)", nslices);
  QSGW_ARG(mode != QSGW_PREC_SPLIT_I8 || nslices == 0 || (nslices >= 2 && nslices <= 4),
           "qsgw_set_precision: SPLIT_I8 takes 2, 3 or 4 slices per operand, or 0 for automatic (got %d)",
           nslices);
  ctx().prec_mode = mode;
  ctx().nslices = (mode == QSGW_PREC_FP64) ? 1 : nslices;
  return QSGW_OK;
}

extern "C" int qsgw_set_accuracy(double sigc_qp_tol_ha, double chi0_rel_tol) {
  QSGW_ARG(sigc_qp_tol_ha > 0.0 && chi0_rel_tol > 0.0, "qsgw_set_accuracy: targets must be positive (%g, %g)",
           sigc_qp_tol_ha, chi0_rel_tol);
  ctx().sigc_qp_tol = sigc_qp_tol_ha;
  ctx().chi0_rel_tol = chi0_rel_tol;
  return QSGW_OK;
}

extern "C" int qsgw_get_precision(int* mode, int* nslices) {
  QSGW_ARG(mode && nslices, "qsgw_get_precision: null pointer");
  *mode = ctx().prec_mode;
  *nslices = ctx().nslices;
  return QSGW_OK;
}

extern "C" int qsgw_last_error(char* buf, int len) {
  if (!buf || len <= 0) return QSGW_ERR_ARG;
  strncpy(buf, g_err, static_cast<size_t>(len) - 1);
  buf[len - 1] = '\0';
  return QSGW_OK;
}

extern "C" long long qsgw_launch_count(void) { return g_launches.load(); }

extern "C" int qsgw_profile(int enable) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(!ctx().capturing, "qsgw_profile: a graph is being recorded");
  QSGW_CUDA(cudaStreamSynchronize(ctx().stream));
  prof_reset();
  g_prof = enable != 0;
  return QSGW_OK;
}

extern "C" int qsgw_profile_get(const char* tag, double* ms, long long* launches) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(tag && ms && launches, "qsgw_profile_get: null pointer");
  QSGW_CUDA(cudaStreamSynchronize(ctx().stream));
  double tot = 0.0;
  long long n = 0;
  for (auto& r : g_prof_recs) {
    if (r.tag != tag) continue;
    float t = 0.f;
    QSGW_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    tot += t;
    ++n;
  }
  *ms = tot;
  *launches = n;
  return QSGW_OK;
}


// ---- CUDA graph of a recorded call sequence
static void graph_free() {
  Context& c = ctx();
  if (c.graph_exec) cudaGraphExecDestroy(c.graph_exec);
  if (c.graph) cudaGraphDestroy(c.graph);
  c.graph_exec = nullptr;
  c.graph = nullptr;
  for (void* p : c.graph_host) cudaFreeHost(p);
  c.graph_host.clear();
}

extern "C" int qsgw_graph_begin(void) {
  int rc = require_init();
  if (rc) return rc;
  Context& c = ctx();
  QSGW_ARG(!c.capturing, "graph_begin: already recording");
  QSGW_ARG(c.stream != nullptr, "graph_begin: the launch stream cannot be the legacy default stream");
  QSGW_CUDA(cudaStreamSynchronize(c.stream));
  graph_free();
  // relaxed: pinned host tables are allocated while recording
  QSGW_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
  c.capturing = true;
  return QSGW_OK;
}

extern "C" int qsgw_graph_end(void) {
  int rc = require_init();
  if (rc) return rc;
  Context& c = ctx();
  QSGW_ARG(c.capturing, "graph_end: not recording");
  c.capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c.stream, &g);
  if (e != cudaSuccess || g == nullptr) {
    if (g) cudaGraphDestroy(g);
    graph_free();
    return check_cuda(e != cudaSuccess ? e : cudaErrorStreamCaptureInvalidated, "graph_end: cudaStreamEndCapture");
  }
  c.graph = g;
  rc = check_cuda(cudaGraphInstantiate(&c.graph_exec, g, 0), "graph_end: cudaGraphInstantiate");
  if (rc) graph_free();
  return rc;
}

extern "C" int qsgw_graph_launch(void) {
  int rc = require_init();
  if (rc) return rc;
  Context& c = ctx();
  QSGW_ARG(c.graph_exec && !c.capturing, "graph_launch: no recorded graph");
  QSGW_CUDA(cudaGraphLaunch(c.graph_exec, c.stream));
  return QSGW_OK;
}

extern "C" int qsgw_graph_destroy(void) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(!ctx().capturing, "graph_destroy: still recording");
  QSGW_CUDA(cudaStreamSynchronize(ctx().stream));
  graph_free();
  return QSGW_OK;
}
