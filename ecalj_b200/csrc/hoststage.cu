// Host-pointer staging and the asynchronous host mode (see hoststage.cuh).
#include <algorithm>
#include <cstring>
#include <vector>
#include "hoststage.cuh"

namespace qsgw {

static bool g_async = false;
static cudaStream_t g_copy = nullptr;

struct AccImage {
  const void* host = nullptr;      // nullptr: free entry
  size_t bytes = 0;
  DevBuf dev;
};
static std::vector<AccImage*> g_acc;
static std::vector<HostRing*> g_rings;

static int copy_stream(cudaStream_t* cs) {
  if (!g_copy) QSGW_CUDA(cudaStreamCreateWithFlags(&g_copy, cudaStreamNonBlocking));
  *cs = g_copy;
  return QSGW_OK;
}

// pinned arena of the asynchronous mode's host tables (NSEC sections, one per call in turn)
constexpr size_t ARENA_SECTION = size_t(16) << 20;     // bytes of one section
constexpr int NSEC = 16;
static char* g_arena = nullptr;
static DevBuf g_darena;                    // device image of the arena: tables land here first
static size_t g_sec_off[NSEC] = {};
static int g_sec = 0;                     // section of the current call
static cudaEvent_t g_sec_done[NSEC] = {};
static bool g_sec_used[NSEC] = {};

// Host -> device copy ordered for the asynchronous mode: on the copy stream, after the compute
// stream's work so far (the destination may still be read there) and ahead of the next call's
// inputs; the compute stream waits for it.  On the compute stream itself such a copy would queue
// in the host -> device engine behind the next call's inputs, which are enqueued meanwhile, and
// the computation waiting for it would no longer overlap them.
// after_compute: the destination may still be read by the compute stream's earlier work.
static cudaEvent_t g_ord[2] = {nullptr, nullptr};
static int ordered_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s, bool after_compute) {
  cudaStream_t cs = nullptr;
  int rc = copy_stream(&cs);
  if (rc) return rc;
  if (!g_ord[0])
    for (auto& e : g_ord) QSGW_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (after_compute) {
    QSGW_CUDA(cudaEventRecord(g_ord[0], s));
    QSGW_CUDA(cudaStreamWaitEvent(cs, g_ord[0], 0));
  }
  QSGW_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs));
  QSGW_CUDA(cudaEventRecord(g_ord[1], cs));
  QSGW_CUDA(cudaStreamWaitEvent(s, g_ord[1], 0));
  return QSGW_OK;
}

// device -> device copy of a staged table on the compute stream (SM threads, not a DMA engine,
// so it never queues behind the host -> device copies)
__global__ void table_copy_kernel(unsigned char* __restrict__ dst, const unsigned char* __restrict__ src, size_t n) {
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 7) == 0) {
    const size_t nw = n >> 3;
    for (size_t w = i; w < nw; w += stride)
      reinterpret_cast<unsigned long long*>(dst)[w] = reinterpret_cast<const unsigned long long*>(src)[w];
    for (size_t b = (nw << 3) + i; b < n; b += stride) dst[b] = src[b];
  } else {
    for (size_t b = i; b < n; b += stride) dst[b] = src[b];
  }
}

// a new host-pointer call: close the current section, open the next once the GPU is past it
static int arena_next_call() {
  if (!g_arena) return QSGW_OK;
  QSGW_CUDA(cudaEventRecord(g_sec_done[g_sec], ctx().stream));
  g_sec_used[g_sec] = true;
  g_sec = (g_sec + 1) % NSEC;
  if (g_sec_used[g_sec]) QSGW_CUDA(cudaEventSynchronize(g_sec_done[g_sec]));
  g_sec_off[g_sec] = 0;
  return QSGW_OK;
}

int async_table_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (!g_arena) {
    int rc = g_darena.ensure(NSEC * ARENA_SECTION);
    if (rc) return rc;
    QSGW_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&g_arena), NSEC * ARENA_SECTION, cudaHostAllocDefault));
    for (auto& e : g_sec_done) QSGW_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (bytes > ARENA_SECTION)                  // larger than a section: copied from the caller's memory
    return ordered_h2d(dst, src, bytes, s, true);
  size_t& off = g_sec_off[g_sec];
  if (off + bytes > ARENA_SECTION) {          // this call's section is full: let the GPU catch up
    QSGW_CUDA(cudaStreamSynchronize(s));
    off = 0;
  }
  const size_t at = static_cast<size_t>(g_sec) * ARENA_SECTION + off;
  std::memcpy(g_arena + at, src, bytes);
  off += (bytes + 255) & ~size_t(255);
  // pinned section -> device section on the copy stream (no reader of this section is left:
  // the host waited for the call that last used it), then into place on the compute stream
  unsigned char* dstage = g_darena.as<unsigned char>() + at;
  int rc = ordered_h2d(dstage, g_arena + at, bytes, s, false);
  if (rc) return rc;
  const int blocks = static_cast<int>(std::min<size_t>((bytes / 8 + 255) / 256 + 1, 1024));
  table_copy_kernel<<<blocks, 256, 0, s>>>(static_cast<unsigned char*>(dst), dstage, bytes);
  count_launch();
  QSGW_LAUNCH_CHECK("table_copy_kernel");
  return QSGW_OK;
}

bool host_async() { return g_async; }


int HostRing::begin(HostSlot** out, cudaStream_t* cs) {
  QSGW_ARG(!ctx().capturing, "host-pointer entry points cannot be recorded in a graph (use the _d entry points)");
  if (!slot[0].ready) {
    for (int i = 0; i < nslot; ++i) {
      HostSlot& sl = slot[i];
      QSGW_CUDA(cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming));
      QSGW_CUDA(cudaEventCreateWithFlags(&sl.freed, cudaEventDisableTiming));
    }
    g_rings.push_back(this);
  }
  const int n = g_async ? nslot : std::min(nslot, 2);     // synchronous calls need two slots
  if (next >= n) next = 0;
  HostSlot& sl = slot[next];
  next = (next + 1) % n;
  int rc = copy_stream(cs);
  if (rc) return rc;
  if (g_async && (rc = arena_next_call())) return rc;
  if (sl.used) QSGW_CUDA(cudaStreamWaitEvent(*cs, sl.freed, 0));
  *out = &sl;
  return QSGW_OK;
}

int HostRing::ready(HostSlot& sl, cudaStream_t cs) {
  QSGW_CUDA(cudaEventRecord(sl.ready, cs));
  QSGW_CUDA(cudaStreamWaitEvent(ctx().stream, sl.ready, 0));
  return QSGW_OK;
}

int HostRing::finish(HostSlot& sl) {
  QSGW_CUDA(cudaEventRecord(sl.freed, ctx().stream));
  sl.used = true;
  if (!g_async) QSGW_CUDA(cudaStreamSynchronize(ctx().stream));
  return QSGW_OK;
}

int host_acc_target(void* host, size_t bytes, cudaStream_t s, void** dev) {
  AccImage* img = nullptr;
  for (AccImage* a : g_acc) {
    if (a->host == host) {
      QSGW_ARG(a->bytes == bytes, "accumulation array %p used with %zu and %zu bytes before a synchronisation",
               host, a->bytes, bytes);
      *dev = a->dev.p;
      return QSGW_OK;
    }
    if (!img && a->host == nullptr) img = a;
  }
  if (!img) {
    img = new AccImage();
    g_acc.push_back(img);
  }
  int rc = img->dev.ensure(bytes);
  if (rc) return rc;
  img->host = host;
  img->bytes = bytes;
  *dev = img->dev.p;
  return ordered_h2d(img->dev.p, host, bytes, s, false);   // a new image has no reader yet
}

int host_stage_sync() {
  if (g_copy) QSGW_CUDA(cudaStreamSynchronize(g_copy));
  for (AccImage* a : g_acc) a->host = nullptr;
  return QSGW_OK;
}

void host_stage_release() {
  for (AccImage* a : g_acc) {
    a->dev.release();
    delete a;
  }
  g_acc.clear();
  for (HostRing* r : g_rings) {
    for (auto& sl : r->slot) {
      for (auto& b : sl.buf) b.release();
      if (sl.ready) cudaEventDestroy(sl.ready);
      if (sl.freed) cudaEventDestroy(sl.freed);
      sl = HostSlot();
    }
    r->next = 0;
  }
  g_rings.clear();
  if (g_arena) cudaFreeHost(g_arena);
  g_arena = nullptr;
  g_darena.release();
  for (int h = 0; h < NSEC; ++h) {
    if (g_sec_done[h]) cudaEventDestroy(g_sec_done[h]);
    g_sec_done[h] = nullptr;
    g_sec_used[h] = false;
    g_sec_off[h] = 0;
  }
  g_sec = 0;
  for (auto& e : g_ord) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  if (g_copy) cudaStreamDestroy(g_copy);
  g_copy = nullptr;
  g_async = false;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_set_host_async(int on) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(on == 0 || on == 1, "qsgw_set_host_async: %d (0 or 1)", on);
  if (!on && g_async) {                    // leaving the mode: finish what it enqueued
    QSGW_CUDA(cudaStreamSynchronize(ctx().stream));
    rc = host_stage_sync();
    if (rc) return rc;
  }
  g_async = on == 1;
  return QSGW_OK;
}
