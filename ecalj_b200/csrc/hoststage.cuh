// Staging of the host-pointer entry points' inputs (qsgw_chi0_lorentz,
// qsgw_sxcf_correlation).  Their inputs travel on a copy stream into a ring
// of slots of device buffers; the compute stream waits for the slot's copy,
// and the copy into a slot waits for the computation that last read it.  In
// the asynchronous mode (qsgw_set_host_async(1)) the calls return once their
// work is enqueued, so the copies of the next calls overlap the computation
// of the current one (as many calls ahead as the ring has slots); outputs are
// valid after qsgw_synchronize().
#pragma once
#include "common.cuh"

namespace qsgw {

struct HostSlot {
  DevBuf buf[3];
  cudaEvent_t ready = nullptr;   // recorded on the copy stream after the slot's copies
  cudaEvent_t freed = nullptr;   // recorded on the compute stream after the slot's last reader
  bool used = false;
};

struct HostRing {
  static constexpr int MAXSLOT = 16;
  explicit HostRing(int n) : nslot(n) {}
  HostSlot slot[MAXSLOT];
  int nslot;                     // slots of the asynchronous mode (<= MAXSLOT; synchronous: 2)
  int next = 0;
  // Picks the next slot; *cs = the copy stream, ordered after the slot's last reader.
  int begin(HostSlot** sl, cudaStream_t* cs);
  // The copies into the slot are enqueued: the compute stream waits for them.
  int ready(HostSlot& sl, cudaStream_t cs);
  // The computation reading the slot is enqueued; synchronous mode: wait for it all.
  int finish(HostSlot& sl);
};

bool host_async();
// Device image of a host accumulation array (Sigma_c's zsec) in the
// asynchronous mode: copied from the host at its first use after a
// synchronisation, accumulated into by every later call with the same array,
// and copied back by each call.  Released by qsgw_synchronize().
int host_acc_target(void* host, size_t bytes, cudaStream_t s, void** dev);
// qsgw_synchronize / qsgw_finalize: wait for the copy stream, forget the accumulation images.
int host_stage_sync();
void host_stage_release();
// Host tables of the asynchronous mode (h2d): copied into a pinned arena of
// sections, one per host-pointer call in turn, so that no copy from pageable
// memory makes the host wait for the compute stream, then to a device image
// of the section on the copy stream and into place by a kernel on the
// compute stream.  A section is reused once the compute stream has passed the
// call that last used it.
int async_table_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);

}  // namespace qsgw
