// Any-hit queries for callers that cannot allocate device memory.
//
// pfxt_occluded_device needs two pieces of scratch beyond its inputs and
// outputs: the work-sharing counter of the persistent traversal kernel and,
// when the caller wants one byte per ray, the 32-bit flag words the kernel
// writes before they are narrowed.  This variant keeps both in file-scope
// __device__ arrays instead of memory owned by the handle or allocated per
// call, so the call itself never allocates.  It is meant for hosts that hand
// all device memory to their own allocator (an engine that reserves its heap up
// front, a process whose caching allocator owns the free memory) and for code
// that must not allocate while other GPU work is in flight.
//
// Limits and rules:
//   * at most PFXT_NOALLOC_MAX_RAYS rays per call (4 MiB of flag words, held
//     by every GPU that loads the library until the process exits);
//   * every call shares the arrays, so calls whose GPU work overlaps (two
//     streams, two threads) race; the counter is cleared on the stream at the
//     start of each call, the flag words are fully rewritten for the rays of
//     the call;
//   * pfxt_create resolves the arrays' device addresses and loads the
//     kernels this entry point launches, with the handle's device current.
//     CUDA loads modules lazily, and loading this file's module is what
//     places the arrays in device memory, so after pfxt_create a call loads
//     nothing and allocates nothing.  A call on a device no handle was created
//     on does that set-up itself; make such a first call before any stream
//     capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kernels.h"
#include "pfxt.h"
#include "pfxt_internal.h"
#include "tracer.h"

static __device__ __align__(256) uint32_t g_noalloc_flags[PFXT_NOALLOC_MAX_RAYS];
static __device__ __align__(256) uint32_t g_noalloc_counter[64];

namespace {

constexpr int kMaxDevices = 64;

struct Resolved {
  uint32_t* flags = nullptr;
  uint32_t* counter = nullptr;
};

std::mutex g_lock;
Resolved g_resolved[kMaxDevices];

// Device addresses of the arrays for `device` (which must be current).  In
// host code the arrays' names are host-side stand-ins, never device pointers.
cudaError_t resolve(int device, Resolved* out) {
  std::lock_guard<std::mutex> hold(g_lock);
  Resolved& r = g_resolved[device];
  if (!r.flags) {
    void* flags = nullptr;
    void* counter = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&flags, g_noalloc_flags);
    if (e != cudaSuccess) return e;
    e = cudaGetSymbolAddress(&counter, g_noalloc_counter);
    if (e != cudaSuccess) return e;
    r.flags = static_cast<uint32_t*>(flags);
    r.counter = static_cast<uint32_t*>(counter);
  }
  *out = r;
  return cudaSuccess;
}

}  // namespace

namespace pfxt {

cudaError_t noalloc_prepare(int device) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  Resolved r;
  cudaError_t e = resolve(device, &r);
  if (e == cudaSuccess) e = prepare_any_queries();
  return e;
}

}  // namespace pfxt

extern "C" int pfxt_occluded_noalloc(pfxt_trace* t, const pfxt_ray* rays, uint32_t count, uint8_t* blocked,
                                     void* stream) {
  using namespace pfxt;
  if (!t || (count && (!rays || !blocked))) {
    set_error("null argument");
    return PFXT_ERR_INVALID;
  }
  if (count > PFXT_NOALLOC_MAX_RAYS) {
    set_error("pfxt_occluded_noalloc takes at most " + std::to_string(PFXT_NOALLOC_MAX_RAYS) + " rays per call, got " +
              std::to_string(count));
    return PFXT_ERR_INVALID;
  }
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess || device != t->device || device < 0 || device >= kMaxDevices) {
    cudaGetLastError();
    set_error("pfxt_occluded_noalloc must be called with the handle's device current");
    return PFXT_ERR_INVALID;
  }
  Resolved r;
  cudaError_t e = resolve(device, &r);
  if (e == cudaSuccess && count) e = launch_any(t->view, rays, count, r.flags, r.counter, (cudaStream_t)stream);
  if (e == cudaSuccess && count) e = launch_pack_flags(r.flags, blocked, count, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("pfxt_occluded_noalloc: ") + cudaGetErrorString(e));
    return PFXT_ERR_CUDA;
  }
  set_error("");
  return PFXT_OK;
}
