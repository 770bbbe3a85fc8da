// Ray-batch kernels: closest hit and any hit over caller-supplied rays.  These
// back pfxt_trace_rays / pfxt_occluded (the parity entry on identical ray
// batches) and the traversal benchmark.
//
// Persistent warps with per-lane refill: the grid fills the GPU once (SM count
// x resident blocks), and whenever lanes of a warp finish their query they
// take the next ray indices from one atomic counter (one atomic per warp per
// refill).  A warp therefore keeps its lanes busy instead of idling behind its
// slowest ray, which is what limits a one-ray-per-thread launch on incoherent
// batches.  Inside a lane the walk alternates an inner-node phase and a leaf
// phase (the "while-while" loop), so lanes of a warp tend to run the same
// phase together.
#include <cuda_runtime.h>

#include <atomic>

#include "kernels.h"
#include "traverse.cuh"

namespace pfxt {

namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ void load_ray(const pfxt_ray* __restrict__ rays, uint32_t i, v3& o, v3& d, float& tmax) {
  const float4* p = reinterpret_cast<const float4*>(rays + i);
  float4 a = __ldg(p), b = __ldg(p + 1);
  o = mk3(a.x, a.y, a.z);
  tmax = a.w;
  d = mk3(b.x, b.y, b.z);
}

// The output word that marks a ray the first walk handed over to the IEEE
// walk (closest hit: the `hit` field; any hit: the flag).
constexpr uint32_t RETRY = 2u;

// MODE 0: closest hit -> pfxt_hit; MODE 1: any hit -> u32 flag;
// MODE 2/3: work counters of closest / any hit -> uint2.  Modes 0 and 1 walk
// bounded rays only (no call in the walk loop) and mark the others RETRY for
// k_trace_retry; the counting modes walk every ray.
template <int MODE>
__global__ void __launch_bounds__(kThreads, TRACE_WARPS_PER_SM * 32 / kThreads) k_trace(SceneView s, const pfxt_ray* __restrict__ rays, uint32_t n,
                                                    void* __restrict__ out, uint32_t* __restrict__ counter) {
  constexpr bool ANY = (MODE == 1 || MODE == 3);
  constexpr bool COUNT = (MODE >= 2);
  constexpr unsigned FULL = 0xffffffffu;
  LaneStack<0> st;  // local memory: a shared-memory top measured slower (more registers, fewer warps)
  Walker<ANY, COUNT, COUNT ? BOX_EITHER : TRACE_BOX, !COUNT && TRACE_SPEC> w;
  const int lane = threadIdx.x & 31;
  uint32_t idx = 0;
  bool have = false, retired = false;
  for (;;) {
    bool need = !have && !retired;
    unsigned m = __ballot_sync(FULL, need);
    if (m) {
      int leader = __ffs(m) - 1;
      uint32_t first = 0;
      if (lane == leader) first = atomicAdd(counter, (uint32_t)__popc(m));
      first = __shfl_sync(FULL, first, leader);
      if (need) {
        idx = first + (uint32_t)__popc(m & ((1u << lane) - 1u));
        if (idx < n) {
          v3 o, d;
          float tmax;
          load_ray(rays, idx, o, d, tmax);
          w.start(s, o, d, tmax);
          have = true;
        } else {
          retired = true;
        }
      }
    }
    if (__all_sync(FULL, retired)) break;
    if (have) {
      w.inner_phase(s, st, [&](v3& o, v3& d) {
        float tmax;
        load_ray(rays, idx, o, d, tmax);
      });
      if (w.leaf_ready()) w.leaf_phase(s, st);
      if (!w.leaf_ready()) {
        if (MODE == 0) {
          reinterpret_cast<uint4*>(out)[idx] =
              make_uint4(__float_as_uint(w.hit.t), w.hit.slot, w.hit.record, w.retry ? RETRY : w.hit.hit);
        } else if (MODE == 1) {
          reinterpret_cast<uint32_t*>(out)[idx] = w.retry ? RETRY : w.hit.hit;
        } else {
          reinterpret_cast<uint2*>(out)[idx] = make_uint2(w.counts.boxes, w.counts.tris);
        }
        have = false;
      }
    }
  }
}

// The rays k_trace marked RETRY, walked again from the start with IEEE
// division throughout (rare: a direction component above 2^20 or an origin
// component beyond the bounded range, in world or instance space).
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_trace_retry(SceneView s, const pfxt_ray* __restrict__ rays, uint32_t n,
                                                          void* __restrict__ out) {
  constexpr bool ANY = (MODE == 1);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t marker = MODE == 0 ? reinterpret_cast<const uint4*>(out)[i].w : reinterpret_cast<const uint32_t*>(out)[i];
    if (marker != RETRY) continue;
    LaneStack<0> st;
    Walker<ANY, false, BOX_IEEE> w;
    v3 o, d;
    float tmax;
    load_ray(rays, i, o, d, tmax);
    w.start(s, o, d, tmax);
    w.run(s, st, [&](v3& wo, v3& wd) {
      wo = o;
      wd = d;
    });
    if (MODE == 0)
      reinterpret_cast<uint4*>(out)[i] = make_uint4(__float_as_uint(w.hit.t), w.hit.slot, w.hit.record, w.hit.hit);
    else
      reinterpret_cast<uint32_t*>(out)[i] = w.hit.hit;
  }
}

// Narrow 32-bit flags to bytes (separate input and output regions).
__global__ void k_pack(const uint32_t* __restrict__ in, uint8_t* __restrict__ out, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] ? 1 : 0;
}

constexpr int kMaxDevices = 64;

// Blocks of a persistent launch on the current device (SM count x resident
// blocks), computed once per device.  Threads that race on a device's first
// launch compute the same number, so the relaxed store is enough.
template <int MODE>
int persistent_blocks() {
  static std::atomic<int> cached[kMaxDevices];
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<int>* slot = (dev >= 0 && dev < kMaxDevices) ? &cached[dev] : nullptr;
  int blocks = slot ? slot->load(std::memory_order_relaxed) : 0;
  if (blocks == 0) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<MODE>, kThreads, 0);
    blocks = (sms > 0 ? sms : 1) * (per > 0 ? per : 1);
    if (slot) slot->store(blocks, std::memory_order_relaxed);
  }
  return blocks;
}

template <int MODE>
cudaError_t launch(const SceneView& s, const pfxt_ray* rays, uint32_t n, void* out, uint32_t* counter,
                   cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  uint32_t need = (n + kThreads - 1) / kThreads;
  uint32_t blocks = (uint32_t)persistent_blocks<MODE>();
  if (need < blocks) blocks = need;
  k_trace<MODE><<<blocks, kThreads, 0, stream>>>(s, rays, n, out, counter);
  if constexpr (MODE < 2) {
    uint32_t scan = (n + kThreads - 1) / kThreads, most = (uint32_t)persistent_blocks<MODE>();
    k_trace_retry<MODE><<<scan < most ? scan : most, kThreads, 0, stream>>>(s, rays, n, out);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_closest(const SceneView& s, const pfxt_ray* rays, uint32_t n, pfxt_hit* hits, uint32_t* counter,
                           cudaStream_t stream) {
  return launch<0>(s, rays, n, hits, counter, stream);
}

cudaError_t launch_any(const SceneView& s, const pfxt_ray* rays, uint32_t n, uint32_t* blocked, uint32_t* counter,
                       cudaStream_t stream) {
  return launch<1>(s, rays, n, blocked, counter, stream);
}

cudaError_t launch_counts(const SceneView& s, const pfxt_ray* rays, uint32_t n, bool any, uint2* counts,
                          uint32_t* counter, cudaStream_t stream) {
  return any ? launch<3>(s, rays, n, counts, counter, stream) : launch<2>(s, rays, n, counts, counter, stream);
}

cudaError_t prepare_any_queries() {
  persistent_blocks<1>();
  cudaFuncAttributes attr;
  cudaError_t e = cudaFuncGetAttributes(&attr, k_trace<1>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&attr, k_trace_retry<1>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&attr, k_pack);
  return e;
}

cudaError_t launch_pack_flags(const uint32_t* flags, uint8_t* bytes, uint32_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_pack<<<(n + 255u) / 256u, 256, 0, stream>>>(flags, bytes, n);
  return cudaGetLastError();
}

}  // namespace pfxt
