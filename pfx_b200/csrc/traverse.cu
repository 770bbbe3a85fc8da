// Ray-batch kernels: closest hit and any hit over caller-supplied rays.  These
// back pfxt_trace_rays / pfxt_occluded (the parity entry on identical ray
// batches) and the traversal benchmark.
#include <cuda_runtime.h>

#include "kernels.h"
#include "traverse.cuh"

namespace pfxt {

namespace {

__device__ __forceinline__ void load_ray(const pfxt_ray* __restrict__ rays, uint32_t i, v3& o, v3& d, float& tmax) {
  const float4* p = reinterpret_cast<const float4*>(rays + i);
  float4 a = __ldg(p), b = __ldg(p + 1);
  o = mk3(a.x, a.y, a.z);
  tmax = a.w;
  d = mk3(b.x, b.y, b.z);
}

__global__ void __launch_bounds__(128) k_closest(SceneView s, const pfxt_ray* __restrict__ rays, uint32_t n,
                                                 pfxt_hit* __restrict__ hits) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  v3 o, d;
  float tmax;
  load_ray(rays, i, o, d, tmax);
  TraceHit h = traverse<false, false>(s, o, d, tmax, nullptr);
  reinterpret_cast<uint4*>(hits)[i] = make_uint4(__float_as_uint(h.t), h.slot, h.record, h.hit);
}

__global__ void __launch_bounds__(128) k_any(SceneView s, const pfxt_ray* __restrict__ rays, uint32_t n,
                                             uint32_t* __restrict__ blocked) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  v3 o, d;
  float tmax;
  load_ray(rays, i, o, d, tmax);
  TraceHit h = traverse<true, false>(s, o, d, tmax, nullptr);
  blocked[i] = h.hit;
}

__global__ void __launch_bounds__(128) k_counts(SceneView s, const pfxt_ray* __restrict__ rays, uint32_t n,
                                                uint32_t any, uint2* __restrict__ counts) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  v3 o, d;
  float tmax;
  load_ray(rays, i, o, d, tmax);
  TraceCounts c{0u, 0u};
  if (any)
    traverse<true, true>(s, o, d, tmax, &c);
  else
    traverse<false, true>(s, o, d, tmax, &c);
  counts[i] = make_uint2(c.boxes, c.tris);
}

// Narrow 32-bit flags to bytes (separate input and output regions).
__global__ void k_pack(const uint32_t* __restrict__ in, uint8_t* __restrict__ out, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] ? 1 : 0;
}

}  // namespace

cudaError_t launch_closest(const SceneView& s, const pfxt_ray* rays, uint32_t n, pfxt_hit* hits, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  uint32_t blocks = (n + 127u) / 128u;
  k_closest<<<blocks, 128, 0, stream>>>(s, rays, n, hits);
  return cudaGetLastError();
}

cudaError_t launch_any(const SceneView& s, const pfxt_ray* rays, uint32_t n, uint32_t* blocked, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  uint32_t blocks = (n + 127u) / 128u;
  k_any<<<blocks, 128, 0, stream>>>(s, rays, n, blocked);
  return cudaGetLastError();
}

cudaError_t launch_pack_flags(const uint32_t* flags, uint8_t* bytes, uint32_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_pack<<<(n + 255u) / 256u, 256, 0, stream>>>(flags, bytes, n);
  return cudaGetLastError();
}

cudaError_t launch_counts(const SceneView& s, const pfxt_ray* rays, uint32_t n, bool any, uint2* counts,
                          cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  uint32_t blocks = (n + 127u) / 128u;
  k_counts<<<blocks, 128, 0, stream>>>(s, rays, n, any ? 1u : 0u, counts);
  return cudaGetLastError();
}

}  // namespace pfxt
