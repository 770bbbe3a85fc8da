// Host-side launchers of the CUDA kernels (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>

#include "pfxt.h"
#include "traverse.cuh"

namespace pfxt {

cudaError_t launch_closest(const SceneView& s, const pfxt_ray* rays, uint32_t n, pfxt_hit* hits, cudaStream_t stream);
cudaError_t launch_any(const SceneView& s, const pfxt_ray* rays, uint32_t n, uint32_t* blocked, cudaStream_t stream);
cudaError_t launch_pack_flags(const uint32_t* flags, uint8_t* bytes, uint32_t n, cudaStream_t stream);
cudaError_t launch_counts(const SceneView& s, const pfxt_ray* rays, uint32_t n, bool any, uint2* counts,
                          cudaStream_t stream);

}  // namespace pfxt
