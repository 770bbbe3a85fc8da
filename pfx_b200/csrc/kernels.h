// Host-side launchers of the CUDA kernels (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>

#include "pfxt.h"
#include "traverse.cuh"

namespace pfxt {

// `counter` is one u32 of device scratch (the work-sharing counter), reset by
// the launcher on `stream` before the kernel starts.
cudaError_t launch_closest(const SceneView& s, const pfxt_ray* rays, uint32_t n, pfxt_hit* hits, uint32_t* counter,
                           cudaStream_t stream);
cudaError_t launch_any(const SceneView& s, const pfxt_ray* rays, uint32_t n, uint32_t* blocked, uint32_t* counter,
                       cudaStream_t stream);
cudaError_t launch_pack_flags(const uint32_t* flags, uint8_t* bytes, uint32_t n, cudaStream_t stream);
// Loads the any-hit and flag-packing kernels on the current device and computes
// the any-hit kernel's persistent grid there (CUDA loads modules lazily, on a
// kernel's first use, which can allocate device memory).
cudaError_t prepare_any_queries();
// The same for the no-allocation entry point's module (noalloc.cu): resolves its
// scratch arrays on `device`, which must be current.
cudaError_t noalloc_prepare(int device);
cudaError_t launch_counts(const SceneView& s, const pfxt_ray* rays, uint32_t n, bool any, uint2* counts,
                          uint32_t* counter, cudaStream_t stream);

}  // namespace pfxt
