// The denoiser: OIDN's RT filter (the reference's crates/denoise, itself
// OIDN 2.5.1's UNetFilter) on sm_100a.  Internal declarations behind the
// pfxt_denoiser_* entry points of include/pfxt.h; denoise.cu.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace pfxt {

// One 3x3 convolution of the U-Net (net.rs:8-21): its sources, whether it
// pools its output or upsamples its first source, the resolution level of its
// input, and its channel counts; device weights in the layout conv_chunks()
// describes.
struct DenoiseLayer {
  std::string name;
  int src0 = -1, src1 = -2;  // -1: the input tensor; -2: none; else a layer
  bool pool = false, upsample = false;
  uint32_t level = 0;
  uint32_t in0 = 0, in1 = 0, out = 0;
  uint32_t c0 = 0, c1 = 0, n = 0;  // padded to 16: channels of each source, output channels
  std::vector<uint16_t> weights;  // host copy, fp16, chunk-major (see denoise.cu)
  std::vector<float> bias;        // n values
  uint16_t* d_weights = nullptr;
  float* d_bias = nullptr;
  uint32_t out_level() const { return level + (pool ? 1u : 0u); }
};

// A tile of the split (tile.rs:4-12), (y, x) pairs.
struct DenoiseTile {
  uint32_t src[2], dst[2], size[2], out_src[2], out_dst[2], out_size[2];
};

struct DenoisePlan {
  uint32_t tile_h = 0, tile_w = 0, overlap = 0;
  std::vector<DenoiseTile> tiles;
};

DenoisePlan denoise_plan(uint32_t height, uint32_t width, uint64_t max_tile_pixels);

struct Denoiser {
  std::vector<DenoiseLayer> layers;
  uint64_t max_tile_pixels = 2160ull * 2160ull;
  int device = 0;
  // per image size: the plan and the tile tensors
  uint32_t width = 0, height = 0;
  DenoisePlan plan;
  std::vector<uint16_t*> tensors;  // [0] the input tensor, [1 + i] layer i's output: hi plane, then lo plane
  std::vector<uint32_t> stored_level;  // the level each tensor is stored at (an upsampled source: one below)
  std::shared_ptr<void> launches;      // per layer: the convolution's arguments and tensor maps (denoise.cu)
  float* d_scale = nullptr;     // autoexposure: one float
  float* d_bins = nullptr;
  size_t bins_capacity = 0;
  uint32_t* d_error = nullptr;  // set by a conv kernel whose bounded wait ran out
  uint32_t wait_limit = 1u << 26;  // polls of the conv kernels' bounded mbarrier waits
  uint32_t conv_shape = 0;         // 0 the per-layer default, 1-9 one shape wherever it fits
  cudaStream_t stream = nullptr;   // host-buffer calls
  float4* d_images = nullptr;      // host-buffer calls: colour, albedo, normal, output
  size_t images_pixels = 0;
  char* h_stage = nullptr;         // host-buffer calls: two pinned halves of DENOISE_STAGE_BYTES
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};  // the last copy through each half
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.0f;          // device time of the last denoise
  uint64_t last_macs = 0;        // multiply-adds of the last denoise (padded channels included)
  ~Denoiser();
};

// Parses an OIDN tensor archive (tza.rs:51-118) and builds the network
// (net.rs:193-232) on the current device; throws Invalid on a bad blob.
Denoiser* denoiser_create(const void* blob, size_t bytes);
void denoiser_prepare(Denoiser& d, uint32_t width, uint32_t height);
void denoise_device(Denoiser& d, uint32_t width, uint32_t height, const float4* color, const float4* albedo,
                    const float4* normal, float4* out, cudaStream_t stream);
// Waits for the last denoise; its device time in ms.  Throws DeviceError when
// a convolution's bounded wait ran out.
float denoiser_finish(Denoiser& d);
// The host-buffer form (pfxt_denoise): the images go up and the result comes
// back through two pinned halves of a staging buffer, host copies into one
// half overlapping the device copy of the other; returns when the result is
// in `out`.
constexpr size_t DENOISE_STAGE_BYTES = 16u << 20;
void denoise_host(Denoiser& d, uint32_t width, uint32_t height, const float* color, const float* albedo,
                  const float* normal, float* out);

}  // namespace pfxt
