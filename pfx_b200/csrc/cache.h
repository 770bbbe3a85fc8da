// The neural radiance cache: a multiresolution hash-grid encoding of the
// hit position (Mueller et al. 2022, "Instant neural graphics primitives")
// with one-blob encoded direction and normal and the surface's albedos,
// feeding a 64-wide MLP with two hidden ReLU layers and an RGB output
// (Mueller et al. 2021, "Real-time neural radiance caching for path
// tracing"), trained online with Adam (Kingma & Ba 2015) on the radiance the
// tracer's own training paths carry.  The reference tracer has no cache:
// this is the learned part of the CUDA path, used by pfxt_set_cache.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "pfxt.h"

namespace pfxt {

constexpr uint32_t NRC_LEVELS = 16;     // hash-grid levels
constexpr uint32_t NRC_FEATURES = 2;    // features per level (FP16 in the table)
constexpr uint32_t NRC_IN = 64;         // network inputs: 32 grid features + 32 extras
constexpr uint32_t NRC_HIDDEN = 64;     // width of the two hidden layers
constexpr uint32_t NRC_OUT = 16;        // output rows of the last layer (RGB in 0..2, the rest zero)
constexpr uint32_t NRC_ROWS = 128;      // rows per tensor-core tile (= TMEM lanes)
constexpr uint32_t NRC_CELLS = 16;      // cells per axis of the error grid (fallback decisions)
// FP32 master parameters of the MLP: W1 [64 x 64], W2 [64 x 64], W3 [16 x 64], row = output.
constexpr uint32_t NRC_W1 = 0, NRC_W2 = NRC_HIDDEN * NRC_IN, NRC_W3 = NRC_W2 + NRC_HIDDEN * NRC_HIDDEN;
constexpr uint32_t NRC_MLP = NRC_W3 + NRC_OUT * NRC_HIDDEN;  // 9216

// The grid's geometry (device-side copy in every kernel's parameters).
struct CacheGrid {
  float lo[3], inv_extent[3];
  float scale[NRC_LEVELS];
  uint32_t resolution[NRC_LEVELS];
  uint32_t dense;         // bit l: level l indexes densely
  uint32_t entries;       // table entries per level (power of two)
  uint32_t wait_limit;    // mbarrier polls before a wait for the tensor cores gives up
};

constexpr uint32_t NRC_WAIT_LIMIT = 1u << 22;  // default of CacheGrid::wait_limit

// Device views the tracer needs from an attached cache.
struct CacheView {
  CacheGrid grid;
  const __half2* table;       // [levels][entries] FP16 features
  const uint16_t* weights;    // bf16 W1, W2, W3 in tile order (umma::tile_offset)
  const uint8_t* cell_ok;     // NRC_CELLS^3: 1 = paths may end into the cache here
  float* cell_stats;          // NRC_CELLS^3 x 4: sum(pred - target), sum(target), count, unused (luma)
};

}  // namespace pfxt

struct pfxt_cache {
  int device = 0;
  pfxt_cache_settings s{};
  pfxt::CacheGrid grid{};
  float* d_mlp = nullptr;        // FP32 master, NRC_MLP
  float* d_mlp_m = nullptr;      // Adam first moments
  float* d_mlp_v = nullptr;      // Adam second moments
  float* d_mlp_g = nullptr;      // gradient accumulator
  uint16_t* d_weights = nullptr; // bf16 copy in tile order
  float* d_table = nullptr;      // FP32 master, levels x entries x 2
  float* d_table_m = nullptr;
  float* d_table_v = nullptr;
  float* d_table_g = nullptr;
  __half2* d_table16 = nullptr;  // FP16 copy
  uint8_t* d_cell_ok = nullptr;
  float* d_cell_stats = nullptr;
  float* d_loss = nullptr;       // [0] loss sum, [1] rows, per step
  uint32_t* d_step = nullptr;    // [0] Adam steps taken, [1] this step ran
  uint32_t* d_error = nullptr;   // device error word (bounded waits)
  void* d_stage = nullptr;       // staging of the host-buffer entry points
  size_t stage_bytes = 0;
  cudaStream_t stream = nullptr;
  uint64_t steps = 0;
  float last_loss = 0.0f;
  uint32_t last_records = 0, last_queries = 0, last_training_paths = 0;
  bool broken = false;           // a drain wait ran out: TMEM may be held, nothing runs again
  std::mutex lock;
};

namespace pfxt {

void cache_validate(const pfxt_cache_settings& s);  // throws Invalid
void cache_create(pfxt_cache& c, const pfxt_cache_settings& s);
void cache_release(pfxt_cache& c);
void cache_set_bounds(pfxt_cache& c, const float lo[3], const float hi[3]);
CacheView cache_view(pfxt_cache& c);
// Device bytes of the encoded inputs of `n` queries (cache_infer_launch's `x`).
size_t cache_x_bytes(uint32_t n);
// Inference over `n` queries (5 float4 each) on `stream`; out[k] = rgb, or
// out[scatter[k]].  `n_dev`, if set, is read on the device instead of `n`
// (an upper bound).  `x` (cache_x_bytes(n), 16-byte aligned) holds the
// encoded inputs between the gather and the MLP.
void cache_infer_launch(pfxt_cache& c, const float4* queries, const uint32_t* n_dev, uint32_t n, const uint32_t* scatter,
                        float4* out, uint8_t* x, cudaStream_t stream);
// One training step over records [first, first + batch) of `records`
// (6 float4 each) when at least first + batch exist (`count_dev` on the
// device, or `count` when it is null); then Adam.
// `batch` 0 means the settings' batch.  Without Adam only the gradients are
// accumulated (d_mlp_g, d_table_g), and nothing else changes.
void cache_train_launch(pfxt_cache& c, const float4* records, const uint32_t* count_dev, uint32_t count,
                        uint32_t first, cudaStream_t stream, bool adam, uint32_t batch);
// After the steps of a pass: refresh the per-cell fallback decisions.
void cache_cells_launch(pfxt_cache& c, cudaStream_t stream);
void cache_check_error(pfxt_cache& c);
// Rewrites the BF16 weights and FP16 table from the FP32 masters.
void cache_copies(pfxt_cache& c);

}  // namespace pfxt
