// Tracer state behind a pfxt_trace handle and the host functions that drive
// the path-tracing kernels (tracer.cu, converge.cu).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "pfxt.h"
#include "pfxt_internal.h"
#include "traverse.cuh"

namespace pfxt {

struct DeviceError : std::runtime_error {
  explicit DeviceError(const std::string& m) : std::runtime_error(m) {}
};

// The per-pass uniform of the reference (Frame, gpu.rs:157-171) for the
// fields this tracer reads.
struct FrameParams {
  uint32_t size[4];    // width, height, accumulated samples, samples this pass
  uint32_t counts[4];  // triangles, shapes, seed, unused
  float origin[4];     // camera origin, w = projection kind
  float forward[4];
  float right[4];      // w = orthographic half width
  float up[4];         // w = orthographic half height
  float sun_dir[4];    // w = cos(sun radius)
  float sun_color[4];  // w = intensity
  float lens[4];       // shift x, shift y, aperture radius, focus distance
  uint32_t window[4];  // full width, full height, tile origin x, y
};

// Pipeline-constant specialisation (gpu.rs:1140-1196).
struct Specialise {
  uint32_t total_bounces, diffuse_bounces, glossy_bounces, transmission_bounces;
  uint32_t sobol;         // SOBOL
  uint32_t sobol_length;  // SOBOL_LENGTH
  float clamp_indirect;   // CLAMP_INDIRECT
  float filter_glossy;    // FILTER_GLOSSY
};

// Everything the shading kernels read, as device pointers.
struct ShadeView {
  const GpuTriangle* __restrict__ triangles;
  const float4* __restrict__ uv;
  const float4* __restrict__ materials;  // rows of 16 B; record m at (m+1)*8
  const GpuSurface* __restrict__ surfaces;
  const GpuEmitter* __restrict__ emitters;
  const float* __restrict__ emitter_cdf;
  const GpuLight* __restrict__ lights;
  const float4* __restrict__ light_trig;  // 2 float4 per light row: its cones' trigonometry (shade.cuh RowTrig)
  const float* __restrict__ sky_rows;
  const float* __restrict__ sky_columns;
  const float4* __restrict__ sobol;
  uint32_t sky_width, sky_height;
  float sky_radiance[3];
  float sky_sun_probability;
  uint32_t material_count;
  uint32_t emitter_count;   // emitters[0].a.x
  uint32_t looped;          // emitters[0].a.y
  uint32_t tree;            // emitters[0].a.w
};

struct Accum {
  float4 color, albedo, normal;
};

// A captured sampling pass and the launch parameters it was captured with.
struct GraphEntry {
  std::vector<unsigned char> key;
  cudaGraphExec_t exec;
  uint32_t kernels;  // kernel launches of the captured pass
};

}  // namespace pfxt

// The handle behind the C ABI.
struct pfxt_trace {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t width = 0, height = 0;
  uint32_t samples = 0;
  pfxt::FrameParams base{};
  pfxt::Specialise spec{};
  uint32_t projection = 0;
  // traversal layout
  pfxt::WideNode* d_wide = nullptr;
  pfxt::TravTri* d_tris = nullptr;
  pfxt::InstRec* d_insts = nullptr;
  pfxt::SceneView view{};
  // shading buffers
  void* d_triangles = nullptr;
  void* d_uv = nullptr;
  void* d_materials = nullptr;
  void* d_surfaces = nullptr;
  void* d_emitters = nullptr;
  void* d_emitter_cdf = nullptr;
  size_t surfaces_bytes = 0, emitters_bytes = 0, emitter_cdf_bytes = 0;  // as uploaded
  void* d_lights = nullptr;
  void* d_sky_rows = nullptr;
  void* d_sky_columns = nullptr;
  void* d_sobol = nullptr;
  pfxt::ShadeView shade{};
  // films
  pfxt::Accum* d_accum = nullptr;
  float4* d_color = nullptr;
  float4* d_albedo = nullptr;
  float4* d_normal = nullptr;
  // adaptive sampling
  float4* d_snaps = nullptr;  // 32 B per pixel: mean, info
  uint32_t* d_running = nullptr;
  // wavefront scratch (allocated on first use)
  void* d_wave = nullptr;
  size_t wave_bytes = 0;
  uint32_t wave_capacity = 0;
  alignas(16) unsigned char wave_layout[256];  // pointers into d_wave (tracer.cu)
  uint32_t light_rows = 0;                     // rows of the light buffer (lights + tree)
  uint32_t* wave_counters = nullptr;           // queue counters and ray totals inside d_wave
  uint8_t* d_mask = nullptr;                   // optional per-pixel mask of the pixels to sample
  bool sort_shading = true;                    // group the shade queue by material every bounce
  uint32_t trace_threads = 128;                // threads per block of the traversal kernels (64, 128, 256)
  bool split_shade = true;                     // shade in three kernels (hit, lights, BSDF) or one
  bool sort_rays = false;                      // group the extend queue of later bounces by ray
  bool shadow_queue = true;                    // light slots' shadow rays through the connect queue
  uint32_t short_stack = 0;                    // traversal stack entries per lane in shared memory (0 or 8)
  bool slot_kernels = true;                    // deferred light slots one kind per launch (or all in one kernel)
  uint64_t tune_key = 0;                       // hash of the scene's buffers, film and settings (autotune cache)
  float tuned_pass_ms = 0.0f;                  // the autotuner's measured pass time, 0 = not tuned
  uint32_t* d_error = nullptr;  // device error word
  uint32_t* d_counters = nullptr;  // ring of work-sharing counters (device scratch)
  uint32_t counter_slot = 0;
  void* d_stage = nullptr;      // staging of the host-memory ray entry points
  size_t stage_bytes = 0;
  std::vector<void*> owned;
  // radiance cache (pfxt_set_cache)
  float bounds_lo[3] = {0, 0, 0}, bounds_hi[3] = {0, 0, 0};  // world box of the scene root
  pfxt_cache* cache = nullptr;
  void* d_cache_scratch = nullptr;  // queries, predictions, training vertices and records
  size_t cache_scratch_bytes = 0;
  // CUDA graphs of the sampling pass (tracer.cu)
  uint32_t* d_vars = nullptr;  // accumulated samples, samples this pass, seed, camera (tracer.cu)
  uint32_t* h_vars = nullptr;  // pinned mirror, copied in by the pass's first node
  // The cache inference runs on `side`, forked from `stream` after the last
  // query bounce and joined before the accumulation, beside the later bounces.
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  // the next bounce's extend, beside the current bounce's connect
  cudaStream_t ahead = nullptr;
  cudaEvent_t ahead_fork = nullptr, ahead_join = nullptr;
  std::vector<pfxt::GraphEntry> graphs;
  bool use_graphs = true;
  uint32_t graph_captures = 0;  // passes captured so far
  uint32_t pass_kernels = 0;    // kernel launches of the last pass replayed from a graph
};

namespace pfxt {

void trace_init(pfxt_trace& t, const pfxt_buffers& b, const pfxt_scene& view, const pfxt_settings& s, uint32_t width,
                uint32_t height);
void trace_release(pfxt_trace& t);
void trace_set_camera(pfxt_trace& t, const pfxt_camera& c);
void trace_set_lens(pfxt_trace& t, const float lens[4]);
void trace_set_window(pfxt_trace& t, const uint32_t full[2], const uint32_t origin[2]);
void trace_sample(pfxt_trace& t, uint32_t count, uint32_t seed);
// The light rows' cone trigonometry (ShadeView::light_trig), once per tracer.
void light_trig_init(pfxt_trace& t);
// Drops the captured passes (their buffers or launch parameters changed).
void trace_forget_graphs(pfxt_trace& t);
void trace_set_projection(pfxt_trace& t, uint32_t projection, const float ortho[2]);
// Uploads the node, surface and emitter buffers of a scene whose instances
// moved (Trace::finish_tops, gpu.rs:2533) and lays the traversal nodes again.
void trace_move_scene(pfxt_trace& t, const pfxt_buffers& b);
void trace_set_tuning(pfxt_trace& t, const pfxt_tuning& k);
pfxt_tuning trace_get_tuning(const pfxt_trace& t);
pfxt_tuning trace_autotune(pfxt_trace& t, uint32_t passes);
// What Trace::sample_adaptive_kept adds (adaptive.rs:136-277): the rounds a
// resumed render had reached (its accumulation, films and snapshots are
// restored by the caller), and a keeper asked after every sample whether a
// checkpoint is due and handed the rounds reached so far when one is.
struct AdaptiveKeeping {
  std::vector<pfxt_round> resumed;
  bool resuming = false;
  std::function<bool(uint32_t samples)> due;                        // empty: no keeper
  std::function<void(const std::vector<pfxt_round>& reached)> keep;
};
void trace_sample_adaptive(pfxt_trace& t, const pfxt_adaptive& a, uint32_t seed, pfxt_round* rounds, uint32_t cap,
                           uint32_t* written, const AdaptiveKeeping* keeping = nullptr);
bool adaptive_valid(const pfxt_adaptive& a);
void trace_adaptive_measure(pfxt_trace& t, bool first);
uint32_t trace_adaptive_mark(pfxt_trace& t, uint32_t min_samples, float threshold);
std::vector<uint32_t> adaptive_rounds(const pfxt_adaptive& a);
void trace_readback(pfxt_trace& t, float* color, float* albedo, float* normal);
void trace_sample_counts(pfxt_trace& t, uint32_t* counts);
void trace_read_accum(pfxt_trace& t, float* accum);
// Next counter of the ring: consecutive launches (possibly on different
// streams) never share a counter.
inline uint32_t* next_counter(pfxt_trace& t) {
  uint32_t* c = t.d_counters + (t.counter_slot % 64u);
  t.counter_slot += 1u;
  return c;
}

}  // namespace pfxt
