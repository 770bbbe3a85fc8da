// The C ABI of libpfxtrace (include/pfxt.h): handle management, uploads and
// the blocking host-memory entry points.  Kernels live in the other .cu files.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "kernels.h"
#include "pfxt.h"
#include "pfxt_internal.h"
#include "tracer.h"
#include "cache.h"
#include "denoise.h"

using namespace pfxt;

namespace pfxt {
static thread_local std::string g_error;
void set_error(const std::string& message) { g_error = message; }
}  // namespace pfxt

struct pfxt_scene_blobs {
  std::unique_ptr<SceneBlobs> blobs;
};

namespace {

struct CudaFailure : std::runtime_error {
  explicit CudaFailure(const std::string& m) : std::runtime_error(m) {}
};

void check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    throw Refused(std::string(what) + ": out of device memory");
  }
  throw CudaFailure(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    set_error("");
    return PFXT_OK;
  } catch (const Invalid& e) {
    set_error(e.what());
    return PFXT_ERR_INVALID;
  } catch (const Refused& e) {
    set_error(e.what());
    return PFXT_ERR_REFUSED;
  } catch (const CudaFailure& e) {
    set_error(e.what());
    return PFXT_ERR_CUDA;
  } catch (const DeviceError& e) {
    set_error(e.what());
    return PFXT_ERR_DEVICE;
  } catch (const std::bad_alloc&) {
    set_error("out of host memory");
    return PFXT_ERR_REFUSED;
  } catch (const std::exception& e) {
    set_error(e.what());
    return PFXT_ERR_INVALID;
  }
}

template <typename T>
T* upload(const void* host, size_t bytes, const char* what) {
  if (bytes == 0) bytes = 16;
  void* d = nullptr;
  check(cudaMalloc(&d, bytes), what);
  if (host) {
    cudaError_t e = cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(d);
      check(e, what);
    }
  } else {
    cudaMemset(d, 0, bytes);
  }
  return static_cast<T*>(d);
}

// Device staging for the host-memory ray entry points: grown on demand and
// kept by the handle, so repeated calls do not allocate.
char* staging(pfxt_trace& t, size_t bytes) {
  if (bytes > t.stage_bytes) {
    if (t.d_stage) cudaFree(t.d_stage);
    t.d_stage = nullptr;
    t.stage_bytes = 0;
    check(cudaMalloc(&t.d_stage, bytes), "ray staging");
    t.stage_bytes = bytes;
  }
  return static_cast<char*>(t.d_stage);
}

void ensure_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n <= 0) {
    cudaGetLastError();
    throw Refused("no CUDA device is available");
  }
}

}  // namespace

extern "C" {

int pfxt_abi_version(void) { return PFXT_ABI_VERSION; }

const char* pfxt_last_error(void) { return g_error.c_str(); }

int pfxt_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return n;
}

int pfxt_scene_build(const pfxt_scene* scene, const pfxt_settings* settings, pfxt_scene_blobs** out) {
  return guarded([&]() {
    if (!scene || !settings || !out) throw Invalid("null argument");
    *out = nullptr;
    auto holder = std::make_unique<pfxt_scene_blobs>();
    holder->blobs.reset(build_scene(*scene, *settings));
    *out = holder.release();
  });
}

void pfxt_scene_free(pfxt_scene_blobs* blobs) { delete blobs; }

int pfxt_scene_buffers(const pfxt_scene_blobs* h, pfxt_buffers* out) {
  return guarded([&]() {
    if (!h || !out) throw Invalid("null argument");
    const SceneBlobs& b = *h->blobs;
    memset(out, 0, sizeof(*out));
    out->triangles = b.triangles.data();
    out->triangles_bytes = b.triangles.size() * sizeof(GpuTriangle);
    out->nodes = b.nodes.data();
    out->nodes_bytes = b.nodes.size() * sizeof(GpuNode);
    out->materials = b.materials.data();
    out->materials_bytes = b.materials.size() * sizeof(GpuHot);
    out->uv = b.uv.data();
    out->uv_bytes = b.uv.size() * 16;
    out->surfaces = b.surfaces.data();
    out->surfaces_bytes = b.surfaces.size() * sizeof(GpuSurface);
    out->emitters = b.emitters.data();
    out->emitters_bytes = b.emitters.size() * sizeof(GpuEmitter);
    out->emitter_cdf = b.emitter_cdf.data();
    out->emitter_cdf_bytes = b.emitter_cdf.size() * 4;
    out->lights = b.lights.data();
    out->lights_bytes = b.lights.size() * sizeof(GpuLight);
    out->triangle_count = b.triangle_count;
    out->shape_count = 0;
    out->emitter_count = b.emitter_count;
    out->light_count = b.light_count;
    out->sky_rows = b.sky_rows.data();
    out->sky_columns = b.sky_columns.data();
    out->sky_width = b.sky_width;
    out->sky_height = b.sky_height;
    memcpy(out->sky_radiance, b.sky_radiance, sizeof(out->sky_radiance));
    out->sky_sun_probability = 0.0f;
    out->sobol = b.sobol.empty() ? nullptr : b.sobol.data();
    out->sobol_length = b.sobol_length;
    out->max_depth = b.max_depth;
  });
}

int pfxt_scene_order(const pfxt_scene_blobs* h, const uint32_t** order, uint32_t* count) {
  return guarded([&]() {
    if (!h || !order || !count) throw Invalid("null argument");
    *order = h->blobs->order.data();
    *count = (uint32_t)h->blobs->order.size();
  });
}

int pfxt_create(const pfxt_buffers* b, const pfxt_scene* view, const pfxt_settings* settings, uint32_t width,
                uint32_t height, pfxt_trace** out) {
  return guarded([&]() {
    if (!b || !view || !settings || !out) throw Invalid("null argument");
    *out = nullptr;
    if (width == 0 || height == 0) throw Invalid("the film needs a width and a height");
    if ((uint64_t)width * height > (1ull << 31)) throw Invalid("the film is too large");
    if (b->shape_count != 0) throw Invalid("analytic shapes are not supported by this tracer");
    if (b->max_depth > REF_STACK) throw Invalid("the BVH needs more than the 64-entry traversal stack");
    if (b->triangles_bytes % sizeof(GpuTriangle) || b->nodes_bytes % sizeof(GpuNode) ||
        b->materials_bytes % sizeof(GpuHot) || b->surfaces_bytes < sizeof(GpuSurface) ||
        b->lights_bytes % sizeof(GpuLight) || b->emitters_bytes < sizeof(GpuEmitter))
      throw Invalid("scene buffers have invalid sizes");
    ensure_device();
    auto t = std::make_unique<pfxt_trace>();
    trace_init(*t, *b, *view, *settings, width, height);
    // load pfxt_occluded_noalloc's module and kernels now, so that it never
    // allocates on its own first call
    check(noalloc_prepare(t->device), "loading the no-allocation kernels");
    *out = t.release();
  });
}

void pfxt_destroy(pfxt_trace* t) {
  if (!t) return;
  trace_release(*t);
  delete t;
}

int pfxt_trace_rays(pfxt_trace* t, const pfxt_ray* rays, uint32_t count, pfxt_hit* hits) {
  return guarded([&]() {
    if (!t || (count && (!rays || !hits))) throw Invalid("null argument");
    if (count == 0) return;
    char* stage = staging(*t, (size_t)count * (sizeof(pfxt_ray) + sizeof(pfxt_hit)));
    pfxt_ray* d_rays = reinterpret_cast<pfxt_ray*>(stage);
    pfxt_hit* d_hits = reinterpret_cast<pfxt_hit*>(stage + (size_t)count * sizeof(pfxt_ray));
    check(cudaMemcpyAsync(d_rays, rays, (size_t)count * sizeof(pfxt_ray), cudaMemcpyHostToDevice, t->stream),
          "ray upload");
    check(launch_closest(t->view, d_rays, count, d_hits, next_counter(*t), t->stream), "closest-hit kernel");
    check(cudaMemcpyAsync(hits, d_hits, (size_t)count * sizeof(pfxt_hit), cudaMemcpyDeviceToHost, t->stream),
          "hit readback");
    check(cudaStreamSynchronize(t->stream), "closest-hit kernel");
  });
}

int pfxt_occluded(pfxt_trace* t, const pfxt_ray* rays, uint32_t count, uint8_t* blocked) {
  return guarded([&]() {
    if (!t || (count && (!rays || !blocked))) throw Invalid("null argument");
    if (count == 0) return;
    char* stage = staging(*t, (size_t)count * (sizeof(pfxt_ray) + 4 + 1));
    pfxt_ray* d_rays = reinterpret_cast<pfxt_ray*>(stage);
    uint32_t* d_blocked = reinterpret_cast<uint32_t*>(stage + (size_t)count * sizeof(pfxt_ray));
    uint8_t* d_bytes = reinterpret_cast<uint8_t*>(stage + (size_t)count * (sizeof(pfxt_ray) + 4));
    check(cudaMemcpyAsync(d_rays, rays, (size_t)count * sizeof(pfxt_ray), cudaMemcpyHostToDevice, t->stream),
          "ray upload");
    check(launch_any(t->view, d_rays, count, d_blocked, next_counter(*t), t->stream), "any-hit kernel");
    check(launch_pack_flags(d_blocked, d_bytes, count, t->stream), "flag packing");
    check(cudaMemcpyAsync(blocked, d_bytes, count, cudaMemcpyDeviceToHost, t->stream), "flag readback");
    check(cudaStreamSynchronize(t->stream), "any-hit kernel");
  });
}

int pfxt_trace_rays_device(pfxt_trace* t, const pfxt_ray* rays, uint32_t count, pfxt_hit* hits, void* stream) {
  return guarded([&]() {
    if (!t || (count && (!rays || !hits))) throw Invalid("null argument");
    check(launch_closest(t->view, rays, count, hits, next_counter(*t), (cudaStream_t)stream), "closest-hit kernel");
  });
}

int pfxt_occluded_device(pfxt_trace* t, const pfxt_ray* rays, uint32_t count, uint32_t* blocked, void* stream) {
  return guarded([&]() {
    if (!t || (count && (!rays || !blocked))) throw Invalid("null argument");
    check(launch_any(t->view, rays, count, blocked, next_counter(*t), (cudaStream_t)stream), "any-hit kernel");
  });
}

/* Work counters per ray (box tests, triangle tests); not part of the public
 * header, used by the measurement harness. */
int pfxt_trace_counts_device(pfxt_trace* t, const pfxt_ray* rays, uint32_t count, uint32_t any, uint32_t* counts,
                             void* stream) {
  return guarded([&]() {
    if (!t || (count && (!rays || !counts))) throw Invalid("null argument");
    check(launch_counts(t->view, rays, count, any != 0, reinterpret_cast<uint2*>(counts), next_counter(*t),
                        (cudaStream_t)stream),
          "counting kernel");
  });
}

int pfxt_set_camera(pfxt_trace* t, const pfxt_camera* camera) {
  return guarded([&]() {
    if (!t || !camera) throw Invalid("null argument");
    trace_set_camera(*t, *camera);
  });
}

int pfxt_set_lens(pfxt_trace* t, const float lens[4]) {
  return guarded([&]() {
    if (!t || !lens) throw Invalid("null argument");
    trace_set_lens(*t, lens);
  });
}

int pfxt_set_window(pfxt_trace* t, const uint32_t full[2], const uint32_t origin[2]) {
  return guarded([&]() {
    if (!t || !full || !origin) throw Invalid("null argument");
    trace_set_window(*t, full, origin);
  });
}

int pfxt_sample(pfxt_trace* t, uint32_t count, uint32_t seed) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    trace_sample(*t, count, seed);
  });
}

int pfxt_sample_paced(pfxt_trace* t, uint32_t count, uint32_t seed, pfxt_between between, void* user,
                      double* wall_ms) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    if ((uint64_t)t->samples + count > 0xffffffffull) throw Invalid("sample count overflow");
    auto start = std::chrono::steady_clock::now();
    cudaEvent_t ev[2] = {nullptr, nullptr};
    check(cudaEventCreate(&ev[0]), "pass timing");
    cudaError_t e = cudaEventCreate(&ev[1]);
    if (e != cudaSuccess) cudaEventDestroy(ev[0]);
    check(e, "pass timing");
    try {
      for (uint32_t i = 0; i < count; ++i) {  // one slice per sample, as Pacer slices a pass
        check(cudaEventRecord(ev[0], t->stream), "pass timing");
        trace_sample(*t, 1u, seed);
        check(cudaEventRecord(ev[1], t->stream), "pass timing");
        check(cudaEventSynchronize(ev[1]), "pass timing");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, ev[0], ev[1]), "pass timing");
        if (between) between(user, (double)ms);
      }
    } catch (...) {
      cudaEventDestroy(ev[0]);
      cudaEventDestroy(ev[1]);
      throw;
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (wall_ms) *wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
  });
}

uint32_t pfxt_samples(const pfxt_trace* t) { return t ? t->samples : 0u; }

int pfxt_adaptive_rounds(const pfxt_adaptive* a, uint32_t* rounds, uint32_t cap, uint32_t* written) {
  return guarded([&]() {
    if (!a || !written) throw Invalid("null argument");
    std::vector<uint32_t> r = adaptive_rounds(*a);
    *written = (uint32_t)std::min<size_t>(r.size(), cap);
    if (rounds)
      for (uint32_t i = 0; i < *written; ++i) rounds[i] = r[i];
    if (r.size() > cap && rounds) throw Invalid("the rounds array is too short");
  });
}

int pfxt_sample_adaptive(pfxt_trace* t, const pfxt_adaptive* a, uint32_t seed, pfxt_round* rounds, uint32_t cap,
                         uint32_t* written) {
  return guarded([&]() {
    if (!t || !a || !written) throw Invalid("null argument");
    trace_sample_adaptive(*t, *a, seed, rounds, cap, written);
  });
}

int pfxt_adaptive_measure(pfxt_trace* t, uint32_t first) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    trace_adaptive_measure(*t, first != 0u);
  });
}

int pfxt_adaptive_mark(pfxt_trace* t, uint32_t min_samples, float threshold, uint32_t* running) {
  return guarded([&]() {
    if (!t || !running) throw Invalid("null argument");
    if (!(threshold > 0.0f) || min_samples < 2) throw Invalid("adaptive sampling needs a positive threshold and at least 2 samples");
    *running = trace_adaptive_mark(*t, min_samples, threshold);
  });
}

int pfxt_adaptive_snaps_device(pfxt_trace* t, float** snaps) {
  return guarded([&]() {
    if (!t || !snaps) throw Invalid("null argument");
    *snaps = reinterpret_cast<float*>(t->d_snaps);
  });
}

int pfxt_readback(pfxt_trace* t, float* color, float* albedo, float* normal) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    trace_readback(*t, color, albedo, normal);
  });
}

int pfxt_sample_counts(pfxt_trace* t, uint32_t* counts) {
  return guarded([&]() {
    if (!t || !counts) throw Invalid("null argument");
    trace_sample_counts(*t, counts);
  });
}

int pfxt_read_accum(pfxt_trace* t, float* accum) {
  return guarded([&]() {
    if (!t || !accum) throw Invalid("null argument");
    trace_read_accum(*t, accum);
  });
}

}  // extern "C"

extern "C" {
/* The base per-pass uniform of a handle (FrameParams: size, counts, camera,
 * sun, lens, window; 160 bytes).  Not part of the public header; the
 * measurement and parity harness reads it to drive the oracle with the same
 * frame. */
int pfxt_debug_frame(const pfxt_trace* t, void* out) {
  return guarded([&]() {
    if (!t || !out) throw Invalid("null argument");
    memcpy(out, &t->base, sizeof(t->base));
  });
}

/* Closest-hit and any-hit queries traced by the sampling passes of a handle
 * so far (two u64), for the measurement harness. */
int pfxt_debug_rays(pfxt_trace* t, uint64_t* out) {
  return guarded([&]() {
    if (!t || !out) throw Invalid("null argument");
    out[0] = out[1] = 0;
    if (!t->wave_counters) return;
    cudaStreamSynchronize(t->stream);
    check(cudaMemcpy(out, t->wave_counters + 8, 16, cudaMemcpyDeviceToHost), "ray counters");
  });
}

/* The handle's CUDA stream (cudaStream_t), so a harness can record events on
 * the stream the passes run on. */
void* pfxt_debug_stream(pfxt_trace* t) { return t ? (void*)t->stream : nullptr; }

/* Turn the per-bounce material sort of the shade queue on (1, the default) or
 * off (0); the image does not change, only the time. */
int pfxt_debug_sort(pfxt_trace* t, uint32_t on) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    t->sort_shading = on != 0u;
  });
}

/* Replay each sampling pass from a captured CUDA graph (1, the default) or
 * launch its kernels one by one (0); the image does not change. */
int pfxt_debug_graphs(pfxt_trace* t, uint32_t on) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    t->use_graphs = on != 0u;
  });
}

/* The light tree's selection (slice::select_nth_unstable_by with total_cmp)
 * on `n` keys: writes the keys' original indices in the order it leaves them.
 * `rounds` (16 as the tree runs it) caps the partition rounds before the
 * deterministic fallback. */
int pfxt_debug_select_nth(const float* keys, uint32_t n, uint32_t index, int32_t rounds, uint32_t* order) {
  return guarded([&]() {
    if (!keys || !order || index >= n) throw Invalid("select: index out of range");
    select_nth_for_test(keys, n, index, rounds, order);
  });
}

/* Large triangle BVHs on the GPU (1, the default, when a device is present) or
 * always on the host (0); returns the previous setting.  The bytes are the same. */
int pfxt_debug_gpu_bvh(int32_t on) { return set_gpu_bvh(on); }

/* How many of a built scene's bottom-level BVHs were built on the GPU. */
uint32_t pfxt_debug_scene_gpu_builds(const pfxt_scene_blobs* b) {
  return b && b->blobs ? b->blobs->gpu_builds : 0u;
}

/* How many sampling passes have been captured as graphs so far. */
uint32_t pfxt_debug_graph_captures(pfxt_trace* t) { return t ? t->graph_captures : 0u; }
uint32_t pfxt_debug_pass_kernels(pfxt_trace* t) { return t ? t->pass_kernels : 0u; }

/* Restrict sampling to the pixels whose mask byte is non-zero (width*height
 * host bytes), or lift the restriction with NULL.  A measurement aid: it lets a
 * high-sample reference be accumulated on a stratified subset of a large film.
 * Restarts the accumulation. */
int pfxt_debug_pixel_mask(pfxt_trace* t, const uint8_t* mask) { return pfxt_set_pixel_mask(t, mask); }

int pfxt_set_pixel_mask(pfxt_trace* t, const uint8_t* mask) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    size_t pixels = (size_t)t->width * t->height;
    if (!mask) {
      if (t->d_mask) cudaMemsetAsync(t->d_mask, 1, pixels, t->stream);
      t->samples = 0;
      return;
    }
    if (!t->d_mask) {
      void* d = nullptr;
      check(cudaMalloc(&d, pixels), "pixel mask");
      t->owned.push_back(d);
      t->d_mask = static_cast<uint8_t*>(d);
    }
    check(cudaMemcpyAsync(t->d_mask, mask, pixels, cudaMemcpyHostToDevice, t->stream), "pixel mask");
    check(cudaStreamSynchronize(t->stream), "pixel mask");
    t->samples = 0;
  });
}

/* The films on the device (RGBA32F, width*height*4 floats each): what the
 * reference exposes as its colour/albedo/normal textures for the denoiser
 * (gpu.rs:328-330).  Valid until pfxt_destroy; written by every pass. */
int pfxt_films_device(pfxt_trace* t, float** color, float** albedo, float** normal) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    check(cudaStreamSynchronize(t->stream), "films");
    if (color) *color = reinterpret_cast<float*>(t->d_color);
    if (albedo) *albedo = reinterpret_cast<float*>(t->d_albedo);
    if (normal) *normal = reinterpret_cast<float*>(t->d_normal);
  });
}

/* ------------------------------------------------------------ checkpoints */

namespace {
constexpr char CKPT_MAGIC[8] = {'P', 'F', 'X', 'C', 'K', 'P', 'T', '1'};
constexpr uint64_t CKPT_ACCUM = 48, CKPT_TEXEL = 16, CKPT_SNAP = 32;

// Saved::read_from (checkpoint.rs:106-158): where each part of a checkpoint lies.
struct Checkpoint {
  uint32_t width = 0, height = 0, samples = 0, rounds = 0xffffffffu;
  const uint8_t* accum = nullptr;
  const uint8_t* films[3] = {nullptr, nullptr, nullptr};
  const uint8_t* round_bytes = nullptr;  // `rounds` x (u32 samples, u64 active)
  const uint8_t* snaps = nullptr;        // 32 B per pixel when rounds are present
};

Checkpoint read_checkpoint(const char* key, const void* bytes, size_t length) {
  if (!key || (!bytes && length)) throw Invalid("null argument");
  const uint8_t* p = static_cast<const uint8_t*>(bytes);
  uint64_t left = length;
  auto take = [&](uint64_t n) {
    if (n > left) throw Invalid("the checkpoint is cut short: failed to fill whole buffer");
    const uint8_t* at = p;
    p += n;
    left -= n;
    return at;
  };
  auto word = [&]() {
    uint32_t v;
    memcpy(&v, take(4), 4);
    return v;
  };
  auto longword = [&]() {
    uint64_t v;
    memcpy(&v, take(8), 8);
    return v;
  };
  if (memcmp(take(8), CKPT_MAGIC, 8) != 0) throw Invalid("not a pfx checkpoint");
  const uint64_t key_length = strlen(key);
  if (longword() != key_length) throw Invalid("the checkpoint was made by another render");
  if (memcmp(take(key_length), key, key_length) != 0) throw Invalid("the checkpoint was made by another render");
  Checkpoint c;
  c.width = word();
  c.height = word();
  c.samples = word();
  const uint64_t pixels = (uint64_t)c.width * c.height;
  if (pixels > (1ull << 40)) throw Invalid("the checkpoint is too large");
  c.accum = take(pixels * CKPT_ACCUM);
  for (auto& film : c.films) film = take(pixels * CKPT_TEXEL);
  c.rounds = word();
  if (c.rounds != 0xffffffffu) {
    c.round_bytes = p;
    for (uint32_t r = 0; r < c.rounds; ++r) {
      word();
      longword();
    }
    c.snaps = take(pixels * CKPT_SNAP);
  }
  if (left != 0) throw Invalid("the checkpoint runs on past its end");
  return c;
}
}  // namespace

int pfxt_checkpoint_read(const char* key, const void* bytes, size_t length, pfxt_checkpoint_info* out) {
  return guarded([&]() {
    Checkpoint c = read_checkpoint(key, bytes, length);
    if (out) *out = pfxt_checkpoint_info{c.width, c.height, c.samples, c.rounds};
  });
}

namespace {

// Saved::write_to (checkpoint.rs:82-104) of the trace's accumulation and films,
// with the adaptive rounds reached and the snapshots when `reached` is given.
uint64_t checkpoint_size(const pfxt_trace& t, const char* key, const std::vector<pfxt_round>* reached) {
  const uint64_t pixels = (uint64_t)t.width * t.height;
  uint64_t need = 8 + 8 + strlen(key) + 12 + pixels * (CKPT_ACCUM + 3 * CKPT_TEXEL) + 4;
  if (reached) need += reached->size() * 12 + pixels * CKPT_SNAP;
  return need;
}

void write_checkpoint(pfxt_trace& t, const char* key, const std::vector<pfxt_round>* reached, uint8_t* p) {
  const uint64_t key_length = strlen(key);
  const uint64_t pixels = (uint64_t)t.width * t.height;
  auto put = [&](const void* src, size_t n) {
    memcpy(p, src, n);
    p += n;
  };
  put(CKPT_MAGIC, 8);
  put(&key_length, 8);
  put(key, key_length);
  uint32_t head[3] = {t.width, t.height, t.samples};
  put(head, 12);
  check(cudaStreamSynchronize(t.stream), "checkpoint");
  check(cudaMemcpy(p, t.d_accum, pixels * CKPT_ACCUM, cudaMemcpyDeviceToHost), "checkpoint");
  p += pixels * CKPT_ACCUM;
  for (const float4* film : {t.d_color, t.d_albedo, t.d_normal}) {
    check(cudaMemcpy(p, film, pixels * CKPT_TEXEL, cudaMemcpyDeviceToHost), "checkpoint");
    p += pixels * CKPT_TEXEL;
  }
  if (!reached) {
    uint32_t none = 0xffffffffu;
    put(&none, 4);
    return;
  }
  uint32_t count = (uint32_t)reached->size();
  put(&count, 4);
  for (const pfxt_round& r : *reached) {
    put(&r.samples, 4);
    put(&r.active, 8);
  }
  check(cudaMemcpy(p, t.d_snaps, pixels * CKPT_SNAP, cudaMemcpyDeviceToHost), "checkpoint");
}

// Trace::restore (checkpoint.rs:188-203): the accumulation, the films and the count.
void restore_checkpoint(pfxt_trace& t, const Checkpoint& c) {
  if (c.width != t.width || c.height != t.height)
    throw Invalid("the checkpoint is " + std::to_string(c.width) + "x" + std::to_string(c.height) +
                  " and the trace " + std::to_string(t.width) + "x" + std::to_string(t.height));
  const uint64_t pixels = (uint64_t)t.width * t.height;
  check(cudaStreamSynchronize(t.stream), "restore");
  check(cudaMemcpy(t.d_accum, c.accum, pixels * CKPT_ACCUM, cudaMemcpyHostToDevice), "restore");
  float4* films[3] = {t.d_color, t.d_albedo, t.d_normal};
  for (int k = 0; k < 3; ++k)
    check(cudaMemcpy(films[k], c.films[k], pixels * CKPT_TEXEL, cudaMemcpyHostToDevice), "restore");
  t.samples = c.samples;
}

}  // namespace

int pfxt_save(pfxt_trace* t, const char* key, void* bytes, size_t capacity, size_t* written) {
  return guarded([&]() {
    if (!t || !key || !written) throw Invalid("null argument");
    const uint64_t need = checkpoint_size(*t, key, nullptr);
    *written = (size_t)need;
    if (!bytes) return;
    if (capacity < need) throw Invalid("the buffer is smaller than the checkpoint");
    write_checkpoint(*t, key, nullptr, static_cast<uint8_t*>(bytes));
  });
}

int pfxt_restore(pfxt_trace* t, const char* key, const void* bytes, size_t length) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    restore_checkpoint(*t, read_checkpoint(key, bytes, length));
  });
}

int pfxt_sample_adaptive_kept(pfxt_trace* t, const pfxt_adaptive* a, uint32_t seed, const char* key,
                              const pfxt_keeper* keeper, pfxt_round* rounds, uint32_t cap, uint32_t* written) {
  return guarded([&]() {
    if (!t || !a || !key || !written) throw Invalid("null argument");
    if (!adaptive_valid(*a))
      throw Invalid("adaptive sampling needs a positive threshold, a growth over 1 and at least 2 samples");
    AdaptiveKeeping keeping;
    if (keeper && keeper->resume) {
      Checkpoint c = read_checkpoint(key, keeper->resume, keeper->resume_length);
      // checked before anything is restored, as the reference checks (adaptive.rs:236-243)
      if (c.rounds == 0xffffffffu || c.rounds >= adaptive_rounds(*a).size())
        throw Invalid("the checkpoint holds no adaptive rounds for this render");
      restore_checkpoint(*t, c);
      const uint64_t pixels = (uint64_t)t->width * t->height;
      check(cudaMemcpy(t->d_snaps, c.snaps, pixels * CKPT_SNAP, cudaMemcpyHostToDevice), "restore");
      for (uint32_t r = 0; r < c.rounds; ++r) {
        pfxt_round round{0u, 0u, 0u};
        memcpy(&round.samples, c.round_bytes + 12 * r, 4);
        memcpy(&round.active, c.round_bytes + 12 * r + 4, 8);
        keeping.resumed.push_back(round);
      }
      keeping.resuming = true;
    }
    if (keeper && keeper->due) {
      if (!keeper->keep) throw Invalid("a keeper that is due must keep");
      keeping.due = [&](uint32_t samples) { return keeper->due(keeper->user, samples) != 0; };
      keeping.keep = [&](const std::vector<pfxt_round>& reached) {
        std::vector<uint8_t> bytes((size_t)checkpoint_size(*t, key, &reached));
        write_checkpoint(*t, key, &reached, bytes.data());
        if (keeper->keep(keeper->user, bytes.data(), bytes.size()) != 0)
          throw Invalid("the keeper could not keep the checkpoint");
      };
    }
    trace_sample_adaptive(*t, *a, seed, rounds, cap, written, &keeping);
  });
}

int pfxt_set_projection(pfxt_trace* t, uint32_t projection, const float ortho[2]) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    trace_set_projection(*t, projection, ortho);
  });
}

/* ------------------------------------------------------- moving instances */

// The radiance cache's grid box: the scene root's box, padded by 1e-3 of its
// extent (plus 1e-4) so that surface points on the box still hash inside.
static void bind_cache_bounds(const pfxt_trace& t, pfxt_cache& c) {
  float lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    float pad = 1e-3f * (t.bounds_hi[k] - t.bounds_lo[k]) + 1e-4f;
    lo[k] = t.bounds_lo[k] - pad;
    hi[k] = t.bounds_hi[k] + pad;
  }
  cache_set_bounds(c, lo, hi);
}

int pfxt_scene_move_instances(pfxt_scene_blobs* h, const float* transforms, uint32_t count, uint32_t* moved) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    bool any = move_instances(*h->blobs, transforms, count);
    if (moved) *moved = any ? 1u : 0u;
  });
}

int pfxt_scene_builds(const pfxt_scene_blobs* h, uint32_t* bottom, uint32_t* top) {
  return guarded([&]() {
    if (!h || !bottom || !top) throw Invalid("null argument");
    *bottom = h->blobs->bottom_builds;
    *top = h->blobs->top_builds;
  });
}

int pfxt_finish_tops(pfxt_trace* t, const pfxt_buffers* b) {
  return guarded([&]() {
    if (!t || !b) throw Invalid("null argument");
    if (b->max_depth > REF_STACK) throw Invalid("the BVH needs more than the 64-entry traversal stack");
    if (b->nodes_bytes % sizeof(GpuNode) || b->triangles_bytes % sizeof(GpuTriangle))
      throw Invalid("scene buffers have invalid sizes");
    trace_move_scene(*t, *b);
    if (t->cache) bind_cache_bounds(*t, *t->cache);
  });
}

int pfxt_set_instance_transforms(pfxt_trace* t, pfxt_scene_blobs* h, const float* transforms, uint32_t count,
                                 uint32_t* moved) {
  return guarded([&]() {
    if (!t || !h) throw Invalid("null argument");
    if (moved) *moved = 0u;
    if (!move_instances(*h->blobs, transforms, count)) return;
    if (h->blobs->max_depth > REF_STACK) throw Invalid("the BVH needs more than the 64-entry traversal stack");
    pfxt_buffers b;
    if (pfxt_scene_buffers(h, &b) != PFXT_OK) throw Invalid(pfxt_last_error());
    trace_move_scene(*t, b);
    if (t->cache) bind_cache_bounds(*t, *t->cache);
    if (moved) *moved = 1u;
  });
}

/* ------------------------------------------------------------ launch tuning */

int pfxt_get_tuning(pfxt_trace* t, pfxt_tuning* out) {
  return guarded([&]() {
    if (!t || !out) throw Invalid("null argument");
    *out = trace_get_tuning(*t);
  });
}

int pfxt_set_tuning(pfxt_trace* t, const pfxt_tuning* k) {
  return guarded([&]() {
    if (!t || !k) throw Invalid("null argument");
    trace_set_tuning(*t, *k);
  });
}

int pfxt_autotune(pfxt_trace* t, uint32_t passes, pfxt_tuning* out) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    pfxt_tuning k = trace_autotune(*t, passes);
    if (out) *out = k;
  });
}

/* ------------------------------------------------------------ radiance cache */

int pfxt_cache_defaults(pfxt_cache_settings* s) {
  return guarded([&]() {
    if (!s) throw Invalid("null argument");
    *s = pfxt_cache_settings{};
    s->log2_entries = 19;
    s->base_resolution = 16;
    s->max_resolution = 2048;
    s->batch = 65536;
    s->steps = 4;
    s->seed = 1;
    s->query_bounce = 1;  // 4K room, relMSE 0.01: 3.65x sooner than plain at vertex 1, 2.47x at vertex 2
    s->record_bounces = 4;
    s->min_roughness = 0.25f;
    s->delay_bounces = 2;
    s->learning_rate = 1e-2f;
    s->beta1 = 0.9f;
    s->beta2 = 0.99f;
    s->epsilon = 1e-15f;
    s->train_fraction = 0.01f;
    s->error_bound = 1.0f;
    for (int k = 0; k < 3; ++k) {
      s->lo[k] = 0.0f;
      s->hi[k] = 1.0f;
    }
  });
}

int pfxt_cache_create(const pfxt_cache_settings* s, pfxt_cache** out) {
  return guarded([&]() {
    if (!s || !out) throw Invalid("null argument");
    *out = nullptr;
    cache_validate(*s);
    ensure_device();
    auto c = std::make_unique<pfxt_cache>();
    try {
      cache_create(*c, *s);
    } catch (...) {
      cache_release(*c);
      throw;
    }
    *out = c.release();
  });
}

void pfxt_cache_destroy(pfxt_cache* c) {
  if (!c) return;
  cache_release(*c);
  delete c;
}

int pfxt_set_cache(pfxt_trace* t, pfxt_cache* c) {
  return guarded([&]() {
    if (!t) throw Invalid("null argument");
    check(cudaStreamSynchronize(t->stream), "set cache");
    if (c) {
      if (c->device != t->device) throw Invalid("the cache belongs to another device");
      if (c->s.record_bounces > 7) throw Invalid("a tracer records at most vertices 0..7 for the cache");
      bind_cache_bounds(*t, *c);
    }
    trace_forget_graphs(*t);
    t->cache = c;
    t->samples = 0;
  });
}

int pfxt_cache_get_stats(pfxt_cache* c, pfxt_cache_stats* out) {
  return guarded([&]() {
    if (!c || !out) throw Invalid("null argument");
    std::lock_guard<std::mutex> g(c->lock);
    check(cudaStreamSynchronize(c->stream), "cache stats");
    uint32_t step[2];
    check(cudaMemcpy(step, c->d_step, 8, cudaMemcpyDeviceToHost), "cache stats");
    std::vector<uint8_t> ok(NRC_CELLS * NRC_CELLS * NRC_CELLS);
    check(cudaMemcpy(ok.data(), c->d_cell_ok, ok.size(), cudaMemcpyDeviceToHost), "cache stats");
    *out = pfxt_cache_stats{};
    out->steps = step[0];
    out->loss = c->last_loss;
    out->records = c->last_records;
    out->queries = c->last_queries;
    out->training_paths = c->last_training_paths;
    for (uint8_t v : ok) out->cells_ok += v;
  });
}

namespace {
// Device staging of the cache's host-buffer entry points.
char* cache_stage(pfxt_cache& c, size_t bytes) {
  if (bytes > c.stage_bytes) {
    if (c.d_stage) cudaFree(c.d_stage);
    c.d_stage = nullptr;
    c.stage_bytes = 0;
    check(cudaMalloc(&c.d_stage, bytes), "cache staging");
    c.stage_bytes = bytes;
  }
  return static_cast<char*>(c.d_stage);
}
}  // namespace

int pfxt_cache_set_wait_limit(pfxt_cache* c, uint32_t polls) {
  return guarded([&]() {
    if (!c) throw Invalid("null argument");
    std::lock_guard<std::mutex> g(c->lock);
    c->grid.wait_limit = polls;
  });
}

int pfxt_cache_infer(pfxt_cache* c, const pfxt_cache_query* q, uint32_t count, float* rgb) {
  return guarded([&]() {
    if (!c || (count && (!q || !rgb))) throw Invalid("null argument");
    if (count == 0) return;
    std::lock_guard<std::mutex> g(c->lock);
    size_t qb = (size_t)count * sizeof(pfxt_cache_query), xo = (qb + (size_t)count * 16u + 255u) & ~size_t(255);
    char* d = cache_stage(*c, xo + cache_x_bytes(count));
    float4* d_out = reinterpret_cast<float4*>(d + qb);
    check(cudaMemcpyAsync(d, q, qb, cudaMemcpyHostToDevice, c->stream), "cache queries");
    cache_infer_launch(*c, reinterpret_cast<const float4*>(d), nullptr, count, nullptr, d_out,
                       reinterpret_cast<uint8_t*>(d + xo), c->stream);
    std::vector<float4> out(count);
    check(cudaMemcpyAsync(out.data(), d_out, (size_t)count * 16u, cudaMemcpyDeviceToHost, c->stream), "cache output");
    check(cudaStreamSynchronize(c->stream), "cache inference");
    cache_check_error(*c);
    for (uint32_t k = 0; k < count; ++k) {
      rgb[3 * k + 0] = out[k].x;
      rgb[3 * k + 1] = out[k].y;
      rgb[3 * k + 2] = out[k].z;
    }
  });
}

int pfxt_cache_gradients(pfxt_cache* c, const pfxt_cache_record* r, uint32_t count, float* mlp, float* table,
                         float* loss) {
  return guarded([&]() {
    if (!c || !r || !mlp) throw Invalid("null argument");
    if (count == 0 || count % NRC_ROWS != 0 || count > (1u << 22))
      throw Invalid("records: a positive multiple of 128, at most 2^22");
    std::lock_guard<std::mutex> g(c->lock);
    const size_t table_n = (size_t)NRC_LEVELS * c->grid.entries * 2u;
    size_t rb = (size_t)count * sizeof(pfxt_cache_record);
    char* d = cache_stage(*c, rb);
    check(cudaMemsetAsync(c->d_mlp_g, 0, NRC_MLP * 4u, c->stream), "cache gradients");
    check(cudaMemsetAsync(c->d_table_g, 0, table_n * 4u, c->stream), "cache gradients");
    check(cudaMemcpyAsync(d, r, rb, cudaMemcpyHostToDevice, c->stream), "cache records");
    cache_train_launch(*c, reinterpret_cast<const float4*>(d), nullptr, count, 0, c->stream, false, count);
    check(cudaMemcpyAsync(mlp, c->d_mlp_g, NRC_MLP * 4u, cudaMemcpyDeviceToHost, c->stream), "cache gradients");
    if (table)
      check(cudaMemcpyAsync(table, c->d_table_g, table_n * 4u, cudaMemcpyDeviceToHost, c->stream), "cache gradients");
    float l = 0.0f;
    check(cudaMemcpyAsync(&l, c->d_loss, 4, cudaMemcpyDeviceToHost, c->stream), "cache loss");
    check(cudaMemsetAsync(c->d_mlp_g, 0, NRC_MLP * 4u, c->stream), "cache gradients");
    check(cudaMemsetAsync(c->d_table_g, 0, table_n * 4u, c->stream), "cache gradients");
    check(cudaStreamSynchronize(c->stream), "cache gradients");
    cache_check_error(*c);
    if (loss) *loss = l / (3.0f * (float)count);
  });
}

int pfxt_cache_train(pfxt_cache* c, const pfxt_cache_record* r, uint32_t count, float* loss) {
  return guarded([&]() {
    if (!c || !r) throw Invalid("null argument");
    if (count == 0 || count % c->s.batch != 0) throw Invalid("records: a positive multiple of the batch");
    std::lock_guard<std::mutex> g(c->lock);
    size_t rb = (size_t)count * sizeof(pfxt_cache_record);
    char* d = cache_stage(*c, rb);
    check(cudaMemcpyAsync(d, r, rb, cudaMemcpyHostToDevice, c->stream), "cache records");
    double sum = 0.0;
    uint32_t steps = count / c->s.batch;
    for (uint32_t s = 0; s < steps; ++s) {
      cache_train_launch(*c, reinterpret_cast<const float4*>(d), nullptr, count, s * c->s.batch, c->stream, true, 0);
      float l = 0.0f;
      check(cudaMemcpyAsync(&l, c->d_loss, 4, cudaMemcpyDeviceToHost, c->stream), "cache loss");
      check(cudaStreamSynchronize(c->stream), "cache training");
      sum += l / (3.0 * c->s.batch);
    }
    cache_check_error(*c);
    c->last_loss = (float)(sum / steps);
    if (loss) *loss = c->last_loss;
  });
}

int pfxt_cache_params(pfxt_cache* c, float* mlp, float* table) {
  return guarded([&]() {
    if (!c) throw Invalid("null argument");
    std::lock_guard<std::mutex> g(c->lock);
    check(cudaStreamSynchronize(c->stream), "cache parameters");
    const size_t table_n = (size_t)NRC_LEVELS * c->grid.entries * 2u;
    if (mlp) check(cudaMemcpy(mlp, c->d_mlp, NRC_MLP * 4u, cudaMemcpyDeviceToHost), "cache parameters");
    if (table) check(cudaMemcpy(table, c->d_table, table_n * 4u, cudaMemcpyDeviceToHost), "cache parameters");
  });
}

int pfxt_cache_set_params(pfxt_cache* c, const float* mlp, const float* table) {
  return guarded([&]() {
    if (!c) throw Invalid("null argument");
    std::lock_guard<std::mutex> g(c->lock);
    check(cudaStreamSynchronize(c->stream), "cache parameters");
    const size_t table_n = (size_t)NRC_LEVELS * c->grid.entries * 2u;
    if (mlp) {
      for (uint32_t i = 3u * NRC_HIDDEN; i < NRC_OUT * NRC_HIDDEN; ++i)
        if (mlp[NRC_W3 + i] != 0.0f) throw Invalid("rows 3..15 of W3 must stay zero");
      check(cudaMemcpy(c->d_mlp, mlp, NRC_MLP * 4u, cudaMemcpyHostToDevice), "cache parameters");
    }
    if (table) check(cudaMemcpy(c->d_table, table, table_n * 4u, cudaMemcpyHostToDevice), "cache parameters");
    cache_copies(*c);
    check(cudaStreamSynchronize(c->stream), "cache parameters");
  });
}

int pfxt_cache_encoding(pfxt_cache* c, float scales[16], uint32_t resolutions[16], uint32_t* dense) {
  return guarded([&]() {
    if (!c) throw Invalid("null argument");
    for (uint32_t l = 0; l < NRC_LEVELS; ++l) {
      if (scales) scales[l] = c->grid.scale[l];
      if (resolutions) resolutions[l] = c->grid.resolution[l];
    }
    if (dense) *dense = c->grid.dense;
  });
}
}  // extern "C"

/* ------------------------------------------------------------ denoiser */

struct pfxt_denoiser {
  std::unique_ptr<pfxt::Denoiser> d;
};

extern "C" {

int pfxt_denoiser_create(const void* tza, size_t bytes, pfxt_denoiser** out) {
  return guarded([&]() {
    if (!out) throw Invalid("null argument");
    *out = nullptr;
    auto h = std::make_unique<pfxt_denoiser>();
    h->d.reset(denoiser_create(tza, bytes));
    *out = h.release();
  });
}

void pfxt_denoiser_destroy(pfxt_denoiser* denoiser) { delete denoiser; }

int pfxt_denoise(pfxt_denoiser* h, uint32_t width, uint32_t height, const float* color, const float* albedo,
                 const float* normal, float* out) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    denoise_host(*h->d, width, height, color, albedo, normal, out);
  });
}

int pfxt_denoise_device(pfxt_denoiser* h, uint32_t width, uint32_t height, const float* color, const float* albedo,
                        const float* normal, float* out, void* stream) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    for (const float* p : {color, albedo, normal, const_cast<const float*>(out)})
      if (!p || (reinterpret_cast<uintptr_t>(p) & 15u)) throw Invalid("device images must be 16-byte aligned");
    denoise_device(*h->d, width, height, reinterpret_cast<const float4*>(color),
                   reinterpret_cast<const float4*>(albedo), reinterpret_cast<const float4*>(normal),
                   reinterpret_cast<float4*>(out), static_cast<cudaStream_t>(stream));
  });
}

int pfxt_denoise_trace(pfxt_denoiser* h, pfxt_trace* t, float* out) {
  return guarded([&]() {
    if (!h || !t || !out) throw Invalid("null argument");
    if (reinterpret_cast<uintptr_t>(out) & 15u) throw Invalid("device images must be 16-byte aligned");
    check(cudaSetDevice(t->device), "trace device");
    denoise_device(*h->d, t->width, t->height, reinterpret_cast<const float4*>(t->d_color),
                   reinterpret_cast<const float4*>(t->d_albedo), reinterpret_cast<const float4*>(t->d_normal),
                   reinterpret_cast<float4*>(out), t->stream);
  });
}

int pfxt_denoiser_tiles(pfxt_denoiser* h, uint32_t* tile_w, uint32_t* tile_h, uint32_t* count) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    const Denoiser& d = *h->d;
    if (tile_w) *tile_w = d.width ? d.plan.tile_w : 0u;
    if (tile_h) *tile_h = d.width ? d.plan.tile_h : 0u;
    if (count) *count = d.width ? (uint32_t)d.plan.tiles.size() : 0u;
  });
}

int pfxt_denoiser_last(pfxt_denoiser* h, float* ms, uint64_t* macs) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    float m = denoiser_finish(*h->d);
    if (ms) *ms = m;
    if (macs) *macs = h->d->last_macs;
  });
}

int pfxt_denoiser_set_max_tile_pixels(pfxt_denoiser* h, uint64_t pixels) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    if (pixels < 16u * 16u) throw Invalid("a tile holds at least 16 x 16 pixels");
    h->d->max_tile_pixels = pixels;
    h->d->width = h->d->height = 0;  // the next denoise plans again
  });
}

// The tile split of a height x width image (test hook): up to `capacity`
// tiles as 12 words each (src, dst, size, out_src, out_dst, out_size as (y, x)),
// then tile_h, tile_w, overlap and the count in `head`.
int pfxt_debug_denoise_plan(uint32_t height, uint32_t width, uint64_t max_tile_pixels, uint32_t* tiles,
                            uint32_t capacity, uint32_t* head) {
  return guarded([&]() {
    if (!head || (capacity && !tiles)) throw Invalid("null argument");
    if (width == 0 || height == 0) throw Invalid("image dimensions must be nonzero");
    DenoisePlan p = denoise_plan(height, width, max_tile_pixels);
    head[0] = p.tile_h;
    head[1] = p.tile_w;
    head[2] = p.overlap;
    head[3] = (uint32_t)p.tiles.size();
    for (size_t i = 0; i < p.tiles.size() && i < capacity; ++i) {
      const DenoiseTile& t = p.tiles[i];
      const uint32_t* parts[6] = {t.src, t.dst, t.size, t.out_src, t.out_dst, t.out_size};
      for (int k = 0; k < 6; ++k) {
        tiles[12 * i + 2 * k] = parts[k][0];
        tiles[12 * i + 2 * k + 1] = parts[k][1];
      }
    }
  });
}

// The conv CTA shape of the layers of up to 64 output channels (test and
// measurement hook): 0 the default, 1-9 a shape of denoise.cu's list, run by
// every layer whose outputs fit it.
int pfxt_debug_denoiser_shape(pfxt_denoiser* h, uint32_t shape) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    if (shape > 9u) throw Invalid("conv shape must be 0-9");
    h->d->conv_shape = shape;
    h->d->width = h->d->height = 0;  // the next denoise prepares its launches again
  });
}

int pfxt_denoiser_set_wait_limit(pfxt_denoiser* h, uint32_t polls) {
  return guarded([&]() {
    if (!h) throw Invalid("null argument");
    h->d->wait_limit = polls;
  });
}

}  // extern "C"
