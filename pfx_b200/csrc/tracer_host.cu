// Host side of the tracer handle: uploads (Trace::new_detailed, gpu.rs:1926),
// camera/lens/window updates (gpu.rs:2817-2890), readback (gpu.rs:3240) and
// sample counts (adaptive.rs:328).
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cache.h"
#include "tracer.h"

namespace pfxt {

namespace {

void check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) throw Refused(std::string(what) + ": out of device memory");
  throw DeviceError(std::string(what) + ": " + cudaGetErrorString(e));
}

void* dev_copy(pfxt_trace& t, const void* host, size_t bytes, const char* what) {
  size_t n = bytes ? bytes : 16;
  void* d = nullptr;
  check(cudaMalloc(&d, n), what);
  t.owned.push_back(d);
  if (host && bytes)
    check(cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice), what);
  else
    check(cudaMemset(d, 0, n), what);
  return d;
}

template <typename T>
T* dev_alloc(pfxt_trace& t, size_t count, const char* what) {
  return static_cast<T*>(dev_copy(t, nullptr, count * sizeof(T), what));
}

bool finite3(const float* p) { return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]); }

}  // namespace

uint64_t fnv(uint64_t h, const void* data, size_t bytes);
uint64_t tune_key_of(const pfxt_buffers& b, const Specialise& spec, uint32_t width, uint32_t height);

void trace_init(pfxt_trace& t, const pfxt_buffers& b, const pfxt_scene& view, const pfxt_settings& s, uint32_t width,
                uint32_t height) {
  check(cudaGetDevice(&t.device), "cudaGetDevice");
  check(cudaStreamCreateWithFlags(&t.stream, cudaStreamNonBlocking), "stream");
  t.width = width;
  t.height = height;
  t.samples = 0;
  if (s.sampler == PFXT_SAMPLER_SOBOL && (!b.sobol || b.sobol_length < 256 || b.sobol_length > 8192 ||
                                          (b.sobol_length & (b.sobol_length - 1)) != 0))
    throw Invalid("the Sobol sampler needs its table (256 patterns x a power-of-two length in [256, 8192])");
  for (int i = 0; i < 4; ++i)
    if (s.bounces[i] > 64) throw Invalid("bounces above 64");
  if (!finite3(view.camera.origin) || !finite3(view.camera.forward) || !finite3(view.camera.right) ||
      !finite3(view.camera.up))
    throw Invalid("camera contains invalid parameters");
  if (b.sky_width == 0 || b.sky_height == 0 || !b.sky_rows || !b.sky_columns) throw Invalid("invalid sky");

  // ---- traversal layout
  TraversalLayout layout = make_layout(b);
  t.d_wide = static_cast<WideNode*>(dev_copy(t, layout.wide.data(), layout.wide.size() * sizeof(WideNode), "nodes"));
  t.d_tris = static_cast<TravTri*>(dev_copy(t, layout.tris.data(), layout.tris.size() * sizeof(TravTri), "triangles"));
  t.d_insts =
      static_cast<InstRec*>(dev_copy(t, layout.insts.data(), layout.insts.size() * sizeof(InstRec), "instances"));
  t.view.wide = t.d_wide;
  t.view.tris = t.d_tris;
  t.view.insts = t.d_insts;
  t.view.root = layout.root;
  t.view.small = layout.small ? 1u : 0u;
  if (b.nodes_bytes >= sizeof(GpuNode)) {
    const GpuNode* root = static_cast<const GpuNode*>(b.nodes);
    for (int k = 0; k < 3; ++k) {
      t.bounds_lo[k] = root->lo[k];
      t.bounds_hi[k] = root->hi[k];
    }
  }

  // ---- shading buffers (reference layouts)
  t.d_triangles = dev_copy(t, b.triangles, b.triangles_bytes, "triangle records");
  t.d_uv = dev_copy(t, b.uv, b.uv_bytes, "uv");
  t.d_materials = dev_copy(t, b.materials, b.materials_bytes, "materials");
  t.d_surfaces = dev_copy(t, b.surfaces, b.surfaces_bytes, "surfaces");
  t.d_emitters = dev_copy(t, b.emitters, b.emitters_bytes, "emitters");
  t.d_emitter_cdf = dev_copy(t, b.emitter_cdf, b.emitter_cdf_bytes, "emitter cdf");
  t.surfaces_bytes = b.surfaces_bytes;
  t.emitters_bytes = b.emitters_bytes;
  t.emitter_cdf_bytes = b.emitter_cdf_bytes;
  t.d_lights = dev_copy(t, b.lights, b.lights_bytes, "lights");
  t.d_sky_rows = dev_copy(t, b.sky_rows, (size_t)b.sky_height * 4, "sky rows");
  t.d_sky_columns = dev_copy(t, b.sky_columns, (size_t)b.sky_width * b.sky_height * 4, "sky columns");
  if (s.sampler == PFXT_SAMPLER_SOBOL)
    t.d_sobol = dev_copy(t, b.sobol, (size_t)b.sobol_length * 256 * 16, "sobol table");
  const GpuEmitter* head = static_cast<const GpuEmitter*>(b.emitters);
  ShadeView& v = t.shade;
  v.triangles = static_cast<const GpuTriangle*>(t.d_triangles);
  v.uv = static_cast<const float4*>(t.d_uv);
  v.materials = static_cast<const float4*>(t.d_materials);
  v.surfaces = static_cast<const GpuSurface*>(t.d_surfaces);
  v.emitters = static_cast<const GpuEmitter*>(t.d_emitters);
  v.emitter_cdf = static_cast<const float*>(t.d_emitter_cdf);
  v.lights = static_cast<const GpuLight*>(t.d_lights);
  v.sky_rows = static_cast<const float*>(t.d_sky_rows);
  v.sky_columns = static_cast<const float*>(t.d_sky_columns);
  v.sobol = static_cast<const float4*>(t.d_sobol);
  v.sky_width = b.sky_width;
  v.sky_height = b.sky_height;
  memcpy(v.sky_radiance, b.sky_radiance, sizeof(v.sky_radiance));
  v.sky_sun_probability = b.sky_sun_probability;
  v.material_count = (uint32_t)(b.materials_bytes / sizeof(GpuHot)) - 1u;
  v.emitter_count = f2u(head->a[0]);
  v.looped = f2u(head->a[1]);
  v.tree = f2u(head->a[3]);
  t.light_rows = (uint32_t)(b.lights_bytes / sizeof(GpuLight));
  if (v.looped > t.light_rows || (v.tree > 0u && v.looped + v.tree >= t.light_rows))
    throw Invalid("the emitter header does not match the light rows");
  // Every index a shading kernel reads must stay inside its buffer.
  {
    uint32_t emitter_rows = (uint32_t)(b.emitters_bytes / sizeof(GpuEmitter));
    if (v.emitter_count + 1u > emitter_rows || b.emitter_cdf_bytes / 4 < v.emitter_count)
      throw Invalid("the emitter list is shorter than its header");
    uint32_t surfaces = (uint32_t)(b.surfaces_bytes / sizeof(GpuSurface));
    const GpuSurface* sf = static_cast<const GpuSurface*>(b.surfaces);
    for (uint32_t r = 0; r < surfaces; ++r)
      if (sf[r].info[1] != NO_MATERIAL && sf[r].info[1] >= v.material_count)
        throw Invalid("an instance record names a missing material");
    const GpuTriangle* tr = static_cast<const GpuTriangle*>(b.triangles);
    size_t tris = b.triangles_bytes / sizeof(GpuTriangle);
    for (size_t i = 0; i < tris; ++i) {
      if (!(tr[i].a[3] >= 0.0f) || f2u(tr[i].a[3]) >= v.material_count)
        throw Invalid("a triangle names a missing material");
      if (!(tr[i].c[3] >= 0.0f) || f2u(tr[i].c[3]) > v.emitter_count)
        throw Invalid("a triangle names a missing emitter");
    }
    const GpuEmitter* em = static_cast<const GpuEmitter*>(b.emitters);
    for (uint32_t e = 1; e <= v.emitter_count; ++e)
      if (f2u(em[e].b[3]) >= surfaces) throw Invalid("an emitter names a missing instance record");
    const GpuLight* lr = static_cast<const GpuLight*>(b.lights);
    uint32_t lights_end = v.looped + v.tree;
    if (v.tree > 0u) {
      for (uint32_t r = lights_end; r < t.light_rows; ++r) {
        uint32_t count = f2u(lr[r].d[1]), link = f2u(lr[r].d[2]);
        if (count > 0u) {
          if (count > 32u || link < v.looped || link + count > lights_end) throw Invalid("a light-tree leaf is malformed");
        } else if (link >= t.light_rows || r + 1u >= t.light_rows) {
          throw Invalid("a light-tree link is out of range");
        } else {
          // a child row with count 1 names its light directly (child_importance)
          const uint32_t kids[2] = {r + 1u, link};
          for (uint32_t k : kids)
            if (f2u(lr[k].d[1]) == 1u && f2u(lr[k].d[2]) >= lights_end) throw Invalid("a light-tree leaf is malformed");
        }
      }
    }
  }
  for (uint32_t m = 0; m < v.material_count; ++m) {
    const GpuHot& h = static_cast<const GpuHot*>(b.materials)[m + 1];
    if (h.thick_sub_film[2] > 0.0f && h.emission_film[3] > 0.0f)
      throw Invalid("thin-film materials are outside this tracer's scope");
    if (f2bits(h.extension[1]) != 0u) throw Invalid("material extension rows are outside this tracer's scope");
  }

  // ---- films: 48 B accumulation + three RGBA32F films per pixel
  size_t pixels = (size_t)width * height;
  t.d_accum = dev_alloc<Accum>(t, pixels, "accumulation");
  t.d_color = dev_alloc<float4>(t, pixels, "colour film");
  t.d_albedo = dev_alloc<float4>(t, pixels, "albedo film");
  t.d_normal = dev_alloc<float4>(t, pixels, "normal film");
  t.d_snaps = dev_alloc<float4>(t, pixels * 2, "adaptive snapshots");
  t.d_running = dev_alloc<uint32_t>(t, 4, "adaptive count");
  t.d_error = dev_alloc<uint32_t>(t, 4, "error word");
  t.d_counters = dev_alloc<uint32_t>(t, 64, "work counters");

  // ---- base frame (gpu.rs:2295-2316)
  FrameParams& f = t.base;
  memset(&f, 0, sizeof(f));
  f.size[0] = width;
  f.size[1] = height;
  f.counts[0] = b.triangle_count;
  f.counts[1] = 0;
  for (int k = 0; k < 3; ++k) {
    f.origin[k] = view.camera.origin[k];
    f.forward[k] = view.camera.forward[k];
    f.right[k] = view.camera.right[k];
    f.up[k] = view.camera.up[k];
    f.sun_dir[k] = view.sun.direction[k];
    f.sun_color[k] = view.sun.color[k];
  }
  f.sun_color[3] = view.sun.intensity;
  for (int k = 0; k < 4; ++k) f.lens[k] = s.lens[k];
  f.lens[2] = s.lens[2] * 0.5f;  // aperture * 0.5
  f.window[0] = width;
  f.window[1] = height;
  // Projection::place (gpu.rs:206-216)
  t.projection = s.projection;
  if (s.projection == PFXT_PROJECTION_ORTHOGRAPHIC) {
    if (!(s.ortho[0] > 0.0f) || !(s.ortho[1] > 0.0f)) throw Invalid("invalid projection");
    f.origin[3] = 1.0f;
    f.right[3] = s.ortho[0] * 0.5f;
    f.up[3] = s.ortho[1] * 0.5f;
  } else if (s.projection == PFXT_PROJECTION_EQUIRECT) {
    f.origin[3] = 2.0f;
  }
  // base.sun_dir[3] = sun_radius_deg.to_radians().cos()
  f.sun_dir[3] = std::cos(view.sun.radius_deg * (PFXT_PI_F / 180.0f));

  Specialise& sp = t.spec;
  sp.total_bounces = s.bounces[0];
  sp.diffuse_bounces = s.bounces[1];
  sp.glossy_bounces = s.bounces[2];
  sp.transmission_bounces = s.bounces[3];
  sp.sobol = s.sampler == PFXT_SAMPLER_SOBOL ? 1u : 0u;
  sp.sobol_length = sp.sobol ? b.sobol_length : 256u;
  sp.clamp_indirect = s.clamp_indirect;
  sp.filter_glossy = s.filter_glossy;
  t.tune_key = tune_key_of(b, sp, width, height);

  light_trig_init(t);
}

void trace_release(pfxt_trace& t) {
  if (t.device >= 0) cudaSetDevice(t.device);
  if (t.stream) cudaStreamSynchronize(t.stream);
  for (void* p : t.owned) cudaFree(p);
  t.owned.clear();
  if (t.d_wave) cudaFree(t.d_wave);
  t.d_wave = nullptr;
  if (t.d_stage) cudaFree(t.d_stage);
  t.d_stage = nullptr;
  if (t.d_cache_scratch) cudaFree(t.d_cache_scratch);
  t.d_cache_scratch = nullptr;
  t.cache = nullptr;
  trace_forget_graphs(t);
  if (t.d_vars) cudaFree(t.d_vars);
  if (t.h_vars) cudaFreeHost(t.h_vars);
  t.d_vars = nullptr;
  t.h_vars = nullptr;
  if (t.side) {
    cudaStreamSynchronize(t.side);
    cudaStreamDestroy(t.side);
  }
  if (t.fork_ev) cudaEventDestroy(t.fork_ev);
  if (t.join_ev) cudaEventDestroy(t.join_ev);
  t.side = nullptr;
  t.fork_ev = t.join_ev = nullptr;
  if (t.ahead) {
    cudaStreamSynchronize(t.ahead);
    cudaStreamDestroy(t.ahead);
  }
  if (t.ahead_fork) cudaEventDestroy(t.ahead_fork);
  if (t.ahead_join) cudaEventDestroy(t.ahead_join);
  t.ahead = nullptr;
  t.ahead_fork = t.ahead_join = nullptr;
  if (t.stream) cudaStreamDestroy(t.stream);
  t.stream = nullptr;
}

void trace_set_camera(pfxt_trace& t, const pfxt_camera& c) {
  if (!finite3(c.origin) || !finite3(c.forward) || !finite3(c.right) || !finite3(c.up))
    throw Invalid("camera contains invalid parameters");
  if (t.projection != PFXT_PROJECTION_PERSPECTIVE) {
    const float* axes[] = {c.forward, c.right, c.up};
    for (auto a : axes)
      if (!(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] > 1e-12f))
        throw Invalid("an orthographic or equirect camera needs forward, right and up");
  }
  for (int k = 0; k < 3; ++k) {
    t.base.origin[k] = c.origin[k];
    t.base.forward[k] = c.forward[k];
    t.base.right[k] = c.right[k];
    t.base.up[k] = c.up[k];
  }
  t.samples = 0;
}

void trace_move_scene(pfxt_trace& t, const pfxt_buffers& b) {
  if (b.surfaces_bytes != t.surfaces_bytes || b.emitters_bytes != t.emitters_bytes ||
      b.emitter_cdf_bytes != t.emitter_cdf_bytes || b.nodes_bytes < sizeof(GpuNode))
    throw Invalid("the moved scene does not match the trace's buffers");
  // The same index checks as at creation for what is uploaded again (the
  // traversal layout checks the nodes and instance records itself).
  {
    const GpuSurface* sf = static_cast<const GpuSurface*>(b.surfaces);
    const uint32_t surfaces = (uint32_t)(b.surfaces_bytes / sizeof(GpuSurface));
    for (uint32_t r = 0; r < surfaces; ++r)
      if (sf[r].info[1] != NO_MATERIAL && sf[r].info[1] >= t.shade.material_count)
        throw Invalid("an instance record names a missing material");
    const GpuEmitter* em = static_cast<const GpuEmitter*>(b.emitters);
    if (f2u(em[0].a[0]) != t.shade.emitter_count || f2u(em[0].a[1]) != t.shade.looped ||
        f2u(em[0].a[3]) != t.shade.tree)
      throw Invalid("the moved emitter list does not match the trace's");
    for (uint32_t e = 1; e <= t.shade.emitter_count; ++e)
      if (f2u(em[e].b[3]) >= surfaces) throw Invalid("an emitter names a missing instance record");
  }
  TraversalLayout layout = make_layout(b);
  check(cudaStreamSynchronize(t.stream), "move instances");
  // New traversal buffers first, so that a failed allocation leaves the trace as it was.
  size_t kept = t.owned.size();
  void* fresh[3] = {nullptr, nullptr, nullptr};
  try {
    fresh[0] = dev_copy(t, layout.wide.data(), layout.wide.size() * sizeof(WideNode), "nodes");
    fresh[1] = dev_copy(t, layout.tris.data(), layout.tris.size() * sizeof(TravTri), "triangles");
    fresh[2] = dev_copy(t, layout.insts.data(), layout.insts.size() * sizeof(InstRec), "instances");
  } catch (...) {
    for (size_t i = kept; i < t.owned.size(); ++i) cudaFree(t.owned[i]);
    t.owned.resize(kept);
    throw;
  }
  void* stale[3] = {t.d_wide, t.d_tris, t.d_insts};
  for (void* p : stale) {
    auto it = std::find(t.owned.begin(), t.owned.end(), p);
    if (it != t.owned.end()) {
      t.owned.erase(it);
      cudaFree(p);
    }
  }
  t.d_wide = static_cast<WideNode*>(fresh[0]);
  t.d_tris = static_cast<TravTri*>(fresh[1]);
  t.d_insts = static_cast<InstRec*>(fresh[2]);
  t.view.wide = t.d_wide;
  t.view.tris = t.d_tris;
  t.view.insts = t.d_insts;
  t.view.root = layout.root;
  t.view.small = layout.small ? 1u : 0u;
  check(cudaMemcpy(t.d_surfaces, b.surfaces, b.surfaces_bytes, cudaMemcpyHostToDevice), "surfaces");
  check(cudaMemcpy(t.d_emitters, b.emitters, b.emitters_bytes, cudaMemcpyHostToDevice), "emitters");
  if (b.emitter_cdf_bytes)
    check(cudaMemcpy(t.d_emitter_cdf, b.emitter_cdf, b.emitter_cdf_bytes, cudaMemcpyHostToDevice), "emitter cdf");
  const GpuNode* root = static_cast<const GpuNode*>(b.nodes);
  for (int k = 0; k < 3; ++k) {
    t.bounds_lo[k] = root->lo[k];
    t.bounds_hi[k] = root->hi[k];
  }
  trace_forget_graphs(t);
  t.samples = 0;
}

void trace_set_lens(pfxt_trace& t, const float lens[4]) {
  for (int k = 0; k < 4; ++k)
    if (!std::isfinite(lens[k])) throw Invalid("invalid lens");
  if (lens[2] < 0.0f || lens[3] <= 0.0f) throw Invalid("invalid lens");
  t.base.lens[0] = lens[0];
  t.base.lens[1] = lens[1];
  t.base.lens[2] = lens[2] * 0.5f;
  t.base.lens[3] = lens[3];
  t.samples = 0;
}

void trace_set_window(pfxt_trace& t, const uint32_t full[2], const uint32_t origin[2]) {
  auto fits = [&](int k, uint32_t side) {
    uint64_t end = (uint64_t)origin[k] + side;
    return end <= full[k];
  };
  if (!fits(0, t.width) || !fits(1, t.height)) throw Invalid("the window must lie inside the full frame");
  if ((uint64_t)full[0] * full[1] > 0xffffffffull) throw Invalid("the full frame is too large");
  t.base.window[0] = full[0];
  t.base.window[1] = full[1];
  t.base.window[2] = origin[0];
  t.base.window[3] = origin[1];
  t.samples = 0;
}

void trace_readback(pfxt_trace& t, float* color, float* albedo, float* normal) {
  size_t bytes = (size_t)t.width * t.height * 16;
  check(cudaStreamSynchronize(t.stream), "readback");
  if (color) check(cudaMemcpy(color, t.d_color, bytes, cudaMemcpyDeviceToHost), "colour readback");
  if (albedo) check(cudaMemcpy(albedo, t.d_albedo, bytes, cudaMemcpyDeviceToHost), "albedo readback");
  if (normal) check(cudaMemcpy(normal, t.d_normal, bytes, cudaMemcpyDeviceToHost), "normal readback");
}

void trace_read_accum(pfxt_trace& t, float* accum) {
  check(cudaStreamSynchronize(t.stream), "readback");
  check(cudaMemcpy(accum, t.d_accum, (size_t)t.width * t.height * sizeof(Accum), cudaMemcpyDeviceToHost),
        "accumulation readback");
}

void trace_sample_counts(pfxt_trace& t, uint32_t* counts) {
  size_t pixels = (size_t)t.width * t.height;
  std::vector<float> accum(pixels * 12);
  trace_read_accum(t, accum.data());
  for (size_t i = 0; i < pixels; ++i) counts[i] = (uint32_t)std::fabs(accum[i * 12 + 3]);
}

// Adaptive::rounds (adaptive.rs:46-63).
bool adaptive_valid(const pfxt_adaptive& a) {  // Adaptive::valid (adaptive.rs:28-33)
  return std::isfinite(a.threshold) && a.threshold > 0.0f && a.min_samples >= 2u && a.max_samples >= a.min_samples &&
         std::isfinite(a.growth) && a.growth > 1.0f;
}

std::vector<uint32_t> adaptive_rounds(const pfxt_adaptive& a) {
  std::vector<uint32_t> rounds{std::max(a.min_samples / 2u, 1u)};
  for (;;) {
    uint32_t last = rounds.back();
    if (last >= a.max_samples) return rounds;
    float grown = std::ceil((float)last * a.growth);
    uint32_t next = f2u(grown);
    next = std::max(next, last + 1u);
    next = std::max(next, rounds.size() == 1 ? a.min_samples : 0u);
    next = std::min(next, a.max_samples);
    rounds.push_back(next);
  }
}

// Trace::set_projection (gpu.rs:2872-2890) with Projection::valid, fits and
// place (gpu.rs:191-218).
void trace_set_projection(pfxt_trace& t, uint32_t projection, const float ortho[2]) {
  if (projection > PFXT_PROJECTION_EQUIRECT) throw Invalid("invalid projection");
  if (projection == PFXT_PROJECTION_ORTHOGRAPHIC &&
      (!ortho || !std::isfinite(ortho[0]) || !std::isfinite(ortho[1]) || !(ortho[0] > 0.0f) || !(ortho[1] > 0.0f)))
    throw Invalid("invalid projection");
  if (projection != PFXT_PROJECTION_PERSPECTIVE) {
    const float* axes[] = {t.base.forward, t.base.right, t.base.up};
    for (auto a : axes)
      if (!(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] > 1e-12f))
        throw Invalid("an orthographic or equirect camera needs forward, right and up");
  }
  float kind = 0.0f, half_width = 0.0f, half_height = 0.0f;
  if (projection == PFXT_PROJECTION_ORTHOGRAPHIC) {
    kind = 1.0f;
    half_width = ortho[0] * 0.5f;
    half_height = ortho[1] * 0.5f;
  } else if (projection == PFXT_PROJECTION_EQUIRECT) {
    kind = 2.0f;
  }
  t.base.origin[3] = kind;
  t.base.right[3] = half_width;
  t.base.up[3] = half_height;
  t.projection = projection;
  t.samples = 0;
}

// ------------------------------------------------------------------ tuning
void trace_set_tuning(pfxt_trace& t, const pfxt_tuning& k) {
  if (k.trace_threads != 64u && k.trace_threads != 128u && k.trace_threads != 256u)
    throw Invalid("trace_threads must be 64, 128 or 256");
  if (k.short_stack != 0u && k.short_stack != 8u) throw Invalid("short_stack must be 0 or 8");
  t.trace_threads = k.trace_threads;
  t.sort_shading = k.sort_shading != 0u;
  t.use_graphs = k.graphs != 0u;
  t.split_shade = k.split_shade != 0u;
  t.sort_rays = k.sort_rays != 0u;
  t.shadow_queue = k.shadow_queue != 0u;
  t.short_stack = k.short_stack;
  t.slot_kernels = k.slot_kernels != 0u;
}

pfxt_tuning trace_get_tuning(const pfxt_trace& t) {
  pfxt_tuning k{};
  k.trace_threads = t.trace_threads;
  k.sort_shading = t.sort_shading ? 1u : 0u;
  k.graphs = t.use_graphs ? 1u : 0u;
  k.split_shade = t.split_shade ? 1u : 0u;
  k.sort_rays = t.sort_rays ? 1u : 0u;
  k.pass_ms = t.tuned_pass_ms;
  k.shadow_queue = t.shadow_queue ? 1u : 0u;
  k.short_stack = t.short_stack;
  k.from_cache = 0u;
  k.slot_kernels = t.slot_kernels ? 1u : 0u;
  return k;
}

// FNV-1a style mixing of 8-byte words (and the bytes left over), continuing
// from `h`: a fingerprint, not a format.
uint64_t fnv(uint64_t h, const void* data, size_t bytes) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  size_t words = bytes / 8;
  for (size_t i = 0; i < words; ++i) {
    uint64_t w;
    memcpy(&w, p + 8 * i, 8);
    h = (h ^ w) * 0x100000001b3ull;
  }
  for (size_t i = 8 * words; i < bytes; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
  return h;
}

// The tuning key of a tracer: its scene's nodes, triangles, lights and
// materials, its film and specialisation (set at creation; the attached cache's
// settings are added when tuning).
uint64_t tune_key_of(const pfxt_buffers& b, const Specialise& spec, uint32_t width, uint32_t height) {
  uint64_t h = 0xcbf29ce484222325ull;
  h = fnv(h, b.nodes, b.nodes_bytes);
  h = fnv(h, b.triangles, b.triangles_bytes);
  h = fnv(h, b.lights, b.lights_bytes);
  h = fnv(h, b.materials, b.materials_bytes);
  h = fnv(h, &spec, sizeof(spec));
  uint32_t film[2] = {width, height};
  return fnv(h, film, sizeof(film));
}

// Median device time of `passes - 1` one-sample passes after one warm-up pass.
static float time_passes(pfxt_trace& t, uint32_t passes, uint32_t& seed) {
  cudaEvent_t e0, e1;
  check(cudaEventCreate(&e0), "autotune events");
  check(cudaEventCreate(&e1), "autotune events");
  std::vector<float> ms;
  for (uint32_t i = 0; i < passes; ++i) {
    check(cudaEventRecord(e0, t.stream), "autotune events");
    trace_sample(t, 1u, seed++);
    check(cudaEventRecord(e1, t.stream), "autotune events");
    check(cudaEventSynchronize(e1), "autotune events");
    float v = 0.0f;
    check(cudaEventElapsedTime(&v, e0, e1), "autotune events");
    if (i > 0) ms.push_back(v);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::sort(ms.begin(), ms.end());
  return ms[ms.size() / 2];
}

// Choices of earlier tunings in this process, by tuning key.
std::mutex g_tuned_lock;
std::map<uint64_t, pfxt_tuning> g_tuned;

pfxt_tuning trace_autotune(pfxt_trace& t, uint32_t passes) {
  if (passes < 2 || passes > 64) throw Invalid("autotune: passes must be in 2..64");
  uint64_t key = t.tune_key;
  if (t.cache) key = fnv(fnv(key, "cache", 5), &t.cache->s, sizeof(t.cache->s));
  {
    std::lock_guard<std::mutex> hold(g_tuned_lock);
    auto found = g_tuned.find(key);
    if (found != g_tuned.end()) {
      pfxt_tuning k = found->second;
      k.graphs = t.use_graphs ? 1u : 0u;
      trace_set_tuning(t, k);
      t.tuned_pass_ms = k.pass_ms;
      t.samples = 0;
      k.from_cache = 1u;
      return k;
    }
  }
  // one choice at a time, the others held at the best so far
  pfxt_tuning best = trace_get_tuning(t);
  uint32_t seed = 0x7e000000u;
  trace_set_tuning(t, best);
  best.pass_ms = time_passes(t, passes, seed);
  auto consider = [&](pfxt_tuning k) {
    trace_set_tuning(t, k);
    k.pass_ms = time_passes(t, passes, seed);
    if (k.pass_ms < best.pass_ms) best = k;
  };
  for (uint32_t threads : {64u, 128u, 256u})
    if (threads != best.trace_threads) {
      pfxt_tuning k = best;
      k.trace_threads = threads;
      consider(k);
    }
  for (int knob = 0; knob < 6; ++knob) {
    pfxt_tuning k = best;
    switch (knob) {
      case 0: k.sort_shading ^= 1u; break;
      case 1: k.split_shade ^= 1u; break;
      case 2: k.sort_rays ^= 1u; break;
      case 3: k.shadow_queue ^= 1u; break;
      case 4: k.slot_kernels ^= 1u; break;
      default: k.short_stack = k.short_stack ? 0u : 8u; break;
    }
    consider(k);
  }
  trace_set_tuning(t, best);
  t.tuned_pass_ms = best.pass_ms;
  t.samples = 0;  // the trial passes are not part of the image
  best.from_cache = 0u;
  {
    std::lock_guard<std::mutex> hold(g_tuned_lock);
    g_tuned[key] = best;
  }
  return best;
}

}  // namespace pfxt
