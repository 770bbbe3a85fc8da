// The wavefront path tracer: Trace::sample (crates/trace/src/gpu.rs:2942) as a
// sequence of kernels over path queues instead of the reference's megakernel
// main() (trace.wgsl:2503-2579).
//
// One wave traces one sample for every active pixel.  Per bounce:
//   extend   closest hit of every queued path (persistent traversal kernel)
//   shade    the body of radiance()'s bounce loop (trace.wgsl:2169-2500):
//            emission, light selection and BSDF sampling; writes up to `cap`
//            shadow-ray slots per path, appends occlusion queries to the shadow
//            queue and surviving paths to the next ray queue (warp-aggregated
//            atomics, so both queues stay compact)
//   connect  any hit of every queued shadow ray (persistent traversal kernel)
// The light-loop contributions of a bounce are added to the path's result at
// the start of the path's next shade (or in finish), in light-slot order, so
// the result is summed in exactly the reference's order; with the draws of
// the reference's random sequence kept in order, a pixel's value equals the
// reference's bit for bit.  Waves run in sample order, so the accumulation of
// samples into the 48 B/pixel Accum also keeps the reference's order.
//
// Zero-valued light-slot contributions (a black sky, a light behind the
// surface) add nothing and trace no shadow ray; their random draws are still
// taken.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cache.h"
#include "kernels.h"
#include "shade.cuh"
#include "tracer.h"
#include "traverse.cuh"

namespace pfxt {

namespace {

constexpr int kThreads = 128;
// Resident blocks of the shade kernel per SM the compiler must allow for: it
// sets the register budget (4: 128 registers, 2: up to 255).
#ifndef SHADE_MIN_BLOCKS
#define SHADE_MIN_BLOCKS 4
#endif
// The light-slot kernel waits on dependent loads (light-tree rows, Sobol table)
// more than it computes, so it runs at 12 blocks per SM (40 registers and some
// spill) rather than at its natural 128 registers: 4K plain pass 141.0 ms at 4
// blocks, 137.4 at 6, 134.9 at 8, 131.4 at 10, 131.0 at 12.
#ifndef SHADE_LIGHTS_MIN_BLOCKS
#define SHADE_LIGHTS_MIN_BLOCKS 12
#endif
constexpr uint32_t CAP_MAX = 8u;
// Pass variables in device memory: samples so far, samples this pass, seed, 0,
// then the camera's origin, forward, right and up as four float4.
constexpr size_t PASS_VAR_BYTES = 16 + 64;

// Path flag word (ray_d.w bits).
constexpr uint32_t F_CARRIED = 0x3u;  // bits 0-1
constexpr int F_LOBE0 = 2, F_LOBE1 = 9, F_LOBE2 = 16;  // 7 bits each
constexpr uint32_t F_LAST = 1u << 23, F_THROUGH = 1u << 24, F_LIT = 1u << 25, F_DIFFUSED = 1u << 26;
constexpr int F_PEND = 27;  // 4 bits: pending light-slot contributions
constexpr uint32_t F_CACHED = 1u << 31;  // the path ended into the radiance cache

struct Wave {
  float4* ray_o;   // o.xyz, previous pdf
  float4* ray_d;   // d.xyz, flag word
  float4* thr;     // throughput.xyz, pcg state
  float4* res;     // result.xyz, pixel index
  float4* alb;     // first albedo
  float4* nrm;     // first normal
  float4* hit;     // t, slot, record, u
  float* hit_v;    // v
  float4* sh_o;    // per slot: origin.xyz, limit
  float4* sh_d;    // per slot: direction.xyz, visible flag
  float4* sh_c;    // per slot: contribution.xyz
  uint32_t* queue[2];
  uint32_t* squeue;
  uint32_t* active;
  uint32_t* counters;  // 0,1: ray queues, 2: shadow queue, 3: active paths, 4: extend work counter,
                       // 16: connect work counter, 17: the connect's shadow-queue count (a copy of 2)
  // shade queue sorted by hit material (counting sort per bounce)
  uint32_t* keys;      // per queue entry: material key
  uint32_t* sorted;    // the queue, grouped by key
  uint32_t* hist;      // SORT_BINS: paths per key
  uint32_t* cursor;    // SORT_BINS: entries handed out per key
  // split shade: the paths that scatter this bounce (count at counters[12]) and their surfaces
  uint32_t* lit;
  float4* surf;        // 9 float4 per path
  uint32_t* rhist;     // RAY_BINS: the extend queue's histogram by ray key
  uint32_t* rcursor;
  // queue items the traversal handed over to the IEEE walk (rays that are not
  // bounded), counted at counters[13] (extend, in eretry) and counters[14]
  // (connect, in retry): the two kernels may run at the same time
  uint32_t* retry;
  uint32_t* eretry;
  // the light tree's pick of each path that scatters (row, pmf), by lit index
  float2* pick;
};

// The radiance cache as the wave sees it (all null/zero when none is attached).
struct CachePass {
  uint32_t enabled;
  uint32_t query_bounce;    // paths end into the cache at this vertex
  uint32_t record_bounces;  // training paths record vertices 0..record_bounces
  uint32_t threshold;       // a path trains when its 24-bit hash is below this
  uint32_t tcap, rcap;      // training-path slots, training records
  float min_roughness;      // smoother (or transmissive) vertices do not end paths; 0 = any
  uint32_t query_last;      // the last vertex a path may end into the cache at
  float4* query;            // 5 float4 per query (compact)
  uint32_t* cqueue;         // path index of each query
  float4* pred;             // per path: the cache's radiance
  uint32_t* tslot;          // per path: training slot (low 24 bits) | recorded-vertex mask << 24, ~0 = none
  float4* tvert;            // per slot and recorded vertex: 5 float4 query, throughput, result so far
  float4* records;          // 6 float4 per training record
  uint8_t* encoded;         // the queries' encoded inputs (cache_x_bytes)
  const uint8_t* cell_ok;   // fallback cells (NRC_CELLS^3)
  float lo[3], inv[3];      // grid bounds
};

struct Pass {
  FrameParams f;
  Specialise sp;
  ShadeView v;
  SceneView s;
  Wave w;
  CachePass c;
  uint32_t sample;     // sample index inside the pass
  uint32_t bounce;
  uint32_t cap;        // shadow slots per path
  uint32_t deferred;   // 1: light-slot shadow rays go through the shadow queue
  uint32_t light_rows;
  uint32_t slots;      // 2 + light_slots()
  uint32_t width, height;
  uint32_t bins;       // 2 x (material keys + 1 for misses); 0 = the shade queue is not sorted
  uint32_t ray_bins;   // RAY_BINS when the extend queue of bounces after the first is sorted by ray key, else 0
  float scene_lo[3], scene_inv[3];  // the scene box, for the ray key's origin cell
  // What changes from pass to pass lives in device memory, written by the
  // pass's first operation, so one captured pass replays for every pass:
  // [0] samples accumulated before the pass, [1] samples in it, [2] seed.
  const uint32_t* vars;
};

__device__ __forceinline__ uint32_t pass_accum(const Pass& P) { return __ldg(P.vars + 0); }
__device__ __forceinline__ uint32_t pass_count(const Pass& P) { return __ldg(P.vars + 1); }
__device__ __forceinline__ uint32_t pass_seed(const Pass& P) { return __ldg(P.vars + 2); }
// Camera origin, forward, right and up (xyz) of this pass, after the counters:
// outside the captured launch parameters, so a moving camera replays one graph.
__device__ __forceinline__ v3 pass_camera(const Pass& P, int k) {
  float4 c = __ldg(reinterpret_cast<const float4*>(P.vars) + 1 + k);
  return mk3(c.x, c.y, c.z);
}

// The fallback grid: may a path end into the cache at p?
__device__ __forceinline__ bool cell_ok(const CachePass& c, v3 p) {
  float q[3] = {p.x, p.y, p.z};
  uint32_t cell[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float u = (q[k] - c.lo[k]) * c.inv[k];
    u = u > 0.0f ? (u < 1.0f ? u : 1.0f) : 0.0f;
    cell[k] = min((uint32_t)(u * (float)NRC_CELLS), NRC_CELLS - 1u);
  }
  return c.cell_ok[(cell[2] * NRC_CELLS + cell[1]) * NRC_CELLS + cell[0]] != 0u;
}

__device__ __forceinline__ uint32_t lobe_count(uint32_t f, int shift) { return (f >> shift) & 127u; }

__device__ __forceinline__ v3 capped(const Pass& P, v3 value, bool deep) {
  float cap = P.sp.clamp_indirect;
  if (!(cap > 0.0f) || !deep) return value;
  float luma = dot3(value, mk3(0.2126f, 0.7152f, 0.0722f));
  if (!(luma > cap)) return value;
  return scl3(value, cap / luma);
}

// Warp-aggregated append to a queue.
__device__ __forceinline__ void append(uint32_t* queue, uint32_t* count, uint32_t value, bool want) {
  unsigned m = __ballot_sync(__activemask(), want);
  if (!want) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(m, base, leader);
  queue[base + (uint32_t)__popc(m & ((1u << lane) - 1u))] = value;
}

// Warp-aggregated claim of one index from `count`; ~0 for threads that do not want one.
__device__ __forceinline__ uint32_t claim(uint32_t* count, bool want) {
  unsigned m = __ballot_sync(__activemask(), want);
  if (!want) return ~0u;
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(m, base, leader);
  return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

// ------------------------------------------------------------------ active
// Pixels that still sample: the reference returns early when accum.color.w
// is negative (trace.wgsl:2517), the mark of a converged pixel.
__global__ void k_collect(const __grid_constant__ Pass P,const Accum* __restrict__ accum, const uint8_t* __restrict__ mask) {
  uint32_t n = P.width * P.height;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    bool live = (pass_accum(P) == 0u || !(accum[i].color.w < 0.0f)) && (mask == nullptr || mask[i] != 0);
    append(P.w.active, P.w.counters + 3, i, live);
  }
}

// ------------------------------------------------------------------ generate
// main() up to the call of radiance(): seeding, pixel filter, camera ray.
__global__ void k_gen(const __grid_constant__ Pass P) {
  const uint32_t n = P.w.counters[3];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t pixel = P.w.active[i];
    uint32_t gx = pixel % P.width, gy = pixel / P.width;
    uint32_t px = gx + P.f.window[2], py = gy + P.f.window[3];
    uint32_t stream = py * P.f.window[0] + px;
    const uint32_t seed = pass_seed(P);
    uint32_t absolute = pass_accum(P) + P.sample;
    uint32_t state = pcg(stream * 1973u + pcg(seed * 9277u + absolute * 7919u + 26699u));
    Rng r{hash_iqnt2d(px, py) ^ seed, absolute, 0u};
    float4 pf = sobol4(P.v, P.sp, r, 0u);
    float jx = rnd(P.sp, state, pf.x);
    float jy = rnd(P.sp, state, pf.y);
    float ndc_x = ((float)px + jx) / (float)P.f.window[0] * 2.0f - 1.0f;
    float ndc_y = ((float)py + jy) / (float)P.f.window[1] * 2.0f - 1.0f;
    uint32_t kind = f2u(rint_(P.f.origin[3]));
    v3 cam_o = pass_camera(P, 0), cam_f = pass_camera(P, 1), cam_r = pass_camera(P, 2), cam_u = pass_camera(P, 3);
    v3 direction = normalize3(add3(add3(cam_f, scl3(cam_r, ndc_x + P.f.lens[0])), scl3(cam_u, -ndc_y + P.f.lens[1])));
    v3 origin = cam_o;
    if (kind == 1u) {
      direction = normalize3(cam_f);
      origin = add3(origin, add3(scl3(normalize3(cam_r), (ndc_x + P.f.lens[0]) * P.f.right[3]),
                                 scl3(normalize3(cam_u), (-ndc_y + P.f.lens[1]) * P.f.up[3])));
    } else if (kind == 2u) {
      float phi = (ndc_x * 0.5f) * 2.0f * SH_PI;
      float theta = (ndc_y * 0.5f + 0.5f) * SH_PI;
      v3 local = mk3(sin_(theta) * sin_(phi), cos_(theta), -sin_(theta) * cos_(phi));
      direction = normalize3(sub3(add3(scl3(normalize3(cam_r), local.x), scl3(normalize3(cam_u), local.y)),
                                  scl3(normalize3(cam_f), local.z)));
    } else if (P.f.lens[2] > 0.0f) {
      v3 focus = add3(origin, scl3(direction, P.f.lens[3] / dot3(direction, normalize3(cam_f))));
      float4 ap = sobol4(P.v, P.sp, r, 1u);
      float radius = sqrtf(rnd(P.sp, state, ap.x)) * P.f.lens[2];
      float phi = 2.0f * SH_PI * rnd(P.sp, state, ap.y);
      origin = add3(origin, add3(scl3(normalize3(cam_r), radius * cos_(phi)), scl3(normalize3(cam_u), radius * sin_(phi))));
      direction = normalize3(sub3(focus, origin));
    }
    P.w.ray_o[i] = make_float4(origin.x, origin.y, origin.z, 0.0f);
    P.w.ray_d[i] = make_float4(direction.x, direction.y, direction.z, __uint_as_float(3u));  // carried = 3
    P.w.thr[i] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(state));
    P.w.res[i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(pixel));
    P.w.alb[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.w.nrm[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.w.queue[0][i] = i;
    if (P.c.enabled) {
      // training paths: a hash of the pixel and the sample, apart from the
      // sampler's own sequence, so the chosen paths draw exactly as the others
      uint32_t h = pcg(stream * 9781u + pcg(seed * 6529u + absolute * 3571u + 40503u));
      uint32_t slot = claim(P.w.counters + 6, (h >> 8) < P.c.threshold);
      P.c.tslot[i] = slot < P.c.tcap ? slot : ~0u;
    }
  }
}

// Before a sample's k_gen: no cache queries and no training slots yet.
__global__ void k_cache_begin(const __grid_constant__ Pass P) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.w.counters[5] = 0u;
    P.w.counters[6] = 0u;
  }
}

__global__ void k_seed_counts(const __grid_constant__ Pass P) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.w.counters[0] = P.w.counters[3];
    P.w.counters[1] = 0u;
    P.w.counters[2] = 0u;
  }
}

// Before a bounce: empty the next ray queue and the shadow queue, rewind the
// work counter of the extend kernel, and count the closest-hit queries of the
// bounce (64-bit totals at counters[8..9] closest, [10..11] any hit).
__global__ void k_reset(const __grid_constant__ Pass P,uint32_t cur) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.w.counters[cur ^ 1u] = 0u;
    P.w.counters[2] = 0u;
    P.w.counters[4] = 0u;
    P.w.counters[12] = 0u;
    P.w.counters[13] = 0u;
    reinterpret_cast<unsigned long long*>(P.w.counters + 8)[0] += P.w.counters[cur];
  }
  if (blockIdx.x == 0) {
    for (uint32_t b = threadIdx.x; b < P.bins; b += blockDim.x) {
      P.w.hist[b] = 0u;
      P.w.cursor[b] = 0u;
    }
    for (uint32_t b = threadIdx.x; b < P.ray_bins; b += blockDim.x) {
      P.w.rhist[b] = 0u;
      P.w.rcursor[b] = 0u;
    }
  }
}

// ------------------------------------------------------------------ sort
// The shade queue grouped by the material of each path's hit (misses last),
// so that the warps of the shade kernel run one BSDF's code; at the vertices
// where paths may end into the radiance cache, the paths that will continue
// are further grouped apart from those that will end.  A counting sort:
// block histograms into the global one, then every block reserves a range
// per key and places its entries with shared-memory atomics.  The order
// inside a key is arbitrary and the key only orders: the shade kernel makes
// every decision itself, so no result depends on it.
constexpr uint32_t SORT_BINS = 1024;

// Key 2 * material + (1 if the path continues past a cache vertex).
__device__ __forceinline__ uint32_t material_key(const Pass& P, uint32_t i) {
  float4 h = P.w.hit[i];
  if (h.x >= 1e19f) return P.bins - 2u;
  uint32_t surface = __float_as_uint(h.y), record = __float_as_uint(h.z);
  uint4 info = __ldg(reinterpret_cast<const uint4*>(P.v.surfaces + record) + 4);
  uint32_t material = info.y == NO_MATERIAL
                          ? f2u(__ldg(reinterpret_cast<const float*>(P.v.triangles + surface) + 3))
                          : info.y;
  material = min(material, P.bins / 2u - 2u);
  uint32_t cont = 0u;
  if (P.c.enabled && P.bounce >= P.c.query_bounce && P.bounce <= P.c.query_last) {
    cont = P.c.tslot[i] != ~0u ? 1u : 0u;
    if (!cont) {
      float4 o = P.w.ray_o[i], d = P.w.ray_d[i];
      cont = cell_ok(P.c, add3(mk3(o.x, o.y, o.z), scl3(mk3(d.x, d.y, d.z), h.x))) ? 0u : 1u;
      if (!cont && P.bounce < P.c.query_last && P.c.min_roughness > 0.0f) {
        const float4* row = P.v.materials + (size_t)(material + 1u) * 8u;
        float rough = fmax_(__ldg(row).w, 0.05f);
        if (P.sp.filter_glossy > 0.0f && (__float_as_uint(d.w) & F_DIFFUSED)) rough = fmax_(rough, P.sp.filter_glossy);
        cont = (rough >= P.c.min_roughness && !(__ldg(row + 2).y > 0.0f)) ? 0u : 1u;
      }
    }
  }
  return 2u * material + cont;
}

// This block's share [first, last) of n queue entries.
__device__ __forceinline__ void block_chunk(uint32_t n, uint32_t& first, uint32_t& last) {
  uint32_t per = (n + gridDim.x - 1u) / gridDim.x;
  first = min(n, blockIdx.x * per);
  last = min(n, first + per);
}

// The extend queue of the bounces after the first grouped by ray: direction
// octant x a 4 x 4 x 4 cell of the origin in the scene box, so that a warp's
// rays walk the same parts of the tree.
constexpr uint32_t RAY_BINS = 512;

__device__ __forceinline__ uint32_t ray_key(const Pass& P, uint32_t i) {
  float4 o = P.w.ray_o[i], d = P.w.ray_d[i];
  float q[3] = {o.x, o.y, o.z};
  uint32_t cell = 0u;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float u = (q[k] - P.scene_lo[k]) * P.scene_inv[k];
    u = u > 0.0f ? (u < 1.0f ? u : 1.0f) : 0.0f;
    cell = cell * 4u + min((uint32_t)(u * 4.0f), 3u);
  }
  uint32_t octant = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  return octant * 64u + cell;
}

// RAYS: the extend queue by ray_key (RAY_BINS); otherwise the shade queue by material_key (P.bins).
template <bool RAYS>
__global__ void __launch_bounds__(256) k_sort_count(const __grid_constant__ Pass P, uint32_t which) {
  __shared__ uint32_t hist[SORT_BINS];
  const uint32_t n = P.w.counters[which];
  const uint32_t* queue = P.w.queue[which];
  const uint32_t bins = RAYS ? P.ray_bins : P.bins;
  for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x) hist[b] = 0u;
  __syncthreads();
  uint32_t first, last;
  block_chunk(n, first, last);
  for (uint32_t q = first + threadIdx.x; q < last; q += blockDim.x) {
    uint32_t key = RAYS ? ray_key(P, queue[q]) : material_key(P, queue[q]);
    P.w.keys[q] = key;
    atomicAdd(&hist[key], 1u);
  }
  __syncthreads();
  uint32_t* global = RAYS ? P.w.rhist : P.w.hist;
  for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x)
    if (hist[b]) atomicAdd(global + b, hist[b]);
}

template <bool RAYS>
__global__ void __launch_bounds__(256) k_sort_place(const __grid_constant__ Pass P, uint32_t which) {
  __shared__ uint32_t base[SORT_BINS];
  __shared__ uint32_t local[SORT_BINS];
  const uint32_t n = P.w.counters[which];
  const uint32_t* queue = P.w.queue[which];
  const uint32_t bins = RAYS ? P.ray_bins : P.bins;
  const uint32_t* global = RAYS ? P.w.rhist : P.w.hist;
  uint32_t* cursor = RAYS ? P.w.rcursor : P.w.cursor;
  // exclusive scan of the global histogram (one thread: the bins are few)
  if (threadIdx.x == 0) {
    uint32_t run = 0u;
    for (uint32_t b = 0; b < bins; ++b) {
      base[b] = run;
      run += global[b];
    }
  }
  for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x) local[b] = 0u;
  __syncthreads();
  uint32_t first, last;
  block_chunk(n, first, last);
  for (uint32_t q = first + threadIdx.x; q < last; q += blockDim.x) atomicAdd(&local[P.w.keys[q]], 1u);
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x) {
    uint32_t c = local[b];
    base[b] += c ? atomicAdd(cursor + b, c) : 0u;
    local[b] = 0u;
  }
  __syncthreads();
  for (uint32_t q = first + threadIdx.x; q < last; q += blockDim.x) {
    uint32_t key = P.w.keys[q];
    P.w.sorted[base[key] + atomicAdd(&local[key], 1u)] = queue[q];
  }
}
// Before the connect: rewind its work counter and take its own copy of the
// shadow-queue count (the next bounce's k_reset may empty the queue count
// while the connect still runs), and count the any-hit queries.
__global__ void k_rewind(const __grid_constant__ Pass P) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.w.counters[16] = 0u;
    P.w.counters[17] = P.w.counters[2];
    P.w.counters[14] = 0u;
    reinterpret_cast<unsigned long long*>(P.w.counters + 8)[1] += P.w.counters[2];
  }
}

// ------------------------------------------------------------------ extend
// THREADS per block is a launch choice of the autotuner: the walk is per lane
// and the refill per warp, so the block size changes only the residency.
// SHORT entries of each lane's traversal stack live in shared memory (a tuning
// choice: 0 or 8), the rest in local memory.
template <bool ANY, int THREADS, int SHORT>
__global__ void __launch_bounds__(THREADS, TRACE_WARPS_PER_SM * 32 / THREADS) k_trace_queue(const __grid_constant__ Pass P,
                                                                                       uint32_t which) {
  constexpr unsigned FULL = 0xffffffffu;
  const uint32_t* queue = ANY ? P.w.squeue : ((P.ray_bins && P.bounce > 0u) ? P.w.sorted : P.w.queue[which]);
  const uint32_t n = ANY ? P.w.counters[17] : P.w.counters[which];
  uint32_t* counter = P.w.counters + (ANY ? 16 : 4);
  __shared__ uint32_t short_ref[SHORT > 0 ? SHORT * THREADS : 1];
  __shared__ float short_near[SHORT > 0 ? SHORT * THREADS : 1];
  LaneStack<SHORT> st;
  if constexpr (SHORT > 0) {
    st.sh_ref = short_ref + threadIdx.x;
    st.sh_near = short_near + threadIdx.x;
    st.lanes = THREADS;
  }
  Walker<ANY, false, TRACE_BOX, TRACE_SPEC> w;
  const int lane = threadIdx.x & 31;
  uint32_t idx = 0, item = 0;
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
          item = queue[idx];
          float4 a = ANY ? P.w.sh_o[item] : P.w.ray_o[item];
          float4 b = ANY ? P.w.sh_d[item] : P.w.ray_d[item];
          w.start(P.s, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), ANY ? a.w : 1e20f);
          have = true;
        } else {
          retired = true;
        }
      }
    }
    if (__all_sync(FULL, retired)) break;
    if (have) {
      w.inner_phase(P.s, st, [&](v3& o, v3& d) {
        float4 a = ANY ? P.w.sh_o[item] : P.w.ray_o[item];
        float4 b = ANY ? P.w.sh_d[item] : P.w.ray_d[item];
        o = mk3(a.x, a.y, a.z);
        d = mk3(b.x, b.y, b.z);
      });
      if (w.leaf_ready()) w.leaf_phase(P.s, st);
      if (!w.leaf_ready()) {
        if (w.retry) {
          (ANY ? P.w.retry : P.w.eretry)[atomicAdd(P.w.counters + (ANY ? 14 : 13), 1u)] = item;
        } else if (ANY) {
          reinterpret_cast<float*>(P.w.sh_d + item)[3] = __uint_as_float(w.hit.hit ? 0u : 1u);
        } else {
          P.w.hit[item] = make_float4(w.hit.t, __uint_as_float(w.hit.slot), __uint_as_float(w.hit.record), w.hit.u);
          P.w.hit_v[item] = w.hit.v;
        }
        have = false;
      }
    }
  }
}

// The queue items k_trace_queue handed over (rays that are not bounded in
// world or instance space), walked again from the start with IEEE division
// throughout; its launch reads the count on the device, so a pass issues it
// whether or not any ray needs it.
template <bool ANY>
__global__ void __launch_bounds__(128) k_trace_queue_retry(const __grid_constant__ Pass P) {
  const uint32_t n = P.w.counters[ANY ? 14 : 13];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const uint32_t item = (ANY ? P.w.retry : P.w.eretry)[k];
    float4 a = ANY ? P.w.sh_o[item] : P.w.ray_o[item];
    float4 b = ANY ? P.w.sh_d[item] : P.w.ray_d[item];
    LaneStack<0> st;
    Walker<ANY, false, BOX_IEEE> w;
    w.start(P.s, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), ANY ? a.w : 1e20f);
    w.run(P.s, st, [&](v3& o, v3& d) {
      o = mk3(a.x, a.y, a.z);
      d = mk3(b.x, b.y, b.z);
    });
    if (ANY) {
      reinterpret_cast<float*>(P.w.sh_d + item)[3] = __uint_as_float(w.hit.hit ? 0u : 1u);
    } else {
      P.w.hit[item] = make_float4(w.hit.t, __uint_as_float(w.hit.slot), __uint_as_float(w.hit.record), w.hit.u);
      P.w.hit_v[item] = w.hit.v;
    }
  }
}

// ------------------------------------------------------------------ shade
struct HitInfo {
  float t;
  v3 n, geometric;
  uint32_t material, surface, record;
};

// tri_fill (trace.wgsl:754-779) + world_hit (:682-694) from the stored hit.
__device__ __forceinline__ HitInfo fill_hit(const Pass& P, float4 h, float hv) {
  HitInfo out;
  out.t = h.x;
  out.surface = __float_as_uint(h.y);
  out.record = __float_as_uint(h.z);
  float u = h.w, v = hv;
  const float4* tp = reinterpret_cast<const float4*>(P.v.triangles + out.surface);
  float4 ta = __ldg(tp), tb = __ldg(tp + 1), tc = __ldg(tp + 2), na = __ldg(tp + 3), nb = __ldg(tp + 4),
         nc = __ldg(tp + 5);
  v3 a = f3of(ta);
  v3 e1 = sub3(f3of(tb), a);
  v3 e2 = sub3(f3of(tc), a);
  v3 geometric = normalize3(cross3(e1, e2));
  v3 shaded = add3(add3(scl3(f3of(na), 1.0f - u - v), scl3(f3of(nb), u)), scl3(f3of(nc), v));
  v3 fallback = out.record > 0u ? splat3(0.0f) : geometric;
  v3 n = dot3(shaded, shaded) > 1e-12f ? normalize3(shaded) : fallback;
  const float4* sp = reinterpret_cast<const float4*>(P.v.surfaces + out.record);
  uint4 info = __ldg(reinterpret_cast<const uint4*>(sp + 4));
  out.material = info.y == NO_MATERIAL ? f2u(ta.w) : info.y;
  if (out.record == 0u) {
    out.n = n;
    out.geometric = geometric;
    return out;
  }
  float mirror = __uint_as_float(info.w) < 0.0f ? -1.0f : 1.0f;
  v3 i0 = f3of(__ldg(sp + 8)), i1 = f3of(__ldg(sp + 9)), i2 = f3of(__ldg(sp + 10));
  v3 wg = scl3(normalize3(add3(add3(scl3(i0, geometric.x), scl3(i1, geometric.y)), scl3(i2, geometric.z))), mirror);
  v3 sh = add3(add3(scl3(i0, n.x), scl3(i1, n.y)), scl3(i2, n.z));
  bool zero = n.x == 0.0f && n.y == 0.0f && n.z == 0.0f;
  out.n = zero ? wg : normalize3(sh);
  out.geometric = wg;
  return out;
}

__device__ __forceinline__ float emitter_weight(const Pass& P, const HitInfo& hit, v3 p, v3 previous_point,
                                                float previous_pdf) {
  float4 em = __ldg(P.v.materials + (size_t)(hit.material + 1u) * 8u + 5u);
  if (previous_pdf <= 0.0f || (em.x <= 0.0f && em.y <= 0.0f && em.z <= 0.0f)) return 1.0f;
  uint32_t index = f2u(__ldg(reinterpret_cast<const float*>(P.v.triangles + hit.surface) + 11));
  if (index == 0u) return 1.0f;
  return mis_power(previous_pdf, emitter_pdf(load_emitter(P.v, index), p, previous_point, hit.geometric));
}

// Adds the pending light-slot contributions of path i (previous bounce) in
// slot order.
__device__ __forceinline__ v3 flush_pending(const Pass& P, uint32_t i, uint32_t flags, v3 result) {
  uint32_t pending = (flags >> F_PEND) & 15u;
  for (uint32_t j = 0; j < pending; ++j) {
    uint32_t slot = i * P.cap + j;
    float vis = reinterpret_cast<const float*>(P.w.sh_d + slot)[3];
    if (__float_as_uint(vis) != 0u) result = add3(result, f3of(P.w.sh_c[slot]));
  }
  return result;
}

// What the radiance cache reads of a shaded hit (5 float4): position and
// roughness, outgoing direction and transmission, normal, diffuse albedo,
// specular albedo (F0: 4 % for dielectrics, the base colour for metals).
__device__ __noinline__ void cache_features(float4* out, v3 p, v3 wo, v3 n, const Shaded& s) {
  float m = s.metalness, tr = s.transmission;
  v3 diffuse = scl3(s.base, (1.0f - m) * (1.0f - tr));
  v3 spec = mix3(splat3(0.04f), s.base, m);
  out[0] = make_float4(p.x, p.y, p.z, s.roughness);
  out[1] = make_float4(wo.x, wo.y, wo.z, tr);
  out[2] = make_float4(n.x, n.y, n.z, 0.0f);
  out[3] = make_float4(diffuse.x, diffuse.y, diffuse.z, 0.0f);
  out[4] = make_float4(spec.x, spec.y, spec.z, 0.0f);
}

// Training records of a finished training path: for every recorded vertex,
// the radiance the path gathered after it, divided by the throughput that
// reached it (the path's estimate of the vertex's scattered radiance).
__device__ __noinline__ void emit_records(const float4* __restrict__ tvert, float4* __restrict__ records,
                                          uint32_t* count, uint32_t rcap, uint32_t vertices, uint32_t ts,
                                          v3 result) {
  uint32_t slot = ts & 0xFFFFFFu, mask = ts >> 24;
  for (uint32_t b = 0; b < vertices; ++b) {
    if (!((mask >> b) & 1u)) continue;
    const float4* vtx = tvert + ((size_t)slot * vertices + b) * 7u;
    float4 T = vtx[5], R = vtx[6];
    float tx = T.x > 0.0f ? fmaxf(result.x - R.x, 0.0f) / T.x : 0.0f;
    float ty = T.y > 0.0f ? fmaxf(result.y - R.y, 0.0f) / T.y : 0.0f;
    float tz = T.z > 0.0f ? fmaxf(result.z - R.z, 0.0f) / T.z : 0.0f;
    uint32_t k = atomicAdd(count, 1u);
    if (k >= rcap) return;
    float4* rec = records + (size_t)k * 6u;
#pragma unroll
    for (int j = 0; j < 5; ++j) rec[j] = vtx[j];
    rec[5] = make_float4(tx, ty, tz, 1.0f);
  }
}

// DEFERRED: light-slot shadow rays go through the shadow queue (the usual
// case); otherwise (more than CAP_MAX light slots) they are traced inline.
template <bool DEFERRED>
__global__ void __launch_bounds__(kThreads, SHADE_MIN_BLOCKS) k_shade(const __grid_constant__ Pass P,uint32_t which) {
  const uint32_t n = P.w.counters[which];
  const uint32_t* queue = P.bins ? P.w.sorted : P.w.queue[which];
  uint32_t* next_queue = P.w.queue[which ^ 1u];
  uint32_t* next_count = P.w.counters + (which ^ 1u);
  const uint32_t bounce = P.bounce;
  const Specialise& sp = P.sp;
  const ShadeView& V = P.v;
  const uint32_t TOTAL = sp.total_bounces;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t qi = base + threadIdx.x;
    bool active = qi < n;
    bool cont = false;
    uint32_t i = active ? queue[qi] : 0u;
    if (active) {
      float4 ro = P.w.ray_o[i], rd = P.w.ray_d[i], th = P.w.thr[i], rs = P.w.res[i];
      v3 o = mk3(ro.x, ro.y, ro.z), d = mk3(rd.x, rd.y, rd.z);
      float previous_pdf = ro.w;
      uint32_t flags = __float_as_uint(rd.w);
      v3 throughput = mk3(th.x, th.y, th.z);
      uint32_t state = __float_as_uint(th.w);
      v3 result = flush_pending(P, i, flags, mk3(rs.x, rs.y, rs.z));
      flags &= ~(15u << F_PEND);
      uint32_t pixel = __float_as_uint(rs.w);
      uint32_t px = pixel % P.width + P.f.window[2], py = pixel / P.width + P.f.window[3];
      Rng r{hash_iqnt2d(px, py) ^ pass_seed(P), pass_accum(P) + P.sample, 16u * (bounce + 1u)};
      float4 h = P.w.hit[i];
      float reach = h.x;
      v3 origin_point = spawn_point(o, neg3(d), o, 0.0f);
      result = add3(result, capped(P, mul3(throughput, light_hits(V, o, d, reach, origin_point, previous_pdf)),
                                   bounce > 1u));
      uint32_t pending = 0u;
      if (h.x >= 1e19f) {
        if (!(bounce == 0u && P.f.forward[3] > 0.0f)) {
          float pdf = sky_pdf(V, d);
          float weight = (bounce > 0u && previous_pdf > 0.0f) ? previous_pdf / (previous_pdf + pdf) : 1.0f;
          result = add3(result, capped(P, scl3(mul3(throughput, sky_radiance(V)), weight), bounce > 1u));
        }
      } else {
        HitInfo hit = fill_hit(P, h, P.w.hit_v[i]);
        v3 p = add3(o, scl3(d, hit.t));
        v3 nn = dot3(hit.n, d) > 0.0f ? neg3(hit.n) : hit.n;
        Shaded s = load_surface(V, hit.material);
        v3 geometric = dot3(hit.geometric, d) > 0.0f ? neg3(hit.geometric) : hit.geometric;
        if (dot3(nn, geometric) < 0.05f) nn = normalize3(add3(nn, scl3(geometric, 0.1f)));
        s.roughness = fmax_(s.roughness, 0.05f);
        s.clearcoat_roughness = fmax_(s.clearcoat_roughness, 0.05f);
        if (sp.filter_glossy > 0.0f && (flags & F_DIFFUSED)) {
          s.roughness = fmax_(s.roughness, sp.filter_glossy);
          s.clearcoat_roughness = fmax_(s.clearcoat_roughness, sp.filter_glossy);
        }
        if (bounce == 0u) {
          P.w.alb[i] = make_float4(s.base.x, s.base.y, s.base.z, 1.0f);
          P.w.nrm[i] = make_float4(nn.x, nn.y, nn.z, 1.0f);
        }
        s.emission = scl3(s.emission, emitter_weight(P, hit, p, origin_point, previous_pdf));
        result = add3(result, capped(P, mul3(throughput, s.emission), bounce > 1u));
        bool to_cache = false;
        if (P.c.enabled && !(flags & F_LAST)) {
          uint32_t ts = P.c.tslot[i];
          if (ts != ~0u) {
            if (bounce <= P.c.record_bounces) {
              float4* vtx = P.c.tvert + ((size_t)(ts & 0xFFFFFFu) * (P.c.record_bounces + 1u) + bounce) * 7u;
              cache_features(vtx, p, neg3(d), nn, s);
              vtx[5] = make_float4(throughput.x, throughput.y, throughput.z, 0.0f);
              vtx[6] = make_float4(result.x, result.y, result.z, 0.0f);
              P.c.tslot[i] = ts | (1u << (24u + bounce));
            }
          } else if (bounce >= P.c.query_bounce && bounce <= P.c.query_last && cell_ok(P.c, p) &&
                     (bounce == P.c.query_last || P.c.min_roughness <= 0.0f ||
                      (s.roughness >= P.c.min_roughness && !(s.transmission > 0.0f)))) {
            uint32_t k = claim(P.w.counters + 5, true);
            cache_features(P.c.query + (size_t)k * 5u, p, neg3(d), nn, s);
            P.c.cqueue[k] = i;
            to_cache = true;
            flags |= F_CACHED;
          }
        }
        if (!(flags & F_LAST) && !to_cache) {
          m3 transform = basis(nn);
          v3 wo = mulmtv(transform, neg3(d));
          v3 origin = spawn_point(p, nn, o, hit.t);
          bool entering = dot3(hit.n, d) < 0.0f;
          for (uint32_t k = 0u; k < P.slots; ++k) {
            float4 u;  // the slot's Sobol sample, looked up once the slot is known to be live
            v3 local = mk3(0.0f, 0.0f, 1.0f), direction = mk3(0.0f, 0.0f, 1.0f), strength = splat3(0.0f);
            float limit = 1e19f, pdf = 0.0f;
            float lit_roughness = s.roughness;
            if (k == 0u) {
              if (P.f.sun_color[3] <= 0.0f) continue;
              u = sobol4(V, sp, r, light_dim(k));
              direction = normalize3(mk3(P.f.sun_dir[0], P.f.sun_dir[1], P.f.sun_dir[2]));
              if (P.f.sun_dir[3] < 1.0f) {
                float height = 1.0f - rnd(sp, state, u.x) * (1.0f - P.f.sun_dir[3]);
                float radius = sqrtf(fmax_(0.0f, 1.0f - height * height));
                float phi = 2.0f * SH_PI * rnd(sp, state, u.y);
                m3 orient = basis(direction);
                direction = normalize3(mulmv(orient, mk3(radius * cos_(phi), radius * sin_(phi), height)));
              }
              local = mulmtv(transform, direction);
              if (local.z <= 0.0f) continue;
              strength = scl3(mk3(P.f.sun_color[0], P.f.sun_color[1], P.f.sun_color[2]), P.f.sun_color[3] * 1.0f);
            } else if (k == 1u) {
              if (V.sky_width == 0u) continue;
              u = sobol4(V, sp, r, light_dim(k));
              float ux = rnd(sp, state, u.x);
              float uy = rnd(sp, state, u.y);
              // a black sky adds nothing (its sample is drawn all the same)
              if (V.sky_radiance[0] == 0.0f && V.sky_radiance[1] == 0.0f && V.sky_radiance[2] == 0.0f) continue;
              SkySample light = sky_sample(V, ux, uy);
              direction = light.direction;
              local = mulmtv(transform, direction);
              if (local.z <= 0.0f) continue;
              strength = scl3(sky_radiance(V), 1.0f);
              pdf = light.pdf;
              if (!(pdf > 0.0f)) continue;
            } else {
              uint32_t slot = k - 2u;
              if (slot == 0u && V.emitter_count == 0u) continue;  // no emissive triangles
              u = sobol4(V, sp, r, light_dim(k));
              Candidate picked;
              if (slot > V.looped) {
                float2 pk = tree_pick(V, P.light_rows, p, transform.c2, rnd(sp, state, u.z), nullptr);
                if (!(pk.y > 0.0f)) {
                  picked = candidate_none();
                } else {
                  picked = light_candidate(sp, V, f2u(pk.x), transform, p, origin, geometric, state, u);
                  picked.scale = divs3(picked.scale, pk.y);
                }
              } else if (slot > 0u) {
                picked = light_candidate(sp, V, slot - 1u, transform, p, origin, geometric, state, u);
              } else if (V.emitter_count == 0u) {
                picked = candidate_none();
              } else {
                picked = emitter_candidate(V, sp, transform, p, origin, state, u);
              }
              if (picked.limit < 0.0f) continue;
              local = picked.wi;
              direction = picked.direction;
              strength = picked.scale;
              pdf = picked.pdf;
              limit = picked.limit;
              lit_roughness = fmax_(s.roughness, picked.roughness);
            }
            if (pdf > 0.0f) {
              float bsdf = bsdf_pdf(s, wo, local);
              if (k == 1u) {
                strength = divs3(strength, pdf + bsdf);
              } else {
                float ratio = bsdf / pdf;
                strength = divs3(strength, pdf * (1.0f + ratio * ratio));
              }
            }
            v3 term = mul3(scl3(scl3(mul3(throughput, bsdf_eval(s, wo, local, lit_roughness)),
                                     pdf > 0.0f ? glossy_share(s) : 1.0f),
                                local.z),
                           strength);
            term = capped(P, term, bounce > 0u);
            if (term.x == 0.0f && term.y == 0.0f && term.z == 0.0f) continue;  // adds nothing, traces nothing
            if (!DEFERRED) {
              if (limit > 0.0f && traverse<true>(P.s, origin, direction, limit).hit) continue;
              result = add3(result, term);
              continue;
            }
            uint32_t slot_index = i * P.cap + pending;
            P.w.sh_c[slot_index] = make_float4(term.x, term.y, term.z, 0.0f);
            P.w.sh_o[slot_index] = make_float4(origin.x, origin.y, origin.z, limit);
            P.w.sh_d[slot_index] = make_float4(direction.x, direction.y, direction.z, __uint_as_float(limit > 0.0f ? 0u : 1u));
            uint32_t at = claim(P.w.counters + 2, limit > 0.0f);  // one atomic per warp
            if (limit > 0.0f) P.w.squeue[at] = slot_index;
            pending += 1u;
          }
          // BSDF sampling and the next ray (trace.wgsl:2472-2500)
          uint32_t carried = flags & F_CARRIED;
          BsdfSample sample = sample_bsdf(sp, s, wo, entering, carried, state, sobol4(V, sp, r, 3u));
          v3 wi = sample.dir;
          uint32_t l0 = lobe_count(flags, F_LOBE0) + (sample.lobe == 0u ? 1u : 0u);
          uint32_t l1 = lobe_count(flags, F_LOBE1) + (sample.lobe == 1u ? 1u : 0u);
          uint32_t l2 = lobe_count(flags, F_LOBE2) + (sample.lobe == 2u ? 1u : 0u);
          bool diffused = (flags & F_DIFFUSED) || sample.lobe == 0u;
          bool last = bounce >= TOTAL || l0 > sp.diffuse_bounces || l1 > sp.glossy_bounces || l2 > sp.transmission_bounces;
          bool lit_vertex = (flags & F_LIT) != 0u;
          bool through = sample.pdf < -1.5f && lit_vertex;
          lit_vertex = sample.pdf > 0.0f || through;
          bool go = true;
          if (sample.pdf < 0.0f) {
            throughput = mul3(throughput, sample.weight);
            carried = sample.channel;
            if (sample.pdf < -1.5f)
              throughput = mul3(throughput, mul3(mk3(sqrtf(clamp_(s.base.x, 0.0f, 1.0f)), sqrtf(clamp_(s.base.y, 0.0f, 1.0f)),
                                                     sqrtf(clamp_(s.base.z, 0.0f, 1.0f))),
                                                 beer(s.thickness, s.subsurface_tint, s.absorption)));
            d = normalize3(mulmv(transform, wi));
            previous_pdf = 0.0f;
          } else if (wi.z <= 0.0f || sample.pdf <= 0.0f) {
            go = false;
          } else {
            throughput = mul3(throughput, scl3(divs3(scl3(scl3(bsdf_eval(s, wo, wi, s.roughness), glossy_share(s)), wi.z), sample.pdf), 1.0f));
            d = normalize3(mulmv(transform, wi));
            previous_pdf = sample.pdf;
          }
          if (go) {
            o = spawn_point(p, d, o, hit.t);
            if (bounce >= 3u) {
              float keep = clamp_(fmax_(throughput.x, fmax_(throughput.y, throughput.z)), 0.05f, 0.95f);
              Rng r0 = r;
              if (rnd(sp, state, sobol4(V, sp, r0, 0u).x) > keep)
                go = false;
              else
                throughput = divs3(throughput, keep);
            }
          }
          flags = (carried & F_CARRIED) | (l0 << F_LOBE0) | (l1 << F_LOBE1) | (l2 << F_LOBE2) | (last ? F_LAST : 0u) |
                  (through ? F_THROUGH : 0u) | (lit_vertex ? F_LIT : 0u) | (diffused ? F_DIFFUSED : 0u);
          cont = go;
        }
      }
      flags |= pending << F_PEND;
      P.w.ray_o[i] = make_float4(o.x, o.y, o.z, previous_pdf);
      P.w.ray_d[i] = make_float4(d.x, d.y, d.z, __uint_as_float(flags));
      P.w.thr[i] = make_float4(throughput.x, throughput.y, throughput.z, __uint_as_float(state));
      P.w.res[i] = make_float4(result.x, result.y, result.z, __uint_as_float(pixel));
    }
    append(next_queue, next_count, i, active && cont);
  }
}

// ------------------------------------------------------------------ split shade
// The same bounce body in three kernels, for an instruction cache that the
// whole body overflows: k_shade_hit (emission, light hits, the cache), then,
// for the paths that scatter, k_shade_lights (the light slots) and
// k_shade_bsdf (the BSDF sample, Russian roulette, the next ray).  The shaded
// surface travels between them in 9 float4 per path; every expression is the
// fused kernel's, in the same order, so the results are identical.

__device__ __forceinline__ void store_surface(float4* out, v3 p, float t, v3 nn, bool entering, v3 geometric,
                                              const Shaded& s) {
  out[0] = make_float4(p.x, p.y, p.z, t);
  out[1] = make_float4(nn.x, nn.y, nn.z, entering ? 1.0f : 0.0f);
  out[2] = make_float4(geometric.x, geometric.y, geometric.z, s.roughness);
  out[3] = make_float4(s.base.x, s.base.y, s.base.z, s.metalness);
  out[4] = make_float4(s.specular, s.clearcoat, s.clearcoat_roughness, s.sheen);
  out[5] = make_float4(s.transmission, s.ior, s.dispersion, s.thickness);
  out[6] = make_float4(s.subsurface, s.subsurface_tint.x, s.subsurface_tint.y, s.subsurface_tint.z);
  out[7] = make_float4(s.absorption, s.emission.x, s.emission.y, s.emission.z);
  out[8] = make_float4(s.fresnel_power, 0.0f, 0.0f, 0.0f);
}

struct Surface {
  v3 p, nn, geometric;
  float t;
  bool entering;
  Shaded s;
};

__device__ __forceinline__ Surface load_surface_record(const float4* in) {
  float4 a = in[0], b = in[1], c = in[2], e = in[3], f = in[4], g = in[5], h = in[6], k = in[7], m = in[8];
  Surface S;
  S.p = mk3(a.x, a.y, a.z);
  S.t = a.w;
  S.nn = mk3(b.x, b.y, b.z);
  S.entering = b.w != 0.0f;
  S.geometric = mk3(c.x, c.y, c.z);
  S.s.roughness = c.w;
  S.s.base = mk3(e.x, e.y, e.z);
  S.s.metalness = e.w;
  S.s.specular = f.x;
  S.s.clearcoat = f.y;
  S.s.clearcoat_roughness = f.z;
  S.s.sheen = f.w;
  S.s.transmission = g.x;
  S.s.ior = g.y;
  S.s.dispersion = g.z;
  S.s.thickness = g.w;
  S.s.subsurface = h.x;
  S.s.subsurface_tint = mk3(h.y, h.z, h.w);
  S.s.absorption = k.x;
  S.s.emission = mk3(k.y, k.z, k.w);
  S.s.fresnel_power = m.x;
  return S;
}

__global__ void __launch_bounds__(kThreads) k_shade_hit(const __grid_constant__ Pass P, uint32_t which) {
  const uint32_t n = P.w.counters[which];
  const uint32_t* queue = P.bins ? P.w.sorted : P.w.queue[which];
  const uint32_t bounce = P.bounce;
  const Specialise& sp = P.sp;
  const ShadeView& V = P.v;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t qi = base + threadIdx.x;
    bool active = qi < n;
    bool lit = false;
    uint32_t i = active ? queue[qi] : 0u;
    if (active) {
      float4 ro = P.w.ray_o[i], rd = P.w.ray_d[i], th = P.w.thr[i], rs = P.w.res[i];
      v3 o = mk3(ro.x, ro.y, ro.z), d = mk3(rd.x, rd.y, rd.z);
      float previous_pdf = ro.w;
      uint32_t flags = __float_as_uint(rd.w);
      v3 throughput = mk3(th.x, th.y, th.z);
      v3 result = flush_pending(P, i, flags, mk3(rs.x, rs.y, rs.z));
      flags &= ~(15u << F_PEND);
      uint32_t pixel = __float_as_uint(rs.w);
      float4 h = P.w.hit[i];
      float reach = h.x;
      v3 origin_point = spawn_point(o, neg3(d), o, 0.0f);
      result = add3(result, capped(P, mul3(throughput, light_hits(V, o, d, reach, origin_point, previous_pdf)),
                                   bounce > 1u));
      if (h.x >= 1e19f) {
        if (!(bounce == 0u && P.f.forward[3] > 0.0f)) {
          float pdf = sky_pdf(V, d);
          float weight = (bounce > 0u && previous_pdf > 0.0f) ? previous_pdf / (previous_pdf + pdf) : 1.0f;
          result = add3(result, capped(P, scl3(mul3(throughput, sky_radiance(V)), weight), bounce > 1u));
        }
      } else {
        HitInfo hit = fill_hit(P, h, P.w.hit_v[i]);
        v3 p = add3(o, scl3(d, hit.t));
        v3 nn = dot3(hit.n, d) > 0.0f ? neg3(hit.n) : hit.n;
        Shaded s = load_surface(V, hit.material);
        v3 geometric = dot3(hit.geometric, d) > 0.0f ? neg3(hit.geometric) : hit.geometric;
        if (dot3(nn, geometric) < 0.05f) nn = normalize3(add3(nn, scl3(geometric, 0.1f)));
        s.roughness = fmax_(s.roughness, 0.05f);
        s.clearcoat_roughness = fmax_(s.clearcoat_roughness, 0.05f);
        if (sp.filter_glossy > 0.0f && (flags & F_DIFFUSED)) {
          s.roughness = fmax_(s.roughness, sp.filter_glossy);
          s.clearcoat_roughness = fmax_(s.clearcoat_roughness, sp.filter_glossy);
        }
        if (bounce == 0u) {
          P.w.alb[i] = make_float4(s.base.x, s.base.y, s.base.z, 1.0f);
          P.w.nrm[i] = make_float4(nn.x, nn.y, nn.z, 1.0f);
        }
        s.emission = scl3(s.emission, emitter_weight(P, hit, p, origin_point, previous_pdf));
        result = add3(result, capped(P, mul3(throughput, s.emission), bounce > 1u));
        bool to_cache = false;
        if (P.c.enabled && !(flags & F_LAST)) {
          uint32_t ts = P.c.tslot[i];
          if (ts != ~0u) {
            if (bounce <= P.c.record_bounces) {
              float4* vtx = P.c.tvert + ((size_t)(ts & 0xFFFFFFu) * (P.c.record_bounces + 1u) + bounce) * 7u;
              cache_features(vtx, p, neg3(d), nn, s);
              vtx[5] = make_float4(throughput.x, throughput.y, throughput.z, 0.0f);
              vtx[6] = make_float4(result.x, result.y, result.z, 0.0f);
              P.c.tslot[i] = ts | (1u << (24u + bounce));
            }
          } else if (bounce >= P.c.query_bounce && bounce <= P.c.query_last && cell_ok(P.c, p) &&
                     (bounce == P.c.query_last || P.c.min_roughness <= 0.0f ||
                      (s.roughness >= P.c.min_roughness && !(s.transmission > 0.0f)))) {
            uint32_t k = claim(P.w.counters + 5, true);
            cache_features(P.c.query + (size_t)k * 5u, p, neg3(d), nn, s);
            P.c.cqueue[k] = i;
            to_cache = true;
            flags |= F_CACHED;
          }
        }
        if (!(flags & F_LAST) && !to_cache) {
          store_surface(P.w.surf + (size_t)i * 9u, p, hit.t, nn, dot3(hit.n, d) < 0.0f, geometric, s);
          lit = true;
        }
      }
      P.w.ray_d[i] = make_float4(d.x, d.y, d.z, __uint_as_float(flags));
      P.w.res[i] = make_float4(result.x, result.y, result.z, __uint_as_float(pixel));
    }
    append(P.w.lit, P.w.counters + 12, i, active && lit);
  }
}

template <bool DEFERRED>
__global__ void __launch_bounds__(kThreads, SHADE_LIGHTS_MIN_BLOCKS) k_shade_lights(const __grid_constant__ Pass P) {
  const uint32_t n = P.w.counters[12];
  const uint32_t bounce = P.bounce;
  const Specialise& sp = P.sp;
  const ShadeView& V = P.v;
  for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < n; qi += gridDim.x * blockDim.x) {
    const uint32_t i = P.w.lit[qi];
    float4 ro = P.w.ray_o[i], rd = P.w.ray_d[i], th = P.w.thr[i], rs = P.w.res[i];
    v3 o = mk3(ro.x, ro.y, ro.z), d = mk3(rd.x, rd.y, rd.z);
    uint32_t flags = __float_as_uint(rd.w);
    v3 throughput = mk3(th.x, th.y, th.z);
    uint32_t state = __float_as_uint(th.w);
    v3 result = mk3(rs.x, rs.y, rs.z);
    uint32_t pixel = __float_as_uint(rs.w);
    uint32_t px = pixel % P.width + P.f.window[2], py = pixel / P.width + P.f.window[3];
    Rng r{hash_iqnt2d(px, py) ^ pass_seed(P), pass_accum(P) + P.sample, 16u * (bounce + 1u)};
    // The surface's geometry is held across the slots; its material record is
    // read again where a slot evaluates the BSDF, so that it is not live across
    // the light-tree descent (fewer values to keep in local memory there).
    const float4* record = P.w.surf + (size_t)i * 9u;
    const float4 g0 = record[0], g1 = record[1], g2 = record[2];
    const v3 p = mk3(g0.x, g0.y, g0.z), nn = mk3(g1.x, g1.y, g1.z), geometric = mk3(g2.x, g2.y, g2.z);
    const float roughness = g2.w;
    m3 transform = basis(nn);
    v3 origin = spawn_point(p, nn, o, g0.w);
    uint32_t pending = 0u;
    for (uint32_t k = 0u; k < P.slots; ++k) {
      float4 u;  // the slot's Sobol sample, looked up once the slot is known to be live
      v3 local = mk3(0.0f, 0.0f, 1.0f), direction = mk3(0.0f, 0.0f, 1.0f), strength = splat3(0.0f);
      float limit = 1e19f, pdf = 0.0f;
      float lit_roughness = roughness;
      if (k == 0u) {
        if (P.f.sun_color[3] <= 0.0f) continue;
        u = sobol4(V, sp, r, light_dim(k));
        direction = normalize3(mk3(P.f.sun_dir[0], P.f.sun_dir[1], P.f.sun_dir[2]));
        if (P.f.sun_dir[3] < 1.0f) {
          float height = 1.0f - rnd(sp, state, u.x) * (1.0f - P.f.sun_dir[3]);
          float radius = sqrtf(fmax_(0.0f, 1.0f - height * height));
          float phi = 2.0f * SH_PI * rnd(sp, state, u.y);
          m3 orient = basis(direction);
          direction = normalize3(mulmv(orient, mk3(radius * cos_(phi), radius * sin_(phi), height)));
        }
        local = mulmtv(transform, direction);
        if (local.z <= 0.0f) continue;
        strength = scl3(mk3(P.f.sun_color[0], P.f.sun_color[1], P.f.sun_color[2]), P.f.sun_color[3] * 1.0f);
      } else if (k == 1u) {
        if (V.sky_width == 0u) continue;
        u = sobol4(V, sp, r, light_dim(k));
        float ux = rnd(sp, state, u.x);
        float uy = rnd(sp, state, u.y);
        // a black sky adds nothing (its sample is drawn all the same)
        if (V.sky_radiance[0] == 0.0f && V.sky_radiance[1] == 0.0f && V.sky_radiance[2] == 0.0f) continue;
        SkySample light = sky_sample(V, ux, uy);
        direction = light.direction;
        local = mulmtv(transform, direction);
        if (local.z <= 0.0f) continue;
        strength = scl3(sky_radiance(V), 1.0f);
        pdf = light.pdf;
        if (!(pdf > 0.0f)) continue;
      } else {
        uint32_t slot = k - 2u;
        if (slot == 0u && V.emitter_count == 0u) continue;  // no emissive triangles
        u = sobol4(V, sp, r, light_dim(k));
        Candidate picked;
        if (slot > V.looped) {
          float2 pk = tree_pick(V, P.light_rows, p, transform.c2, rnd(sp, state, u.z), nullptr);
          if (!(pk.y > 0.0f)) {
            picked = candidate_none();
          } else {
            picked = light_candidate(sp, V, f2u(pk.x), transform, p, origin, geometric, state, u);
            picked.scale = divs3(picked.scale, pk.y);
          }
        } else if (slot > 0u) {
          picked = light_candidate(sp, V, slot - 1u, transform, p, origin, geometric, state, u);
        } else if (V.emitter_count == 0u) {
          picked = candidate_none();
        } else {
          picked = emitter_candidate(V, sp, transform, p, origin, state, u);
        }
        if (picked.limit < 0.0f) continue;
        local = picked.wi;
        direction = picked.direction;
        strength = picked.scale;
        pdf = picked.pdf;
        limit = picked.limit;
        lit_roughness = fmax_(roughness, picked.roughness);
      }
      const Surface S = load_surface_record(record);
      const Shaded& s = S.s;
      const v3 wo = mulmtv(transform, neg3(d));
      if (pdf > 0.0f) {
        float bsdf = bsdf_pdf(s, wo, local);
        if (k == 1u) {
          strength = divs3(strength, pdf + bsdf);
        } else {
          float ratio = bsdf / pdf;
          strength = divs3(strength, pdf * (1.0f + ratio * ratio));
        }
      }
      v3 term = mul3(scl3(scl3(mul3(throughput, bsdf_eval(s, wo, local, lit_roughness)),
                               pdf > 0.0f ? glossy_share(s) : 1.0f),
                          local.z),
                     strength);
      term = capped(P, term, bounce > 0u);
      if (term.x == 0.0f && term.y == 0.0f && term.z == 0.0f) continue;  // adds nothing, traces nothing
      if (!DEFERRED) {
        if (limit > 0.0f && traverse<true>(P.s, origin, direction, limit).hit) continue;
        result = add3(result, term);
        continue;
      }
      uint32_t slot_index = i * P.cap + pending;
      P.w.sh_c[slot_index] = make_float4(term.x, term.y, term.z, 0.0f);
      P.w.sh_o[slot_index] = make_float4(origin.x, origin.y, origin.z, limit);
      P.w.sh_d[slot_index] = make_float4(direction.x, direction.y, direction.z, __uint_as_float(limit > 0.0f ? 0u : 1u));
      uint32_t at = claim(P.w.counters + 2, limit > 0.0f);  // one atomic per warp
      if (limit > 0.0f) P.w.squeue[at] = slot_index;
      pending += 1u;
    }
    P.w.ray_d[i] = make_float4(d.x, d.y, d.z, __uint_as_float(flags | (pending << F_PEND)));
    P.w.thr[i] = make_float4(throughput.x, throughput.y, throughput.z, __uint_as_float(state));
    if (!DEFERRED) P.w.res[i] = make_float4(result.x, result.y, result.z, __uint_as_float(pixel));
  }
}

// ------------------------------------------------------------------ light slots, one kind per launch
// The light slots of the paths that scatter, one launch per live slot in slot
// order (sun, sky, emissive triangles, each looped light, the light tree)
// instead of every slot of a path in one thread.  A launch holds the state of
// one slot kind only, which fits its registers, where the kernel of all slots
// keeps the union of every kind's state in local memory.  The values are the
// same: a path's draws come in the same order (slot k's after slot k-1's; the
// pcg state travels in thr.w between launches), and the k-th live slot of a
// path writes shadow entry i * cap + pending, the pending count travelling in
// the flag word.  The tree's slot is two launches: the descent (k_tree_pick,
// one (row, pmf) per path), then its light's candidate and the BSDF.
constexpr int SLOT_SUN = 0, SLOT_SKY = 1, SLOT_EMITTER = 2, SLOT_LOOPED = 3, SLOT_TREE = 4;

// Whether the next bounce's extend runs beside the current bounce's connect (enqueue_pass).
// Plain 4K pass: 90.6 ms ahead, 91.4 in line; cached pass 41.5 against 42.0 ms.
#ifndef TRACE_AHEAD
#define TRACE_AHEAD 1
#endif
#ifndef SLOT_MIN_BLOCKS
#define SLOT_MIN_BLOCKS 8
#endif
#ifndef PICK_MIN_BLOCKS
#define PICK_MIN_BLOCKS 8
#endif
// Whether the descent kernel runs the light-tree functions inline or through their out-of-line copies.
// Plain 4K pass: out of line at 12 blocks per SM 93.1 ms, at 8 blocks 92.5; inline at 12, 10 and 8
// blocks 102.8, 104.8 and 108.1 ms (more code, fewer lanes per instruction).  Later, with the one-light
// leaves reusing the descent's importance: 8 blocks (64 registers) 91.5 ms, 6 blocks (72 registers, no
// spills) 91.7, 4 blocks 91.8.
#ifndef PICK_INLINE
#define PICK_INLINE false
#endif

__device__ __forceinline__ Rng slot_rng(const Pass& P, uint32_t pixel) {
  uint32_t px = pixel % P.width + P.f.window[2], py = pixel / P.width + P.f.window[3];
  return Rng{hash_iqnt2d(px, py) ^ pass_seed(P), pass_accum(P) + P.sample, 16u * (P.bounce + 1u)};
}

// The light tree's descent for every scattering path (slot k of tree_pick's
// caller in k_shade_lights): the pick (light row, pmf) at P.w.pick[qi].
__global__ void __launch_bounds__(kThreads, PICK_MIN_BLOCKS) k_tree_pick(const __grid_constant__ Pass P, uint32_t k) {
  const uint32_t n = P.w.counters[12];
  const Specialise& sp = P.sp;
  const ShadeView& V = P.v;
  for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < n; qi += gridDim.x * blockDim.x) {
    const uint32_t i = P.w.lit[qi];
    const float4* record = P.w.surf + (size_t)i * 9u;
    const float4 g0 = record[0], g1 = record[1];
    uint32_t state = __float_as_uint(reinterpret_cast<const float*>(P.w.thr + i)[3]);
    float start;
    if (sp.sobol) {
      start = sobol4(V, sp, slot_rng(P, __float_as_uint(reinterpret_cast<const float*>(P.w.res + i)[3])),
                     light_dim(k)).z;
    } else {
      start = random01(state);
      reinterpret_cast<float*>(P.w.thr + i)[3] = __uint_as_float(state);
    }
    P.w.pick[qi] = tree_pick_b<PICK_INLINE>(V, P.light_rows, mk3(g0.x, g0.y, g0.z), mk3(g1.x, g1.y, g1.z), start,
                                           nullptr);
  }
}

// Slot k of kind KIND for every scattering path: the body of k_shade_lights'
// slot loop for that kind, with the deferred shadow entry.
template <int KIND>
__global__ void __launch_bounds__(kThreads, SLOT_MIN_BLOCKS) k_light_slot(const __grid_constant__ Pass P, uint32_t k) {
  const uint32_t n = P.w.counters[12];
  const uint32_t bounce = P.bounce;
  const Specialise& sp = P.sp;
  const ShadeView& V = P.v;
  for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < n; qi += gridDim.x * blockDim.x) {
    const uint32_t i = P.w.lit[qi];
    float2 pk = make_float2(0.0f, 0.0f);
    if (KIND == SLOT_TREE) {
      pk = P.w.pick[qi];
      if (!(pk.y > 0.0f)) continue;  // no light picked: the slot adds nothing and draws nothing more
    }
    const float4 rd = P.w.ray_d[i], th = P.w.thr[i];
    const v3 d = mk3(rd.x, rd.y, rd.z);
    const uint32_t flags = __float_as_uint(rd.w);
    uint32_t state = __float_as_uint(th.w);
    const uint32_t state_in = state;
    const float4* record = P.w.surf + (size_t)i * 9u;
    const float4 g0 = record[0], g1 = record[1], g2 = record[2];
    const v3 p = mk3(g0.x, g0.y, g0.z), nn = mk3(g1.x, g1.y, g1.z);
    const m3 transform = basis(nn);
    float4 u = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (sp.sobol) u = sobol4(V, sp, slot_rng(P, __float_as_uint(reinterpret_cast<const float*>(P.w.res + i)[3])),
                             light_dim(k));
    v3 local = mk3(0.0f, 0.0f, 1.0f), direction = mk3(0.0f, 0.0f, 1.0f), strength = splat3(0.0f);
    v3 origin = p;
    float limit = 1e19f, pdf = 0.0f;
    float lit_roughness = g2.w;
    bool live = true;
    if (KIND == SLOT_SUN) {
      direction = normalize3(mk3(P.f.sun_dir[0], P.f.sun_dir[1], P.f.sun_dir[2]));
      if (P.f.sun_dir[3] < 1.0f) {
        float height = 1.0f - rnd(sp, state, u.x) * (1.0f - P.f.sun_dir[3]);
        float radius = sqrtf(fmax_(0.0f, 1.0f - height * height));
        float phi = 2.0f * SH_PI * rnd(sp, state, u.y);
        m3 orient = basis(direction);
        direction = normalize3(mulmv(orient, mk3(radius * cos_(phi), radius * sin_(phi), height)));
      }
      local = mulmtv(transform, direction);
      live = local.z > 0.0f;
      strength = scl3(mk3(P.f.sun_color[0], P.f.sun_color[1], P.f.sun_color[2]), P.f.sun_color[3] * 1.0f);
      const float4 ro = P.w.ray_o[i];
      origin = spawn_point(p, nn, mk3(ro.x, ro.y, ro.z), g0.w);
    } else if (KIND == SLOT_SKY) {
      float ux = rnd(sp, state, u.x);
      float uy = rnd(sp, state, u.y);
      if (V.sky_radiance[0] == 0.0f && V.sky_radiance[1] == 0.0f && V.sky_radiance[2] == 0.0f) {
        live = false;
      } else {
        SkySample light = sky_sample(V, ux, uy);
        direction = light.direction;
        local = mulmtv(transform, direction);
        strength = scl3(sky_radiance(V), 1.0f);
        pdf = light.pdf;
        live = local.z > 0.0f && pdf > 0.0f;
        const float4 ro = P.w.ray_o[i];
        origin = spawn_point(p, nn, mk3(ro.x, ro.y, ro.z), g0.w);
      }
    } else {
      const float4 ro = P.w.ray_o[i];
      origin = spawn_point(p, nn, mk3(ro.x, ro.y, ro.z), g0.w);
      Candidate picked;
      if (KIND == SLOT_TREE) {
        picked = light_candidate(sp, V, f2u(pk.x), transform, p, origin, mk3(g2.x, g2.y, g2.z), state, u);
        picked.scale = divs3(picked.scale, pk.y);
      } else if (KIND == SLOT_LOOPED) {
        picked = light_candidate(sp, V, k - 3u, transform, p, origin, mk3(g2.x, g2.y, g2.z), state, u);
      } else {
        picked = emitter_candidate(V, sp, transform, p, origin, state, u);
      }
      live = !(picked.limit < 0.0f);
      local = picked.wi;
      direction = picked.direction;
      strength = picked.scale;
      pdf = picked.pdf;
      limit = picked.limit;
      lit_roughness = fmax_(lit_roughness, picked.roughness);
    }
    if (live) {
      const Surface S = load_surface_record(record);
      const Shaded& s = S.s;
      const v3 wo = mulmtv(transform, neg3(d));
      if (pdf > 0.0f) {
        float bsdf = bsdf_pdf(s, wo, local);
        if (KIND == SLOT_SKY) {
          strength = divs3(strength, pdf + bsdf);
        } else {
          float ratio = bsdf / pdf;
          strength = divs3(strength, pdf * (1.0f + ratio * ratio));
        }
      }
      const float4 t4 = th;
      v3 term = mul3(scl3(scl3(mul3(mk3(t4.x, t4.y, t4.z), bsdf_eval(s, wo, local, lit_roughness)),
                               pdf > 0.0f ? glossy_share(s) : 1.0f),
                          local.z),
                     strength);
      term = capped(P, term, bounce > 0u);
      live = !(term.x == 0.0f && term.y == 0.0f && term.z == 0.0f);  // adds nothing, traces nothing
      if (live) {
        const uint32_t pending = (flags >> F_PEND) & 15u;
        uint32_t slot_index = i * P.cap + pending;
        P.w.sh_c[slot_index] = make_float4(term.x, term.y, term.z, 0.0f);
        P.w.sh_o[slot_index] = make_float4(origin.x, origin.y, origin.z, limit);
        P.w.sh_d[slot_index] =
            make_float4(direction.x, direction.y, direction.z, __uint_as_float(limit > 0.0f ? 0u : 1u));
        reinterpret_cast<float*>(P.w.ray_d + i)[3] =
            __uint_as_float((flags & ~(15u << F_PEND)) | ((pending + 1u) << F_PEND));
      }
    }
    uint32_t at = claim(P.w.counters + 2, live && limit > 0.0f);  // one atomic per warp
    if (live && limit > 0.0f) P.w.squeue[at] = i * P.cap + ((flags >> F_PEND) & 15u);
    if (state != state_in) reinterpret_cast<float*>(P.w.thr + i)[3] = __uint_as_float(state);
  }
}

__global__ void __launch_bounds__(kThreads) k_shade_bsdf(const __grid_constant__ Pass P, uint32_t which) {
  const uint32_t n = P.w.counters[12];
  uint32_t* next_queue = P.w.queue[which ^ 1u];
  uint32_t* next_count = P.w.counters + (which ^ 1u);
  const uint32_t bounce = P.bounce;
  const Specialise& sp = P.sp;
  const ShadeView& V = P.v;
  const uint32_t TOTAL = sp.total_bounces;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t qi = base + threadIdx.x;
    bool active = qi < n;
    bool cont = false;
    uint32_t i = active ? P.w.lit[qi] : 0u;
    if (active) {
      float4 ro = P.w.ray_o[i], rd = P.w.ray_d[i], th = P.w.thr[i];
      v3 o = mk3(ro.x, ro.y, ro.z), d = mk3(rd.x, rd.y, rd.z);
      float previous_pdf = ro.w;
      uint32_t flags = __float_as_uint(rd.w);
      const uint32_t pending = (flags >> F_PEND) & 15u;
      v3 throughput = mk3(th.x, th.y, th.z);
      uint32_t state = __float_as_uint(th.w);
      uint32_t pixel = __float_as_uint(P.w.res[i].w);
      uint32_t px = pixel % P.width + P.f.window[2], py = pixel / P.width + P.f.window[3];
      Rng r{hash_iqnt2d(px, py) ^ pass_seed(P), pass_accum(P) + P.sample, 16u * (bounce + 1u)};
      const Surface S = load_surface_record(P.w.surf + (size_t)i * 9u);
      const Shaded& s = S.s;
      const v3 p = S.p;
      m3 transform = basis(S.nn);
      v3 wo = mulmtv(transform, neg3(d));
      bool entering = S.entering;
      // BSDF sampling and the next ray (trace.wgsl:2472-2500)
      uint32_t carried = flags & F_CARRIED;
      BsdfSample sample = sample_bsdf(sp, s, wo, entering, carried, state, sobol4(V, sp, r, 3u));
      v3 wi = sample.dir;
      uint32_t l0 = lobe_count(flags, F_LOBE0) + (sample.lobe == 0u ? 1u : 0u);
      uint32_t l1 = lobe_count(flags, F_LOBE1) + (sample.lobe == 1u ? 1u : 0u);
      uint32_t l2 = lobe_count(flags, F_LOBE2) + (sample.lobe == 2u ? 1u : 0u);
      bool diffused = (flags & F_DIFFUSED) || sample.lobe == 0u;
      bool last = bounce >= TOTAL || l0 > sp.diffuse_bounces || l1 > sp.glossy_bounces || l2 > sp.transmission_bounces;
      bool lit_vertex = (flags & F_LIT) != 0u;
      bool through = sample.pdf < -1.5f && lit_vertex;
      lit_vertex = sample.pdf > 0.0f || through;
      bool go = true;
      if (sample.pdf < 0.0f) {
        throughput = mul3(throughput, sample.weight);
        carried = sample.channel;
        if (sample.pdf < -1.5f)
          throughput = mul3(throughput, mul3(mk3(sqrtf(clamp_(s.base.x, 0.0f, 1.0f)), sqrtf(clamp_(s.base.y, 0.0f, 1.0f)),
                                                 sqrtf(clamp_(s.base.z, 0.0f, 1.0f))),
                                             beer(s.thickness, s.subsurface_tint, s.absorption)));
        d = normalize3(mulmv(transform, wi));
        previous_pdf = 0.0f;
      } else if (wi.z <= 0.0f || sample.pdf <= 0.0f) {
        go = false;
      } else {
        throughput = mul3(throughput, scl3(divs3(scl3(scl3(bsdf_eval(s, wo, wi, s.roughness), glossy_share(s)), wi.z), sample.pdf), 1.0f));
        d = normalize3(mulmv(transform, wi));
        previous_pdf = sample.pdf;
      }
      if (go) {
        o = spawn_point(p, d, o, S.t);
        if (bounce >= 3u) {
          float keep = clamp_(fmax_(throughput.x, fmax_(throughput.y, throughput.z)), 0.05f, 0.95f);
          Rng r0 = r;
          if (rnd(sp, state, sobol4(V, sp, r0, 0u).x) > keep)
            go = false;
          else
            throughput = divs3(throughput, keep);
        }
      }
      flags = (carried & F_CARRIED) | (l0 << F_LOBE0) | (l1 << F_LOBE1) | (l2 << F_LOBE2) | (last ? F_LAST : 0u) |
              (through ? F_THROUGH : 0u) | (lit_vertex ? F_LIT : 0u) | (diffused ? F_DIFFUSED : 0u);
      flags |= pending << F_PEND;
      cont = go;
      P.w.ray_o[i] = make_float4(o.x, o.y, o.z, previous_pdf);
      P.w.ray_d[i] = make_float4(d.x, d.y, d.z, __uint_as_float(flags));
      P.w.thr[i] = make_float4(throughput.x, throughput.y, throughput.z, __uint_as_float(state));
    }
    append(next_queue, next_count, i, active && cont);
  }
}

// ------------------------------------------------------------------ finish
// Pending contributions of the last bounce, then Accum += (result, first
// albedo, first normal) in sample order (trace.wgsl:2564-2567).
__global__ void k_finish(const __grid_constant__ Pass P,Accum* __restrict__ accum) {
  const uint32_t n = P.w.counters[3];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 rs = P.w.res[i];
    uint32_t flags = __float_as_uint(P.w.ray_d[i].w);
    v3 result = flush_pending(P, i, flags, mk3(rs.x, rs.y, rs.z));
    if (flags & F_CACHED) {
      // the cache's radiance at the vertex the path ended at, through its throughput
      float4 pr = P.c.pred[i], th = P.w.thr[i];
      v3 radiance = mk3(fmaxf(pr.x, 0.0f), fmaxf(pr.y, 0.0f), fmaxf(pr.z, 0.0f));
      result = add3(result, capped(P, mul3(mk3(th.x, th.y, th.z), radiance), true));
    }
    if (P.c.enabled) {
      uint32_t ts = P.c.tslot[i];
      if (ts != ~0u)
        emit_records(P.c.tvert, P.c.records, P.w.counters + 7, P.c.rcap, P.c.record_bounces + 1u, ts, result);
    }
    uint32_t pixel = __float_as_uint(rs.w);
    Accum a = accum[pixel];
    float4 al = P.w.alb[i], nr = P.w.nrm[i];
    a.color.x = a.color.x + result.x;
    a.color.y = a.color.y + result.y;
    a.color.z = a.color.z + result.z;
    a.albedo = make_float4(a.albedo.x + al.x, a.albedo.y + al.y, a.albedo.z + al.z, a.albedo.w + al.w);
    a.normal = make_float4(a.normal.x + nr.x, a.normal.y + nr.y, a.normal.z + nr.z, a.normal.w + nr.w);
    accum[pixel] = a;
  }
}

// Films (trace.wgsl:2568-2578) for the pixels of this pass.
__global__ void k_films(const __grid_constant__ Pass P,Accum* __restrict__ accum, float4* color, float4* albedo, float4* normal) {
  const uint32_t n = P.w.counters[3];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t pixel = P.w.active[i];
    Accum a = accum[pixel];
    a.color.w = (float)(pass_accum(P) + pass_count(P));
    accum[pixel] = a;
    float count = fmax_(a.color.w, 1.0f);
    v3 nn = divs3(mk3(a.normal.x, a.normal.y, a.normal.z), count);
    color[pixel] = make_float4(a.color.x / count, a.color.y / count, a.color.z / count,
                               P.f.forward[3] > 0.0f ? a.albedo.w / count : 1.0f);
    albedo[pixel] = make_float4(a.albedo.x / count, a.albedo.y / count, a.albedo.z / count, a.albedo.w / count);
    v3 nv = length3(nn) > 1e-6f ? normalize3(nn) : splat3(0.0f);
    normal[pixel] = make_float4(nv.x, nv.y, nv.z, a.normal.w / count);
  }
}

// ------------------------------------------------------------------ host
void check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) throw Refused(std::string(what) + ": out of device memory");
  throw DeviceError(std::string(what) + ": " + cudaGetErrorString(e));
}

int grid_for(const void* kernel, int threads) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0);
  return sms * (per > 0 ? per : 1);
}

// Persistent grids of the traversal kernels for 64, 128 and 256 threads per block.
struct Grids {
  // [threads choice (64, 128, 256)][shared-memory stack entries (0, 8)]
  int trace_closest[3][2] = {}, trace_any[3][2] = {}, shade = 0, shade_inline = 0, flat = 0;
  int shade_hit = 0, shade_lights = 0, shade_lights_inline = 0, shade_bsdf = 0;
  int retry = 0;  // blocks of the retry walks: one per SM (their work is rare)
  int tree_pick = 0, slot[5] = {};  // the light slots, one kind per launch
};
Grids& grids() {
  static Grids g;
  if (g.shade == 0) {
    g.trace_closest[0][0] = grid_for((const void*)k_trace_queue<false, 64, 0>, 64);
    g.trace_closest[1][0] = grid_for((const void*)k_trace_queue<false, 128, 0>, 128);
    g.trace_closest[2][0] = grid_for((const void*)k_trace_queue<false, 256, 0>, 256);
    g.trace_any[0][0] = grid_for((const void*)k_trace_queue<true, 64, 0>, 64);
    g.trace_any[1][0] = grid_for((const void*)k_trace_queue<true, 128, 0>, 128);
    g.trace_any[2][0] = grid_for((const void*)k_trace_queue<true, 256, 0>, 256);
    g.trace_closest[0][1] = grid_for((const void*)k_trace_queue<false, 64, 8>, 64);
    g.trace_closest[1][1] = grid_for((const void*)k_trace_queue<false, 128, 8>, 128);
    g.trace_closest[2][1] = grid_for((const void*)k_trace_queue<false, 256, 8>, 256);
    g.trace_any[0][1] = grid_for((const void*)k_trace_queue<true, 64, 8>, 64);
    g.trace_any[1][1] = grid_for((const void*)k_trace_queue<true, 128, 8>, 128);
    g.trace_any[2][1] = grid_for((const void*)k_trace_queue<true, 256, 8>, 256);
    g.shade = grid_for((const void*)k_shade<true>, kThreads);
    g.shade_inline = grid_for((const void*)k_shade<false>, kThreads);
    g.shade_hit = grid_for((const void*)k_shade_hit, kThreads);
    g.shade_lights = grid_for((const void*)k_shade_lights<true>, kThreads);
    g.shade_lights_inline = grid_for((const void*)k_shade_lights<false>, kThreads);
    g.shade_bsdf = grid_for((const void*)k_shade_bsdf, kThreads);
    g.tree_pick = grid_for((const void*)k_tree_pick, kThreads);
    g.slot[SLOT_SUN] = grid_for((const void*)k_light_slot<SLOT_SUN>, kThreads);
    g.slot[SLOT_SKY] = grid_for((const void*)k_light_slot<SLOT_SKY>, kThreads);
    g.slot[SLOT_EMITTER] = grid_for((const void*)k_light_slot<SLOT_EMITTER>, kThreads);
    g.slot[SLOT_LOOPED] = grid_for((const void*)k_light_slot<SLOT_LOOPED>, kThreads);
    g.slot[SLOT_TREE] = grid_for((const void*)k_light_slot<SLOT_TREE>, kThreads);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g.flat = sms * 8;
    g.retry = sms;
  }
  return g;
}

// The traversal launches for the tuned block size (0: 64, 1: 128, 2: 256 threads).
template <bool ANY, int SHORT>
void launch_trace_queue_short(int sel, const Pass& P, uint32_t which, cudaStream_t st) {
  Grids& g = grids();
  const int k = SHORT > 0 ? 1 : 0;
  const int* grid = ANY ? &g.trace_any[sel][k] : &g.trace_closest[sel][k];
  if (sel == 0)
    k_trace_queue<ANY, 64, SHORT><<<*grid, 64, 0, st>>>(P, which);
  else if (sel == 2)
    k_trace_queue<ANY, 256, SHORT><<<*grid, 256, 0, st>>>(P, which);
  else
    k_trace_queue<ANY, 128, SHORT><<<*grid, 128, 0, st>>>(P, which);
}

template <bool ANY>
void launch_trace_queue(int sel, uint32_t short_stack, const Pass& P, uint32_t which, cudaStream_t st) {
  if (short_stack > 0u)
    launch_trace_queue_short<ANY, 8>(sel, P, which, st);
  else
    launch_trace_queue_short<ANY, 0>(sel, P, which, st);
  k_trace_queue_retry<ANY><<<grids().retry, 128, 0, st>>>(P);
}

int thread_select(uint32_t threads) { return threads == 64u ? 0 : (threads == 256u ? 2 : 1); }

// The deferred light slots one kind per launch, in slot order, each launched
// only where the scene has that kind (the slots k_shade_lights skips without
// a draw: no sun, no sky, no emissive triangles, no looped lights, no tree).
// A black sky's slot adds nothing; it still draws two numbers from a path's
// pcg state, so it is launched for the pcg sampler only.
void launch_light_slots(const Pass& P, cudaStream_t st) {
  Grids& g = grids();
  const bool black_sky = P.v.sky_radiance[0] == 0.0f && P.v.sky_radiance[1] == 0.0f && P.v.sky_radiance[2] == 0.0f;
  if (P.f.sun_color[3] > 0.0f) k_light_slot<SLOT_SUN><<<g.slot[SLOT_SUN], kThreads, 0, st>>>(P, 0u);
  if (P.v.sky_width != 0u && !(black_sky && P.sp.sobol))
    k_light_slot<SLOT_SKY><<<g.slot[SLOT_SKY], kThreads, 0, st>>>(P, 1u);
  if (P.v.emitter_count != 0u) k_light_slot<SLOT_EMITTER><<<g.slot[SLOT_EMITTER], kThreads, 0, st>>>(P, 2u);
  for (uint32_t s = 1u; s <= P.v.looped; ++s)
    k_light_slot<SLOT_LOOPED><<<g.slot[SLOT_LOOPED], kThreads, 0, st>>>(P, 2u + s);
  if (P.slots > 3u + P.v.looped) {
    const uint32_t k = 3u + P.v.looped;
    k_tree_pick<<<g.tree_pick, kThreads, 0, st>>>(P, k);
    k_light_slot<SLOT_TREE><<<g.slot[SLOT_TREE], kThreads, 0, st>>>(P, k);
  }
}

// Path-state buffers for `capacity` paths and `cap` slots per path.
void ensure_wave(pfxt_trace& t, uint32_t capacity, uint32_t cap) {
  size_t need = 0;
  auto add = [&](size_t bytes) {
    size_t at = (need + 255) & ~size_t(255);
    need = at + bytes;
    return at;
  };
  size_t o_ray_o = add(16ull * capacity), o_ray_d = add(16ull * capacity), o_thr = add(16ull * capacity),
         o_res = add(16ull * capacity), o_alb = add(16ull * capacity), o_nrm = add(16ull * capacity),
         o_hit = add(16ull * capacity), o_hitv = add(4ull * capacity), o_sho = add(16ull * capacity * cap),
         o_shd = add(16ull * capacity * cap), o_shc = add(16ull * capacity * cap), o_q0 = add(4ull * capacity),
         o_q1 = add(4ull * capacity), o_sq = add(4ull * capacity * cap), o_act = add(4ull * capacity),
         o_cnt = add(128), o_keys = add(4ull * capacity), o_sorted = add(4ull * capacity),
         o_hist = add(4ull * SORT_BINS), o_cursor = add(4ull * SORT_BINS), o_lit = add(4ull * capacity),
         o_surf = add(144ull * capacity), o_rhist = add(4ull * RAY_BINS), o_rcursor = add(4ull * RAY_BINS),
         o_retry = add(4ull * capacity * (cap > 0 ? cap : 1)), o_eretry = add(4ull * capacity),
         o_pick = add(8ull * capacity);
  if (need > t.wave_bytes) {
    if (t.d_wave) cudaFree(t.d_wave);
    t.d_wave = nullptr;
    t.wave_bytes = 0;
    trace_forget_graphs(t);  // captured passes name the old buffers
    check(cudaMalloc(&t.d_wave, need), "wavefront path state");
    check(cudaMemset(static_cast<char*>(t.d_wave) + o_cnt, 0, 128), "counters");
    t.wave_bytes = need;
  }
  t.wave_counters = reinterpret_cast<uint32_t*>(static_cast<char*>(t.d_wave) + o_cnt);
  t.wave_capacity = capacity;
  char* b = static_cast<char*>(t.d_wave);
  Wave& w = *reinterpret_cast<Wave*>(&t.wave_layout);
  w.ray_o = reinterpret_cast<float4*>(b + o_ray_o);
  w.ray_d = reinterpret_cast<float4*>(b + o_ray_d);
  w.thr = reinterpret_cast<float4*>(b + o_thr);
  w.res = reinterpret_cast<float4*>(b + o_res);
  w.alb = reinterpret_cast<float4*>(b + o_alb);
  w.nrm = reinterpret_cast<float4*>(b + o_nrm);
  w.hit = reinterpret_cast<float4*>(b + o_hit);
  w.hit_v = reinterpret_cast<float*>(b + o_hitv);
  w.sh_o = reinterpret_cast<float4*>(b + o_sho);
  w.sh_d = reinterpret_cast<float4*>(b + o_shd);
  w.sh_c = reinterpret_cast<float4*>(b + o_shc);
  w.queue[0] = reinterpret_cast<uint32_t*>(b + o_q0);
  w.queue[1] = reinterpret_cast<uint32_t*>(b + o_q1);
  w.squeue = reinterpret_cast<uint32_t*>(b + o_sq);
  w.active = reinterpret_cast<uint32_t*>(b + o_act);
  w.counters = reinterpret_cast<uint32_t*>(b + o_cnt);
  w.keys = reinterpret_cast<uint32_t*>(b + o_keys);
  w.sorted = reinterpret_cast<uint32_t*>(b + o_sorted);
  w.hist = reinterpret_cast<uint32_t*>(b + o_hist);
  w.cursor = reinterpret_cast<uint32_t*>(b + o_cursor);
  w.lit = reinterpret_cast<uint32_t*>(b + o_lit);
  w.surf = reinterpret_cast<float4*>(b + o_surf);
  w.rhist = reinterpret_cast<uint32_t*>(b + o_rhist);
  w.rcursor = reinterpret_cast<uint32_t*>(b + o_rcursor);
  w.retry = reinterpret_cast<uint32_t*>(b + o_retry);
  w.eretry = reinterpret_cast<uint32_t*>(b + o_eretry);
  w.pick = reinterpret_cast<float2*>(b + o_pick);
}

// Cache scratch for `pixels` paths: queries, their path indices and
// predictions, training slots, training vertices and records.
CachePass ensure_cache(pfxt_trace& t, uint32_t pixels) {
  CachePass c;
  memset(&c, 0, sizeof(c));
  if (!t.cache) return c;
  pfxt_cache& k = *t.cache;
  const pfxt_cache_settings& s = k.s;
  c.enabled = 1u;
  c.query_bounce = s.query_bounce;
  c.record_bounces = s.record_bounces;
  c.threshold = (uint32_t)std::min(16777216.0, (double)s.train_fraction * 16777216.0);
  c.tcap = std::min<uint32_t>(pixels, (uint32_t)((double)s.train_fraction * pixels * 1.25) + 4096u);
  c.rcap = s.steps * s.batch;
  c.min_roughness = s.min_roughness;
  // the inference runs after the shade of bounce query_last, which the bounce loop must reach
  c.query_last = std::min(s.query_bounce + (s.min_roughness > 0.0f ? s.delay_bounces : 0u),
                          t.spec.total_bounces + 1u);
  c.query_bounce = std::min(c.query_bounce, c.query_last);
  const uint32_t vertices = s.record_bounces + 1u;
  size_t need = 0;
  auto add = [&](size_t bytes) {
    size_t at = (need + 255) & ~size_t(255);
    need = at + bytes;
    return at;
  };
  size_t o_q = add(80ull * pixels), o_cq = add(4ull * pixels), o_pred = add(16ull * pixels),
         o_ts = add(4ull * pixels), o_tv = add(112ull * c.tcap * vertices), o_rec = add(96ull * std::max(c.rcap, 1u)),
         o_x = add(cache_x_bytes(pixels));
  if (need > t.cache_scratch_bytes) {
    if (t.d_cache_scratch) cudaFree(t.d_cache_scratch);
    t.d_cache_scratch = nullptr;
    t.cache_scratch_bytes = 0;
    trace_forget_graphs(t);
    check(cudaMalloc(&t.d_cache_scratch, need), "radiance cache scratch");
    t.cache_scratch_bytes = need;
  }
  char* b = static_cast<char*>(t.d_cache_scratch);
  c.query = reinterpret_cast<float4*>(b + o_q);
  c.cqueue = reinterpret_cast<uint32_t*>(b + o_cq);
  c.pred = reinterpret_cast<float4*>(b + o_pred);
  c.tslot = reinterpret_cast<uint32_t*>(b + o_ts);
  c.tvert = reinterpret_cast<float4*>(b + o_tv);
  c.records = reinterpret_cast<float4*>(b + o_rec);
  c.encoded = reinterpret_cast<uint8_t*>(b + o_x);
  c.cell_ok = k.d_cell_ok;
  for (int j = 0; j < 3; ++j) {
    c.lo[j] = k.grid.lo[j];
    c.inv[j] = k.grid.inv_extent[j];
  }
  return c;
}

// The pass variables (PASS_VAR_BYTES: counters, seed, camera) and their pinned
// host mirror, the side stream and events of the cache inference, and those
// of the extend that runs ahead beside the connect.
void ensure_vars(pfxt_trace& t) {
  if (t.d_vars) return;
  check(cudaMalloc(&t.d_vars, PASS_VAR_BYTES), "pass variables");
  check(cudaHostAlloc(&t.h_vars, PASS_VAR_BYTES, cudaHostAllocDefault), "pass variables");
  check(cudaStreamCreateWithFlags(&t.side, cudaStreamNonBlocking), "side stream");
  check(cudaEventCreateWithFlags(&t.fork_ev, cudaEventDisableTiming), "side stream events");
  check(cudaEventCreateWithFlags(&t.join_ev, cudaEventDisableTiming), "side stream events");
  check(cudaStreamCreateWithFlags(&t.ahead, cudaStreamNonBlocking), "side stream");
  check(cudaEventCreateWithFlags(&t.ahead_fork, cudaEventDisableTiming), "side stream events");
  check(cudaEventCreateWithFlags(&t.ahead_join, cudaEventDisableTiming), "side stream events");
}

void enqueue_pass(pfxt_trace& t, Pass& P, uint32_t count, bool deferred, uint32_t pixels);

}  // namespace

namespace {
// RowTrig of every light row (shade.cuh), by the functions and expressions the
// importance of a row used to evaluate at each visit.
__global__ void k_light_trig(const __grid_constant__ ShadeView V, uint32_t rows, float4* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    LightRow r = load_light(V, i);
    float theta_o = r.c.w, theta_e = r.d.x;
    out[2u * i] = make_float4(cos_(theta_o), sin_(theta_o), cos_(theta_o + theta_e), cos_(theta_e - theta_o));
    float cone = f2u(r.a.w) == 1u ? acos_(clamp_(-r.d.y / r.d.x, -1.0f, 1.0f)) : SH_PI / 2.0f;
    out[2u * i + 1u] = make_float4(cone, cos_(cone), cos_(0.0f), sin_(0.0f));
  }
}
}  // namespace

void light_trig_init(pfxt_trace& t) {
  uint32_t rows = std::max<uint32_t>(t.light_rows, 1u);
  void* d = nullptr;
  check(cudaMalloc(&d, (size_t)rows * 32u), "light-row trigonometry");
  t.owned.push_back(d);
  t.shade.light_trig = static_cast<const float4*>(d);
  if (t.light_rows) {
    k_light_trig<<<(t.light_rows + 127u) / 128u, 128, 0, t.stream>>>(t.shade, t.light_rows, static_cast<float4*>(d));
    check(cudaGetLastError(), "light-row trigonometry");
  }
  check(cudaStreamSynchronize(t.stream), "light-row trigonometry");
}

void trace_forget_graphs(pfxt_trace& t) {
  for (auto& e : t.graphs) cudaGraphExecDestroy(e.exec);
  t.graphs.clear();
}

static_assert(sizeof(Wave) <= sizeof(((pfxt_trace*)nullptr)->wave_layout), "wave layout storage");

void trace_sample(pfxt_trace& t, uint32_t count, uint32_t seed) {
  if (count == 0) return;
  uint32_t pixels = t.width * t.height;
  uint32_t light_slots = 1u + t.shade.looped + (t.shade.tree > 0u ? 1u : 0u);
  uint32_t slots = 2u + light_slots;
  uint32_t cap = std::min(slots, CAP_MAX);
  bool deferred = slots <= CAP_MAX && t.shadow_queue;
  ensure_wave(t, pixels, cap);
  Pass P;
  memset(&P, 0, sizeof(P));
  P.f = t.base;  // the accumulated samples, the count, the seed and the camera travel in P.vars
  P.f.size[2] = 0u;
  P.f.size[3] = 0u;
  P.f.counts[2] = 0u;
  for (int k = 0; k < 3; ++k) P.f.origin[k] = P.f.forward[k] = P.f.right[k] = P.f.up[k] = 0.0f;
  P.sp = t.spec;
  P.v = t.shade;
  P.s = t.view;
  P.w = *reinterpret_cast<Wave*>(&t.wave_layout);
  P.cap = cap;
  P.deferred = deferred ? 1u : 0u;
  P.light_rows = t.light_rows;
  P.slots = slots;
  P.width = t.width;
  P.height = t.height;
  P.c = ensure_cache(t, pixels);
  P.ray_bins = t.sort_rays ? RAY_BINS : 0u;
  for (int k = 0; k < 3; ++k) {
    float extent = t.bounds_hi[k] - t.bounds_lo[k];
    P.scene_lo[k] = t.bounds_lo[k];
    P.scene_inv[k] = extent > 0.0f ? 1.0f / extent : 0.0f;
  }
  P.bins = t.sort_shading ? 2u * std::max<uint32_t>(std::min<uint32_t>(t.shade.material_count + 1u, SORT_BINS / 2u), 2u)
                          : 0u;
  ensure_vars(t);
  P.vars = t.d_vars;
  t.h_vars[0] = t.samples;
  t.h_vars[1] = count;
  t.h_vars[2] = seed;
  t.h_vars[3] = 0u;
  {
    const float* rows[4] = {t.base.origin, t.base.forward, t.base.right, t.base.up};
    float* cam = reinterpret_cast<float*>(t.h_vars + 4);
    for (int r = 0; r < 4; ++r) {
      for (int k = 0; k < 3; ++k) cam[4 * r + k] = rows[r][k];
      cam[4 * r + 3] = 0.0f;
    }
  }
  cudaStream_t st = t.stream;
  if (t.samples == 0) check(cudaMemsetAsync(t.d_accum, 0, (size_t)pixels * sizeof(Accum), st), "accumulation reset");
  if (!t.use_graphs) {
    enqueue_pass(t, P, count, deferred, pixels);
  } else {
    // the launch sequence depends only on P (with the pass's variables in
    // device memory), the sample count and the buffers: captured once, replayed
    std::vector<unsigned char> key(sizeof(P) + 64);
    memcpy(key.data(), &P, sizeof(P));
    uint64_t extra[8] = {count, (uint64_t)(uintptr_t)t.d_mask, (uint64_t)(uintptr_t)t.cache, deferred ? 1u : 0u,
                         t.cache ? (uint64_t)t.cache->s.steps : 0u, t.cache ? (uint64_t)t.cache->s.batch : 0u,
                         (uint64_t)(uintptr_t)t.d_accum,
                         (uint64_t)pixels | ((uint64_t)t.trace_threads << 32) | ((uint64_t)t.split_shade << 48) |
                             ((uint64_t)t.short_stack << 52) | ((uint64_t)t.slot_kernels << 60)};
    memcpy(key.data() + sizeof(P), extra, sizeof(extra));
    cudaGraphExec_t exec = nullptr;
    for (auto& e : t.graphs)
      if (e.key == key) exec = e.exec;
    if (!exec) {
      check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "pass capture");
      cudaGraph_t graph = nullptr;
      try {
        enqueue_pass(t, P, count, deferred, pixels);
      } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      check(cudaStreamEndCapture(st, &graph), "pass capture");
      // the pass's kernel launches: the graph's kernel nodes
      uint32_t kernels = 0;
      size_t nodes = 0;
      if (cudaGraphGetNodes(graph, nullptr, &nodes) == cudaSuccess && nodes > 0) {
        std::vector<cudaGraphNode_t> list(nodes);
        if (cudaGraphGetNodes(graph, list.data(), &nodes) == cudaSuccess)
          for (size_t k = 0; k < nodes; ++k) {
            cudaGraphNodeType type;
            if (cudaGraphNodeGetType(list[k], &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) ++kernels;
          }
      }
      cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      check(e, "pass graph");
      if (t.graphs.size() >= 8) {
        cudaGraphExecDestroy(t.graphs.front().exec);
        t.graphs.erase(t.graphs.begin());
      }
      t.graphs.push_back(GraphEntry{std::move(key), exec, kernels});
      t.graph_captures += 1u;
    }
    for (auto& e : t.graphs)
      if (e.exec == exec) t.pass_kernels = e.kernels;
    check(cudaGraphLaunch(exec, st), "pass graph launch");
  }
  check(cudaGetLastError(), "tracer launch");
  check(cudaStreamSynchronize(st), "tracer pass");
  if (P.c.enabled) {
    uint32_t c[3];
    check(cudaMemcpy(c, P.w.counters + 5, 12, cudaMemcpyDeviceToHost), "cache counters");
    t.cache->last_queries = c[0];
    t.cache->last_training_paths = std::min(c[1], P.c.tcap);
    t.cache->last_records = std::min(c[2], P.c.rcap);
    float loss = 0.0f;
    check(cudaMemcpy(&loss, t.cache->d_loss, 4, cudaMemcpyDeviceToHost), "cache loss");
    t.cache->last_loss = loss / (3.0f * (float)t.cache->s.batch);
    cache_check_error(*t.cache);
  }
  t.samples += count;
}

namespace {

// One pass's operations on t.stream: the variables' copy, the queues' reset,
// the samples' bounce loops, the films, and the cache's training.
void enqueue_pass(pfxt_trace& t, Pass& P, uint32_t count, bool deferred, uint32_t pixels) {
  Grids& g = grids();
  cudaStream_t st = t.stream;
  check(cudaMemcpyAsync(t.d_vars, t.h_vars, PASS_VAR_BYTES, cudaMemcpyHostToDevice, st), "pass variables");
  check(cudaMemsetAsync(P.w.counters, 0, 32, st), "counters");  // queues; the ray totals at [8..11] persist
  k_collect<<<g.flat, 256, 0, st>>>(P, t.d_accum, t.d_mask);
  bool inferred = false;
  // A bounce's extend: empty the next queues, sort the rays (when chosen), walk.
  auto extend = [&](const Pass& Q, uint32_t cur, cudaStream_t s) {
    k_reset<<<1, 32, 0, s>>>(Q, cur);
    if (Q.ray_bins && Q.bounce > 0u) {
      k_sort_count<true><<<g.flat, 256, 0, s>>>(Q, cur);
      k_sort_place<true><<<g.flat, 256, 0, s>>>(Q, cur);
    }
    launch_trace_queue<false>(thread_select(t.trace_threads), t.short_stack, Q, cur, s);
  };
  // With deferred light slots, the extend of bounce b + 1 needs only the rays
  // that bounce b's BSDF kernel wrote, and the connect of bounce b only the
  // shadow queue: the extend runs ahead on its own stream beside the connect
  // (its own work counter, retry list and queue count), and the bounce joins
  // it before shading.
  const bool ahead = TRACE_AHEAD && deferred;
  for (uint32_t sample = 0; sample < count; ++sample) {
    P.sample = sample;
    if (P.c.enabled) k_cache_begin<<<1, 32, 0, st>>>(P);
    k_gen<<<g.flat, 256, 0, st>>>(P);
    k_seed_counts<<<1, 32, 0, st>>>(P);
    const uint32_t last = t.spec.total_bounces + 1u;
    for (uint32_t bounce = 0; bounce <= last; ++bounce) {
      uint32_t cur = bounce & 1u;
      P.bounce = bounce;
      if (ahead && bounce > 0u)
        check(cudaStreamWaitEvent(st, t.ahead_join, 0), "extend join");
      else
        extend(P, cur, st);
      if (P.bins) {
        k_sort_count<false><<<g.flat, 256, 0, st>>>(P, cur);
        k_sort_place<false><<<g.flat, 256, 0, st>>>(P, cur);
      }
      if (t.split_shade) {
        k_shade_hit<<<g.shade_hit, kThreads, 0, st>>>(P, cur);
        if (deferred && t.slot_kernels)
          launch_light_slots(P, st);
        else if (deferred)
          k_shade_lights<true><<<g.shade_lights, kThreads, 0, st>>>(P);
        else
          k_shade_lights<false><<<g.shade_lights_inline, kThreads, 0, st>>>(P);
        k_shade_bsdf<<<g.shade_bsdf, kThreads, 0, st>>>(P, cur);
      } else if (deferred) {
        k_shade<true><<<g.shade, kThreads, 0, st>>>(P, cur);
      } else {
        k_shade<false><<<g.shade_inline, kThreads, 0, st>>>(P, cur);
      }
      if (P.c.enabled && bounce == P.c.query_last) {
        // Every query is written by now, and the later bounces (training and
        // fallback paths) neither read the queries nor write the predictions,
        // so the inference runs beside them until the accumulation.
        check(cudaEventRecord(t.fork_ev, st), "inference fork");
        check(cudaStreamWaitEvent(t.side, t.fork_ev, 0), "inference fork");
        cache_infer_launch(*t.cache, P.c.query, P.w.counters + 5, pixels, P.c.cqueue, P.c.pred, P.c.encoded, t.side);
        check(cudaEventRecord(t.join_ev, t.side), "inference join");
        inferred = true;
      }
      if (deferred) {
        k_rewind<<<1, 32, 0, st>>>(P);
        if (ahead && bounce < last) {
          Pass Q = P;
          Q.bounce = bounce + 1u;
          check(cudaEventRecord(t.ahead_fork, st), "extend fork");
          check(cudaStreamWaitEvent(t.ahead, t.ahead_fork, 0), "extend fork");
          extend(Q, (bounce + 1u) & 1u, t.ahead);
          check(cudaEventRecord(t.ahead_join, t.ahead), "extend join");
        }
        launch_trace_queue<true>(thread_select(t.trace_threads), t.short_stack, P, 0u, st);
      }
    }
    if (inferred) check(cudaStreamWaitEvent(st, t.join_ev, 0), "inference join");
    inferred = false;
    k_finish<<<g.flat, 256, 0, st>>>(P, t.d_accum);
  }
  k_films<<<g.flat, 256, 0, st>>>(P, t.d_accum, t.d_color, t.d_albedo, t.d_normal);
  if (P.c.enabled) {
    // online training on this pass's records, then the fallback cells
    for (uint32_t s = 0; s < t.cache->s.steps; ++s)
      cache_train_launch(*t.cache, P.c.records, P.w.counters + 7, P.c.rcap, s * t.cache->s.batch, st, true, 0);
    cache_cells_launch(*t.cache, st);
  }
}

// measure (converge.wgsl:9-30): the half-buffer error of every pixel against
// its snapshot of the previous round.  snaps: 2 float4 per pixel (mean, info).
__global__ void k_measure(const Accum* __restrict__ accum, float4* __restrict__ snaps, uint32_t W, uint32_t H) {
  uint32_t n = W * H;
  for (uint32_t index = blockIdx.x * blockDim.x + threadIdx.x; index < n; index += gridDim.x * blockDim.x) {
    Accum sum = accum[index];
    float count = sum.color.w;
    if (count <= 0.0f) {
      snaps[2 * index + 1].y = 0.0f;
      continue;
    }
    float now[4] = {sum.color.x / count, sum.color.y / count, sum.color.z / count, sum.albedo.w / count};
    float4 mean = snaps[2 * index];
    float prior = snaps[2 * index + 1].x;
    float m[4] = {mean.x, mean.y, mean.z, mean.w};
    float error = 1e9f;
    if (prior > 0.0f && count > prior) {
      float scale = sqrtf(1.0f / count) / sqrtf(1.0f / prior + 1.0f / (count - prior));
      float gap[4];
      for (int k = 0; k < 4; ++k) {
        float rest = (now[k] * count - m[k] * prior) / (count - prior);
        gap[k] = abs_(m[k] - rest) * scale;
      }
      error = (gap[0] + gap[1] + gap[2]) / (1e-4f + sqrtf(fmax_(now[0] + now[1] + now[2], 0.0f))) + gap[3];
    }
    snaps[2 * index] = make_float4(now[0], now[1], now[2], now[3]);
    snaps[2 * index + 1] = make_float4(count, error, 0.0f, 0.0f);
  }
}

// mark (converge.wgsl:32-51): stop a pixel whose 3x3 neighbourhood error is
// under the threshold once it has min_samples; count the pixels still running
// (warp-aggregated into one atomic per warp).
__global__ void k_mark(Accum* __restrict__ accum, const float4* __restrict__ snaps, uint32_t W, uint32_t H,
                       uint32_t min_samples, float threshold, uint32_t* running) {
  uint32_t n = W * H;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t index = base + threadIdx.x;
    bool run = false;
    if (index < n) {
      float count = accum[index].color.w;
      if (count > 0.0f) {
        int gx = (int)(index % W), gy = (int)(index / W);
        float worst = 0.0f;
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int x = min(max(gx + dx, 0), (int)W - 1);
            int y = min(max(gy + dy, 0), (int)H - 1);
            worst = fmax_(worst, __ldg(&snaps[2 * ((uint32_t)y * W + (uint32_t)x) + 1].y));
          }
        if (count >= (float)min_samples && worst < threshold)
          accum[index].color.w = -count;
        else
          run = true;
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, run);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(running, (uint32_t)__popc(m));
  }
}

}  // namespace

// One adaptive round split in its two kernels, for a frame whose pixels are
// shared between tracers (one per GPU): measure, then, after the caller has
// written the errors of neighbouring rows other tracers own into the
// snapshots, mark.  `first` clears the snapshots (a new adaptive render).
void trace_adaptive_measure(pfxt_trace& t, bool first) {
  cudaStream_t st = t.stream;
  if (first) check(cudaMemsetAsync(t.d_snaps, 0, (size_t)t.width * t.height * 32, st), "snapshots");
  k_measure<<<grids().flat, 256, 0, st>>>(t.d_accum, t.d_snaps, t.width, t.height);
  check(cudaGetLastError(), "measure");
  check(cudaStreamSynchronize(st), "measure");
}

uint32_t trace_adaptive_mark(pfxt_trace& t, uint32_t min_samples, float threshold) {
  cudaStream_t st = t.stream;
  check(cudaMemsetAsync(t.d_running, 0, 4, st), "running count");
  k_mark<<<grids().flat, 256, 0, st>>>(t.d_accum, t.d_snaps, t.width, t.height, min_samples, threshold, t.d_running);
  check(cudaGetLastError(), "mark");
  uint32_t running = 0;
  check(cudaMemcpyAsync(&running, t.d_running, 4, cudaMemcpyDeviceToHost, st), "running count");
  check(cudaStreamSynchronize(st), "mark");
  return running;
}

// Trace::sample_adaptive_kept without a keeper (adaptive.rs:136-325).
void trace_sample_adaptive(pfxt_trace& t, const pfxt_adaptive& a, uint32_t seed, pfxt_round* rounds, uint32_t cap,
                           uint32_t* written, const AdaptiveKeeping* keeping) {
  if (!adaptive_valid(a))
    throw Invalid("adaptive sampling needs a positive threshold, a growth over 1 and at least 2 samples");
  uint32_t pixels = t.width * t.height;
  cudaStream_t st = t.stream;
  std::vector<uint32_t> targets = adaptive_rounds(a);
  std::vector<pfxt_round> reached;
  if (keeping && keeping->resuming) {
    // the caller restored the accumulation, the films, the snapshots and the sample count
    if (keeping->resumed.size() >= targets.size())
      throw Invalid("the checkpoint holds no adaptive rounds for this render");
    reached = keeping->resumed;
  } else {
    t.samples = 0;
    check(cudaMemsetAsync(t.d_snaps, 0, (size_t)pixels * 32, st), "snapshots");
  }
  Grids& g = grids();
  uint32_t n = 0;
  for (const pfxt_round& r : reached) {
    if (rounds && n < cap) rounds[n] = r;
    ++n;
  }
  for (size_t step = reached.size(); step < targets.size(); ++step) {
    uint32_t target = targets[step];
    uint32_t count = target > t.samples ? target - t.samples : 0u;
    if (keeping && keeping->due) {
      // one sample at a time, offering a checkpoint after each (adaptive.rs:258-277)
      for (uint32_t s = 0; s < count; ++s) {
        trace_sample(t, 1u, seed);
        if (keeping->due(t.samples)) keeping->keep(reached);
      }
    } else {
      trace_sample(t, count, seed);
    }
    check(cudaMemsetAsync(t.d_running, 0, 4, st), "running count");
    k_measure<<<g.flat, 256, 0, st>>>(t.d_accum, t.d_snaps, t.width, t.height);
    if (step > 0) k_mark<<<g.flat, 256, 0, st>>>(t.d_accum, t.d_snaps, t.width, t.height, a.min_samples, a.threshold,
                                                  t.d_running);
    uint32_t running = 0;
    check(cudaMemcpyAsync(&running, t.d_running, 4, cudaMemcpyDeviceToHost, st), "running count");
    check(cudaStreamSynchronize(st), "convergence");
    uint64_t active = step > 0 ? (uint64_t)running : (uint64_t)pixels;
    pfxt_round round{target, 0u, active};
    reached.push_back(round);
    if (rounds && n < cap) rounds[n] = round;
    ++n;
    if (active == 0) break;
  }
  *written = std::min(n, cap);
}

}  // namespace pfxt
