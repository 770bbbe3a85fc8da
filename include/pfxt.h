/*
 * pfxt.h - C ABI of the B200 path tracer (libpfxtrace.so).
 *
 * It stands in for the trace crate of pfx (crates/trace): a scene, a camera and
 * a sample budget go in, RGBA32F films come out.  Each entry point below names
 * the reference interface it replaces (file:line inside the pfx repository).
 *
 * Conventions (crates/trace/src/gpu.rs:269-307 TraceError, docs/trace.md:121):
 *   - every call returns an int status, PFXT_OK (0) or a PFXT_ERR_* code; the
 *     message of the last failure on the calling thread is pfxt_last_error();
 *   - the library owns all device memory; host arrays passed in are copied;
 *   - a pfxt_trace handle is used by one thread at a time (the Rust Trace takes
 *     &mut self); calls block until the GPU work they start has finished, as
 *     Trace::sample does (docs/trace.md:466), except the *_device entry points,
 *     which enqueue on the caller's stream and return.
 */
#ifndef PFXT_H
#define PFXT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFXT_ABI_VERSION 1

#define PFXT_OK 0
#define PFXT_ERR_INVALID 1 /* invalid scene, settings or arguments (TraceError::Setup) */
#define PFXT_ERR_REFUSED 2 /* the device refused: no CUDA device, out of memory (TraceError::Refused) */
#define PFXT_ERR_CUDA 3    /* a CUDA call failed */
#define PFXT_ERR_DEVICE 4  /* a kernel set its error word (a bounded loop ran out) */

/* ------------------------------------------------------------ scene input */

/* TriangleDetail without the second uv set (crates/trace/src/detail.rs:7-13). */
typedef struct pfxt_triangle {
  float v[3][3];
  float n[3][3];
  float uv[3][2];
  uint32_t material;
} pfxt_triangle;

typedef struct pfxt_mesh {
  const pfxt_triangle* triangles;
  uint32_t count;
} pfxt_mesh;

/* Instance (detail.rs:53-60); meshes shared by several instances become one
 * bottom-level BVH, as Arc-shared triangle lists do in levels.rs:252-350. */
typedef struct pfxt_instance {
  uint32_t mesh;
  uint32_t shadow_only;  /* Instance::shadow_only -> SHADOW_ONLY */
  uint32_t two_sided;    /* Instance::two_sided; 0 sets ONE_SIDED */
  uint32_t casts_shadow; /* InstanceSurface::casts_shadow; 0 sets CASTS_NO_SHADOW */
  float transform[16];   /* column-major affine 4x4 (detail.rs Transform) */
} pfxt_instance;

/* The hot material record fields (materials/src/material.rs:827-843). */
typedef struct pfxt_material {
  float base[3];
  float roughness;
  float metalness, specular, clearcoat, clearcoat_roughness;
  float sheen, transmission, ior, dispersion;
  float thickness, subsurface, thin_film, thin_film_ior;
  float subsurface_tint[3];
  float absorption;
  float emission[3];
  float thin_film_amount;
  float fresnel_power;
  float pad[3];
} pfxt_material;

#define PFXT_LIGHT_POINT 0u
#define PFXT_LIGHT_SPOT 1u
#define PFXT_LIGHT_RECT 2u
#define PFXT_LIGHT_DISC 3u

/* LocalLight (crates/trace/src/lights.rs:11-39). */
typedef struct pfxt_light {
  uint32_t shape;     /* PFXT_LIGHT_* */
  uint32_t shadow;    /* casts shadows */
  uint32_t two_sided; /* rect and disc */
  uint32_t pad;
  float position[3];
  float colour[3];
  float intensity;
  float radius; /* point/spot source radius */
  float range;  /* point/spot range; rect and disc are unlimited */
  float direction[3]; /* spot axis, or disc normal */
  float inner_deg, outer_deg;  /* spot cone */
  float half_u[3], half_v[3];  /* rect half extents */
  float disc_radius;
} pfxt_light;

/* Camera (gpu.rs:173-179). */
typedef struct pfxt_camera {
  float origin[3];
  float forward[3];
  float right[3];
  float up[3];
} pfxt_camera;

/* Sun (gpu.rs:231-236) plus Detail::sun_radius_deg. */
typedef struct pfxt_sun {
  float direction[3];
  float color[3];
  float intensity;
  float radius_deg;
} pfxt_sun;

typedef struct pfxt_scene {
  const pfxt_triangle* triangles; /* world triangles (not instanced) */
  uint32_t triangle_count;
  const pfxt_mesh* meshes;
  uint32_t mesh_count;
  const pfxt_instance* instances;
  uint32_t instance_count;
  const pfxt_material* materials;
  uint32_t material_count;
  const pfxt_light* lights;
  uint32_t light_count;
  float sky[3];        /* uniform environment radiance; 0 = black sky */
  uint32_t sky_width;  /* sky CDF columns (the reference uses 256) */
  uint32_t sky_height; /* sky CDF rows (the reference uses 128) */
  uint32_t pad;
  pfxt_camera camera;
  pfxt_sun sun;
} pfxt_scene;

#define PFXT_SAMPLER_PCG 0u
#define PFXT_SAMPLER_SOBOL 1u
#define PFXT_PROJECTION_PERSPECTIVE 0u
#define PFXT_PROJECTION_ORTHOGRAPHIC 1u
#define PFXT_PROJECTION_EQUIRECT 2u

/* Detail settings that specialise the tracer (detail.rs:374-455, gpu.rs:1140-1196). */
typedef struct pfxt_settings {
  uint32_t bounces[4];     /* total, diffuse, glossy, transmission (Bounces) */
  uint32_t sampler;        /* PFXT_SAMPLER_* */
  uint32_t sobol_samples;  /* Sampler::Sobol { samples } */
  float clamp_indirect;    /* CLAMP_INDIRECT, 0 = off */
  float filter_glossy;     /* FILTER_GLOSSY, 0 = off */
  uint32_t projection;     /* PFXT_PROJECTION_* */
  float ortho[2];          /* orthographic width, height */
  float lens[4];           /* shift x, shift y, aperture, focus distance (Lens) */
  uint32_t pad;
} pfxt_settings;

/* ------------------------------------------------- packed scene buffers
 * The byte layouts of SceneBuffers (gpu.rs:412-436): the seam at which a host
 * that packs its own buffers hands them over. */
typedef struct pfxt_buffers {
  const void* triangles; size_t triangles_bytes;     /* GpuTriangle, 96 B each, BVH slot order */
  const void* nodes; size_t nodes_bytes;             /* Node, 48 B each */
  const void* materials; size_t materials_bytes;     /* Hot records, 128 B each, row 0 = effects */
  const void* uv; size_t uv_bytes;                   /* [v0 v1 v2 0] per triangle */
  const void* surfaces; size_t surfaces_bytes;       /* GpuSurface, 176 B each, record 0 = world */
  const void* emitters; size_t emitters_bytes;       /* GpuEmitter, 64 B, entry 0 = header */
  const void* emitter_cdf; size_t emitter_cdf_bytes; /* f32 per emitter */
  const void* lights; size_t lights_bytes;           /* GpuLight, 64 B, tree rows after the lights */
  uint32_t triangle_count, shape_count, emitter_count, light_count;
  const float* sky_rows;    /* sky_height floats */
  const float* sky_columns; /* sky_width * sky_height floats */
  uint32_t sky_width, sky_height;
  float sky_radiance[3];
  float sky_sun_probability;
  const float* sobol; /* RGBA32F table, 256 patterns x sobol_length, or NULL for PCG */
  uint32_t sobol_length;
  uint32_t max_depth; /* deepest traversal stack the node array can need */
} pfxt_buffers;

typedef struct pfxt_scene_blobs pfxt_scene_blobs;
typedef struct pfxt_trace pfxt_trace;

/* ------------------------------------------------------------ ray batches */
typedef struct pfxt_ray {
  float origin[3];
  float tmax;     /* limit: 1e20 for camera rays in scene(), the shadow limit for occluded() */
  float direction[3];
  uint32_t pad;
} pfxt_ray; /* 32 bytes */

typedef struct pfxt_hit {
  float t;        /* hit distance; tmax when nothing was hit */
  uint32_t slot;  /* triangle slot (Hit.surface) */
  uint32_t record;/* instance record (Hit.record), 0 = world */
  uint32_t hit;   /* 1 when a triangle was hit */
} pfxt_hit; /* 16 bytes */

/* Rounds (adaptive.rs:73-77). */
typedef struct pfxt_round {
  uint32_t samples;
  uint32_t pad;
  uint64_t active;
} pfxt_round;

/* Adaptive (adaptive.rs:10-15). */
typedef struct pfxt_adaptive {
  float threshold;
  uint32_t min_samples;
  uint32_t max_samples;
  float growth;
} pfxt_adaptive;

/* ---------------------------------------------------------------- library */
int pfxt_abi_version(void);
/* Message of the last failed call on this thread; "" when none. */
const char* pfxt_last_error(void);
/* Number of CUDA devices, or a negative value when the runtime has none. */
int pfxt_device_count(void);

/* SceneBuffers::build (crates/trace/src/gpu.rs:566-1061): BVH layout
 * (bvh.rs:95-266, levels.rs:225-470), light tree (tree.rs:220-395), light rows
 * and emitter CDF (lights.rs:182-243, 391-440), material records
 * (record.rs:57-180), sky CDF (sky.rs:212-275) and the Sobol table
 * (sobol.rs:109-153).  Host only; no device is needed. */
int pfxt_scene_build(const pfxt_scene* scene, const pfxt_settings* settings,
                     pfxt_scene_blobs** out);
void pfxt_scene_free(pfxt_scene_blobs* blobs);
/* The packed buffers of a built scene (pointers stay valid until pfxt_scene_free). */
int pfxt_scene_buffers(const pfxt_scene_blobs* blobs, pfxt_buffers* out);
/* Triangle slot order of the world triangles (Bvh::order, bvh.rs:38). */
int pfxt_scene_order(const pfxt_scene_blobs* blobs, const uint32_t** order, uint32_t* count);

/* Trace::new_detailed (crates/trace/src/gpu.rs:1926-2360): uploads the scene
 * and allocates the 48 B/pixel accumulation and the three films. */
int pfxt_create(const pfxt_buffers* buffers, const pfxt_scene* view, const pfxt_settings* settings,
                uint32_t width, uint32_t height, pfxt_trace** out);
void pfxt_destroy(pfxt_trace* trace);

/* Trace::set_camera / set_lens / set_projection (gpu.rs:2817-2890); they
 * restart the accumulation. */
int pfxt_set_camera(pfxt_trace* trace, const pfxt_camera* camera);
int pfxt_set_lens(pfxt_trace* trace, const float lens[4]);
/* Trace::set_window (gpu.rs:2834): full frame size and this tile's origin. */
int pfxt_set_window(pfxt_trace* trace, const uint32_t full[2], const uint32_t origin[2]);

/* Trace::sample (gpu.rs:2942): `count` more samples per pixel with `seed`. */
int pfxt_sample(pfxt_trace* trace, uint32_t count, uint32_t seed);
/* Trace::sample_paced (gpu.rs:2951-3110): the same samples taken one pass at a
 * time, `between(user, ms)` called after each with the pass's device time (the
 * reference reports each settled slice to `between`; it slices passes to keep
 * a display responsive, which a compute GPU does not need).  The image equals
 * pfxt_sample's.  *wall_ms (may be NULL) receives the host time of the call. */
typedef void (*pfxt_between)(void* user, double milliseconds);
int pfxt_sample_paced(pfxt_trace* trace, uint32_t count, uint32_t seed, pfxt_between between, void* user,
                      double* wall_ms);
/* Trace::samples (gpu.rs:3233). */
uint32_t pfxt_samples(const pfxt_trace* trace);
/* Trace::sample_adaptive (adaptive.rs:112-325): rounds of samples with the
 * per-pixel convergence test between them; writes up to `cap` rounds. */
int pfxt_sample_adaptive(pfxt_trace* trace, const pfxt_adaptive* adaptive, uint32_t seed,
                         pfxt_round* rounds, uint32_t cap, uint32_t* written);
/* Keeper (checkpoint.rs:30-34) as callbacks: `resume` (NULL for none) is the
 * checkpoint Keeper::resume hands back; `due(user, samples)` is Keeper::due,
 * nonzero when a checkpoint is due after `samples` samples (NULL: never);
 * `keep(user, bytes, length)` is Keeper::keep, handed a checkpoint in the
 * pfxt_save layout with the adaptive rounds and snapshots (the bytes live for
 * the call only); it returns 0 when the checkpoint is kept. */
typedef struct pfxt_keeper {
  void* user;
  const void* resume;
  size_t resume_length;
  int (*due)(void* user, uint32_t samples);
  int (*keep)(void* user, const void* bytes, size_t length);
} pfxt_keeper;
/* Trace::sample_adaptive_kept (adaptive.rs:136-325): pfxt_sample_adaptive,
 * resumed from `keeper->resume` when given (its rounds are written first) and,
 * with a keeper that can be due, one sample at a time with a checkpoint under
 * `key` offered after each.  The rounds and the image equal an uninterrupted
 * pfxt_sample_adaptive's. */
int pfxt_sample_adaptive_kept(pfxt_trace* trace, const pfxt_adaptive* adaptive, uint32_t seed, const char* key,
                              const pfxt_keeper* keeper, pfxt_round* rounds, uint32_t cap, uint32_t* written);
/* One adaptive round in its two steps, measure then mark (converge.wgsl:9-51,
 * run by adaptive.rs:282-307 after every round), for a frame whose 8-row
 * strips are shared between several tracers (one per GPU, each sampling its
 * own strips through pfxt_set_pixel_mask).  Between the two steps the caller
 * writes into the snapshots the errors of the rows next to its strips that
 * other tracers own (a one-row halo per strip edge), so mark's 3x3 maximum
 * sees what a single tracer of the whole frame sees.  pfxt_adaptive_measure
 * with `first` nonzero clears the snapshots (a new adaptive render);
 * pfxt_adaptive_mark stops converged pixels and returns this tracer's running
 * count; the frame's count is the sum over tracers. */
int pfxt_adaptive_measure(pfxt_trace* trace, uint32_t first);
int pfxt_adaptive_mark(pfxt_trace* trace, uint32_t min_samples, float threshold, uint32_t* running);
/* The snapshots in device memory: width*height records of 8 floats (mean rgb,
 * mean coverage, samples, error, 0, 0), the error at float 5 of a record.
 * Valid until pfxt_destroy. */
int pfxt_adaptive_snaps_device(pfxt_trace* trace, float** snaps);
/* Sample only the pixels whose mask byte (width*height host bytes) is
 * non-zero, or every pixel with NULL; restarts the accumulation.  A pixel's
 * samples depend only on the pixel, the sample index and the seed
 * (trace.wgsl:2503-2579), so a masked pixel's value equals the whole frame's. */
int pfxt_set_pixel_mask(pfxt_trace* trace, const uint8_t* mask);
/* Adaptive::rounds (adaptive.rs:46-63). */
int pfxt_adaptive_rounds(const pfxt_adaptive* adaptive, uint32_t* rounds, uint32_t cap,
                         uint32_t* written);
/* Trace::readback (gpu.rs:3240): RGBA32F colour, albedo and normal films,
 * width*height*4 floats each; any pointer may be NULL. */
int pfxt_readback(pfxt_trace* trace, float* color, float* albedo, float* normal);
/* The three films in device memory (RGBA32F, width*height*4 floats each), as
 * the reference hands its colour/albedo/normal textures to the denoiser
 * without a readback (gpu.rs:328-330).  Valid until pfxt_destroy. */
int pfxt_films_device(pfxt_trace* trace, float** color, float** albedo, float** normal);
/* Trace::sample_counts (adaptive.rs:328): |accum.color.w| per pixel. */
int pfxt_sample_counts(pfxt_trace* trace, uint32_t* counts);
/* The raw 48 B/pixel accumulation (Accum, trace.wgsl:84). */
int pfxt_read_accum(pfxt_trace* trace, float* accum);

/* scene() closest hit (crates/trace/src/trace.wgsl:999-1075) over a batch of
 * rays in host memory; the parity entry for identical ray batches. */
int pfxt_trace_rays(pfxt_trace* trace, const pfxt_ray* rays, uint32_t count, pfxt_hit* hits);
/* occluded() any hit (trace.wgsl:1096-1168); blocked[i] = 1 when ray i is
 * blocked before its tmax. */
int pfxt_occluded(pfxt_trace* trace, const pfxt_ray* rays, uint32_t count, uint8_t* blocked);
/* The same two queries on device memory, enqueued on `stream` (a
 * cudaStream_t, NULL = the legacy default stream); no host synchronisation. */
int pfxt_trace_rays_device(pfxt_trace* trace, const pfxt_ray* rays, uint32_t count,
                           pfxt_hit* hits, void* stream);
int pfxt_occluded_device(pfxt_trace* trace, const pfxt_ray* rays, uint32_t count,
                         uint32_t* blocked, void* stream);

/* Any-hit queries that allocate nothing, for callers that cannot call
 * cudaMalloc (a host whose own allocator owns the device heap, or code that must
 * not allocate while GPU work is in flight).  No counterpart in the reference.
 * `rays` and `blocked` (one byte per ray, 1 = blocked) are device memory; the
 * call enqueues on `stream` and returns.  Its scratch (the traversal work
 * counter and the 32-bit flag words) lives in fixed device arrays sized for
 * PFXT_NOALLOC_MAX_RAYS rays, which every GPU that loads the library holds until
 * exit; larger batches are refused with PFXT_ERR_INVALID.  All calls share the
 * arrays: calls whose GPU work overlaps race.  The handle's device must be
 * current.  CUDA loads a library's kernels and places its device arrays
 * lazily, on first use; pfxt_create does that for this entry point on the
 * handle's device, so its calls load and allocate nothing. */
#define PFXT_NOALLOC_MAX_RAYS (1u << 20)
int pfxt_occluded_noalloc(pfxt_trace* trace, const pfxt_ray* rays, uint32_t count, uint8_t* blocked,
                          void* stream);

/* ------------------------------------------------------------ checkpoints
 * The reference's checkpoint byte layout (crates/trace/src/checkpoint.rs:8-158):
 * "PFXCKPT1", the key's length (u64) and bytes, width, height, samples (u32),
 * the 48 B/pixel accumulation, the colour, albedo and normal films (16 B/pixel
 * each), then u32 0xffffffff, or a round count, the rounds (u32 samples, u64
 * active) and 32 B/pixel adaptive snapshots; all little-endian. */
typedef struct pfxt_checkpoint_info {
  uint32_t width, height, samples;
  uint32_t rounds; /* adaptive rounds recorded; 0xffffffff when none */
} pfxt_checkpoint_info;

/* Trace::save + Saved::write_to (checkpoint.rs:82-104, 161-172): the
 * accumulation and films under `key`, without adaptive rounds.  With bytes ==
 * NULL, *written receives the size needed; otherwise capacity must hold it. */
int pfxt_save(pfxt_trace* trace, const char* key, void* bytes, size_t capacity, size_t* written);
/* Saved::read_from + Trace::restore (checkpoint.rs:106-158, 174-203): refuses a
 * checkpoint of another key or size, cut short or running past its end; the
 * adaptive part is read and checked but, as in the reference, not restored. */
int pfxt_restore(pfxt_trace* trace, const char* key, const void* bytes, size_t length);
/* Saved::read_from alone, on the host: checks a checkpoint and describes it. */
int pfxt_checkpoint_read(const char* key, const void* bytes, size_t length, pfxt_checkpoint_info* out);

/* Trace::set_projection (gpu.rs:2872-2890): PFXT_PROJECTION_*, the
 * orthographic width and height; restarts the accumulation. */
int pfxt_set_projection(pfxt_trace* trace, uint32_t projection, const float ortho[2]);

/* ------------------------------------------------------- moving instances
 * Trace::move_instances (gpu.rs:2433-2530) on the host buffers of a built
 * scene: new column-major 4x4 transforms (16 floats each) for its first `count`
 * instances.  Moved instances get new surface records and emitter vertices and
 * the top-level BVH is laid again; every buffer keeps its size and address.
 * *moved (may be NULL) is 1 when any transform differed bit for bit. */
int pfxt_scene_move_instances(pfxt_scene_blobs* blobs, const float* transforms, uint32_t count, uint32_t* moved);
/* Trace::builds (gpu.rs:2356, Builds gpu.rs:400-403): bottom-level BVHs built
 * (the world's and one per distinct mesh) and top-level BVHs laid (1 for a
 * scene with instances, one more per move). */
int pfxt_scene_builds(const pfxt_scene_blobs* blobs, uint32_t* bottom, uint32_t* top);
/* Trace::set_instance_transforms (gpu.rs:2422-2431): the same on the blobs the
 * trace was created from, then the moved buffers are uploaded (finish_tops,
 * gpu.rs:2533-2540) and the accumulation restarts when anything moved.  If the
 * upload fails (an error after the blobs moved), the blobs hold the new poses
 * and the trace the old ones: pfxt_finish_tops with the blobs' buffers retries. */
int pfxt_set_instance_transforms(pfxt_trace* trace, pfxt_scene_blobs* blobs, const float* transforms, uint32_t count,
                                 uint32_t* moved);
/* Trace::finish_tops (gpu.rs:2533-2546) for a host that moves instances in
 * buffers it packs itself: uploads the nodes, surface records, emitters and
 * emitter CDF of `buffers` (the same sizes as at pfxt_create; the triangles
 * are read only to lay the traversal nodes again) and restarts the
 * accumulation. */
int pfxt_finish_tops(pfxt_trace* trace, const pfxt_buffers* buffers);

/* ------------------------------------------------------------ launch tuning
 * Launch choices that change how long a sampling pass takes but no value it
 * computes.  No counterpart in the reference (wgpu sizes its own dispatches). */
typedef struct pfxt_tuning {
  uint32_t trace_threads; /* threads per block of the persistent traversal kernels: 64, 128 or 256 (128) */
  uint32_t sort_shading;  /* sort the shade queue by hit material every bounce (1) */
  uint32_t graphs;        /* replay each pass from a captured CUDA graph (1) */
  uint32_t split_shade;   /* shade a bounce in three kernels (hit, light slots, BSDF) instead of one (1) */
  uint32_t sort_rays;     /* sort the rays of every bounce after the first by direction and origin (0) */
  float pass_ms;          /* from pfxt_autotune: the chosen configuration's median pass time */
  uint32_t shadow_queue;  /* queue capacity of the light slots' shadow rays: 1 = one queue entry per slot and
                           * path, traced by the connect kernel; 0 = no queue, each slot's shadow ray traced
                           * inside the light-slot kernel (1; scenes with more slots per path than the queue
                           * holds always trace inside) */
  uint32_t short_stack;   /* traversal stack entries per lane kept in shared memory, the rest in local memory:
                           * 0 or 8 (0) */
  uint32_t from_cache;    /* set by pfxt_autotune: 1 when the choice came from an earlier tuning of the same
                           * scene, film and settings in this process */
  uint32_t slot_kernels;  /* with the shadow queue and three shade kernels: the light slots one launch per slot
                           * kind, slot after slot (1), or every slot of a path in one kernel (0) (1) */
} pfxt_tuning;

int pfxt_get_tuning(pfxt_trace* trace, pfxt_tuning* out);
int pfxt_set_tuning(pfxt_trace* trace, const pfxt_tuning* tuning);
/* Times `passes` one-sample passes (at least 2; the first of each
 * configuration warms up and is not counted) of this tracer's scene, one
 * choice at a time with the others held at the best so far: the traversal
 * block size, the material sort, one shade kernel or three, the ray sort, the
 * shadow queue and the shared-memory stack entries; keeps the fastest and
 * remembers it for this scene (a hash of its nodes, triangles, lights and
 * materials), film size, settings and attached cache, so a later tracer of
 * the same scene takes it without timing anything.  `out` (may be NULL)
 * receives it.  Restarts the accumulation; with a radiance cache attached,
 * the trial passes also train it. */
int pfxt_autotune(pfxt_trace* trace, uint32_t passes, pfxt_tuning* out);

/* ------------------------------------------------------------ radiance cache
 *
 * A neural radiance cache: a 16-level hash-grid encoding (2 FP16 features per
 * level) of the position plus one-blob direction/normal and the surface's
 * albedos, into an MLP of two 64-wide ReLU layers and an RGB output, BF16
 * operands on the tensor cores with FP32 accumulation and FP32 master
 * weights, trained online with Adam.  The reference has no cache: none of
 * these entry points has a counterpart in pfx.  Attached to a tracer, paths
 * end into the cache at vertex `query_bounce` (the vertex after that many
 * scattering events), or at the first vertex after it that is at least
 * `min_roughness` rough and not transmissive, `delay_bounces` vertices later
 * at most; a fraction of paths continue to make the training targets; where
 * the measured bias of the cache in a cell of a 16^3 grid exceeds
 * `error_bound`, paths continue as plain paths. */
typedef struct pfxt_cache pfxt_cache;

typedef struct pfxt_cache_settings {
  uint32_t log2_entries;    /* table entries per level = 2^log2_entries (10..22; 19) */
  uint32_t base_resolution; /* grid resolution of the coarsest level (16) */
  uint32_t max_resolution;  /* grid resolution of the finest level (2048) */
  uint32_t batch;           /* training records per step, a multiple of 128 (65536) */
  uint32_t steps;           /* training steps per sampling pass, at most (4) */
  uint32_t seed;            /* parameter initialisation */
  uint32_t query_bounce;    /* the path vertex that ends into the cache (1) */
  uint32_t record_bounces;  /* training records from vertices 0..record_bounces (4) */
  float learning_rate;      /* Adam (1e-2) */
  float beta1, beta2, epsilon; /* Adam (0.9, 0.99, 1e-15) */
  float train_fraction;     /* fraction of paths that make training targets (0.01) */
  float error_bound;        /* relative bias of a cell above which its paths stay plain (1) */
  float min_roughness;      /* a vertex smoother than this, or transmissive, does not end a path (0.25) */
  uint32_t delay_bounces;   /* ... for at most this many vertices after query_bounce (2) */
  float lo[3], hi[3];       /* bounds of the grid; pfxt_set_cache sets them to the scene's */
} pfxt_cache_settings;

/* One cache query (80 B): the hit point and what the network reads of it. */
typedef struct pfxt_cache_query {
  float position[3];
  float roughness;
  float direction[3];       /* towards the previous vertex (outgoing), unit */
  float transmission;
  float normal[3];          /* shading normal, unit */
  float pad0;
  float diffuse[3];
  float pad1;
  float specular[3];
  float pad2;
} pfxt_cache_query;

/* One training record (96 B): a query and the radiance the path carried. */
typedef struct pfxt_cache_record {
  pfxt_cache_query query;
  float target[3];
  float weight; /* 1 */
} pfxt_cache_record;

typedef struct pfxt_cache_stats {
  uint64_t steps;          /* Adam steps taken */
  float loss;              /* relative L2 loss of the last step */
  uint32_t records;        /* training records made by the last pass */
  uint32_t queries;        /* paths that ended into the cache in the last pass */
  uint32_t training_paths; /* training paths of the last pass */
  uint32_t cells_ok;       /* cells where paths may end into the cache */
  uint32_t pad;
} pfxt_cache_stats;

/* Fills the defaults above. */
int pfxt_cache_defaults(pfxt_cache_settings* settings);
/* Creates a cache on the current CUDA device with seeded parameters. */
int pfxt_cache_create(const pfxt_cache_settings* settings, pfxt_cache** out);
void pfxt_cache_destroy(pfxt_cache* cache);
/* Attaches the cache to a tracer (NULL detaches); sets the grid bounds to the
 * scene's and restarts the accumulation.  The cache must outlive the
 * attachment and belong to the tracer's device. */
int pfxt_set_cache(pfxt_trace* trace, pfxt_cache* cache);
int pfxt_cache_get_stats(pfxt_cache* cache, pfxt_cache_stats* stats);
/* Network output for `count` queries (host memory): rgb[3 * k + c]. */
int pfxt_cache_infer(pfxt_cache* cache, const pfxt_cache_query* queries, uint32_t count, float* rgb);
/* Gradients of the mean relative L2 loss over `count` records (a multiple
 * of 128) with the current parameters; nothing is updated.  mlp: 9216 floats
 * (W1 64x64, W2 64x64, W3 16x64, row = output); table: 16 * 2^log2 * 2
 * floats (NULL skips it); loss: the loss. */
int pfxt_cache_gradients(pfxt_cache* cache, const pfxt_cache_record* records, uint32_t count, float* mlp,
                         float* table, float* loss);
/* count / batch training steps (Adam) over the records in order; loss: the
 * mean loss of the steps. */
int pfxt_cache_train(pfxt_cache* cache, const pfxt_cache_record* records, uint32_t count, float* loss);
/* The FP32 master parameters (layouts as pfxt_cache_gradients); either may be NULL. */
int pfxt_cache_params(pfxt_cache* cache, float* mlp, float* table);
int pfxt_cache_set_params(pfxt_cache* cache, const float* mlp, const float* table);
/* The encoding: per level the position scale and grid resolution, and a bit
 * mask of the levels indexed densely (the others are hashed). */
int pfxt_cache_encoding(pfxt_cache* cache, float scales[16], uint32_t resolutions[16], uint32_t* dense);
/* The cache's kernels wait for their tensor-core work on an mbarrier with a
 * bounded number of polls (default 2^22).  A wait that runs out makes the
 * call fail with PFXT_ERR_CUDA ("a tensor-core wait ran out of its limit")
 * after the kernel has drained the work it issued; the cache stays usable.
 * Sets that limit (0 makes every wait run out: a way to test the error path). */
int pfxt_cache_set_wait_limit(pfxt_cache* cache, uint32_t polls);

/* ------------------------------------------------------------ denoiser
 *
 * OIDN's RT filter (U-Net over colour, albedo and normal), as the reference's
 * crates/denoise runs it (Denoiser, crates/denoise/src/lib.rs:58-361): the
 * same weights, autoexposure, transfer function and tile split.  Images are
 * row-major RGBA32F, width x height pixels; alpha passes through from the
 * colour; normals in any space in [-1, 1], albedo in [0, 1], colour linear
 * HDR.  The convolutions run on the tensor cores with FP32 accumulation; the
 * result is within 1e-3 x (1 + |v|) of OIDN's FP32 output, the reference's
 * own bar (crates/denoise/tests/oidn.rs). */
typedef struct pfxt_denoiser pfxt_denoiser;

/* Denoiser::new (lib.rs:81-110): parses an OIDN tensor archive (version 2;
 * the reference embeds rt_hdr_alb_nrm.tza, OIDN 2.5.1's default RT weights)
 * and uploads the network to the current device.  The blob is not kept.
 * PFXT_ERR_INVALID: "invalid or corrupted weights blob", "unsupported weights
 * blob version", "invalid tensor dimension|layout|data type", "<layer>: the
 * weights do not match the network", "<layer>: weights not exact in half
 * precision". */
int pfxt_denoiser_create(const void* tza, size_t bytes, pfxt_denoiser** out);
void pfxt_denoiser_destroy(pfxt_denoiser* denoiser);
/* Denoiser::denoise (lib.rs:112-140): host images in, the denoised colour
 * out (host), waits.  PFXT_ERR_INVALID for a zero size ("image dimensions
 * must be nonzero"). */
int pfxt_denoise(pfxt_denoiser* denoiser, uint32_t width, uint32_t height, const float* color, const float* albedo,
                 const float* normal, float* out);
/* Denoiser::denoise_textures_into (lib.rs:157-183): device images in and out
 * (16-byte aligned), enqueued on `stream` (a cudaStream_t; NULL: the legacy
 * stream); returns without waiting. */
int pfxt_denoise_device(pfxt_denoiser* denoiser, uint32_t width, uint32_t height, const float* color,
                        const float* albedo, const float* normal, float* out, void* stream);
/* The same with a tracer's colour, albedo and normal films
 * (pfxt_films_device) as the inputs, on the tracer's stream: what pfx does
 * with Trace::color/albedo/normal after a frame's last sample. */
int pfxt_denoise_trace(pfxt_denoiser* denoiser, pfxt_trace* trace, float* out_device);
/* Denoiser::tiles (lib.rs:112-116): the tile size and count of the split for
 * the last image size (0s before the first denoise). */
int pfxt_denoiser_tiles(pfxt_denoiser* denoiser, uint32_t* tile_w, uint32_t* tile_h, uint32_t* count);
/* Waits for the last denoise: its device time (ms) and multiply-adds.
 * PFXT_ERR_DEVICE when a convolution's bounded wait ran out (see below). */
int pfxt_denoiser_last(pfxt_denoiser* denoiser, float* ms, uint64_t* macs);
/* The largest tile in pixels (default 2160 x 2160, OIDN's); smaller values
 * split a frame into more tiles, as OIDN does on a device with less memory. */
int pfxt_denoiser_set_max_tile_pixels(pfxt_denoiser* denoiser, uint64_t pixels);
/* The convolutions wait for their tensor-core work and weight copies on
 * mbarriers with a bounded number of polls (default 2^26).  A wait that runs
 * out makes the denoise fail with PFXT_ERR_DEVICE once the kernel has drained
 * its own work; the denoiser stays usable.  0 makes every wait run out. */
int pfxt_denoiser_set_wait_limit(pfxt_denoiser* denoiser, uint32_t polls);

#ifdef __cplusplus
}
#endif
#endif /* PFXT_H */
