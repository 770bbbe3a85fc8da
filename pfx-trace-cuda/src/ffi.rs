//! Raw declarations of include/pfxt.h, the C ABI of libpfxtrace.  Every struct
//! is `#[repr(C)]` and matches the header field for field; every function of
//! the header is declared here (the safe wrapper lives in lib.rs).
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

pub const PFXT_OK: c_int = 0;
pub const PFXT_ERR_INVALID: c_int = 1;
pub const PFXT_ERR_REFUSED: c_int = 2;
pub const PFXT_ERR_CUDA: c_int = 3;
pub const PFXT_ERR_DEVICE: c_int = 4;

pub const PFXT_LIGHT_POINT: u32 = 0;
pub const PFXT_LIGHT_SPOT: u32 = 1;
pub const PFXT_LIGHT_RECT: u32 = 2;
pub const PFXT_LIGHT_DISC: u32 = 3;
pub const PFXT_SAMPLER_PCG: u32 = 0;
pub const PFXT_SAMPLER_SOBOL: u32 = 1;
pub const PFXT_PROJECTION_PERSPECTIVE: u32 = 0;
pub const PFXT_PROJECTION_ORTHOGRAPHIC: u32 = 1;
pub const PFXT_PROJECTION_EQUIRECT: u32 = 2;
pub const PFXT_NOALLOC_MAX_RAYS: u32 = 1 << 20;

/// TriangleDetail without the second uv set (detail.rs:7-13).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtTriangle {
    pub v: [[f32; 3]; 3],
    pub n: [[f32; 3]; 3],
    pub uv: [[f32; 2]; 3],
    pub material: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct PfxtMesh {
    pub triangles: *const PfxtTriangle,
    pub count: u32,
}

/// Instance (detail.rs:53-60).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtInstance {
    pub mesh: u32,
    pub shadow_only: u32,
    pub two_sided: u32,
    pub casts_shadow: u32,
    /// column-major affine 4x4 (detail::Transform)
    pub transform: [f32; 16],
}

/// The hot material record's fields (materials/src/material.rs:827-843).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtMaterial {
    pub base: [f32; 3],
    pub roughness: f32,
    pub metalness: f32,
    pub specular: f32,
    pub clearcoat: f32,
    pub clearcoat_roughness: f32,
    pub sheen: f32,
    pub transmission: f32,
    pub ior: f32,
    pub dispersion: f32,
    pub thickness: f32,
    pub subsurface: f32,
    pub thin_film: f32,
    pub thin_film_ior: f32,
    pub subsurface_tint: [f32; 3],
    pub absorption: f32,
    pub emission: [f32; 3],
    pub thin_film_amount: f32,
    pub fresnel_power: f32,
    pub pad: [f32; 3],
}

/// LocalLight (lights.rs:11-39).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtLight {
    pub shape: u32,
    pub shadow: u32,
    pub two_sided: u32,
    pub pad: u32,
    pub position: [f32; 3],
    pub colour: [f32; 3],
    pub intensity: f32,
    pub radius: f32,
    pub range: f32,
    pub direction: [f32; 3],
    pub inner_deg: f32,
    pub outer_deg: f32,
    pub half_u: [f32; 3],
    pub half_v: [f32; 3],
    pub disc_radius: f32,
}

/// Camera (gpu.rs:173-179).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtCamera {
    pub origin: [f32; 3],
    pub forward: [f32; 3],
    pub right: [f32; 3],
    pub up: [f32; 3],
}

/// Sun (gpu.rs:231-236) with Detail::sun_radius_deg.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtSun {
    pub direction: [f32; 3],
    pub color: [f32; 3],
    pub intensity: f32,
    pub radius_deg: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct PfxtScene {
    pub triangles: *const PfxtTriangle,
    pub triangle_count: u32,
    pub meshes: *const PfxtMesh,
    pub mesh_count: u32,
    pub instances: *const PfxtInstance,
    pub instance_count: u32,
    pub materials: *const PfxtMaterial,
    pub material_count: u32,
    pub lights: *const PfxtLight,
    pub light_count: u32,
    pub sky: [f32; 3],
    pub sky_width: u32,
    pub sky_height: u32,
    pub pad: u32,
    pub camera: PfxtCamera,
    pub sun: PfxtSun,
}

/// Detail settings that specialise the tracer (detail.rs:374-455).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtSettings {
    pub bounces: [u32; 4],
    pub sampler: u32,
    pub sobol_samples: u32,
    pub clamp_indirect: f32,
    pub filter_glossy: f32,
    pub projection: u32,
    pub ortho: [f32; 2],
    pub lens: [f32; 4],
    pub pad: u32,
}

/// The byte blobs of SceneBuffers (gpu.rs:412-436).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct PfxtBuffers {
    pub triangles: *const c_void,
    pub triangles_bytes: usize,
    pub nodes: *const c_void,
    pub nodes_bytes: usize,
    pub materials: *const c_void,
    pub materials_bytes: usize,
    pub uv: *const c_void,
    pub uv_bytes: usize,
    pub surfaces: *const c_void,
    pub surfaces_bytes: usize,
    pub emitters: *const c_void,
    pub emitters_bytes: usize,
    pub emitter_cdf: *const c_void,
    pub emitter_cdf_bytes: usize,
    pub lights: *const c_void,
    pub lights_bytes: usize,
    pub triangle_count: u32,
    pub shape_count: u32,
    pub emitter_count: u32,
    pub light_count: u32,
    pub sky_rows: *const f32,
    pub sky_columns: *const f32,
    pub sky_width: u32,
    pub sky_height: u32,
    pub sky_radiance: [f32; 3],
    pub sky_sun_probability: f32,
    pub sobol: *const f32,
    pub sobol_length: u32,
    pub max_depth: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtRay {
    pub origin: [f32; 3],
    pub tmax: f32,
    pub direction: [f32; 3],
    pub pad: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtHit {
    pub t: f32,
    pub slot: u32,
    pub record: u32,
    pub hit: u32,
}

/// Rounds (adaptive.rs:73-77).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtRound {
    pub samples: u32,
    pub pad: u32,
    pub active: u64,
}

/// Adaptive (adaptive.rs:10-15).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtAdaptive {
    pub threshold: f32,
    pub min_samples: u32,
    pub max_samples: u32,
    pub growth: f32,
}

/// The Keeper trait (checkpoint.rs:30-34) as callbacks.
#[repr(C)]
#[derive(Clone, Copy)]
pub struct PfxtKeeper {
    pub user: *mut c_void,
    pub resume: *const c_void,
    pub resume_length: usize,
    pub due: Option<unsafe extern "C" fn(*mut c_void, u32) -> c_int>,
    pub keep: Option<unsafe extern "C" fn(*mut c_void, *const c_void, usize) -> c_int>,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtCheckpointInfo {
    pub width: u32,
    pub height: u32,
    pub samples: u32,
    pub rounds: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtTuning {
    pub trace_threads: u32,
    pub sort_shading: u32,
    pub graphs: u32,
    pub split_shade: u32,
    pub sort_rays: u32,
    pub pass_ms: f32,
    pub shadow_queue: u32,
    pub short_stack: u32,
    pub from_cache: u32,
    pub slot_kernels: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtCacheSettings {
    pub log2_entries: u32,
    pub base_resolution: u32,
    pub max_resolution: u32,
    pub batch: u32,
    pub steps: u32,
    pub seed: u32,
    pub query_bounce: u32,
    pub record_bounces: u32,
    pub learning_rate: f32,
    pub beta1: f32,
    pub beta2: f32,
    pub epsilon: f32,
    pub train_fraction: f32,
    pub error_bound: f32,
    pub min_roughness: f32,
    pub delay_bounces: u32,
    pub lo: [f32; 3],
    pub hi: [f32; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtCacheQuery {
    pub position: [f32; 3],
    pub roughness: f32,
    pub direction: [f32; 3],
    pub transmission: f32,
    pub normal: [f32; 3],
    pub pad0: f32,
    pub diffuse: [f32; 3],
    pub pad1: f32,
    pub specular: [f32; 3],
    pub pad2: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtCacheRecord {
    pub query: PfxtCacheQuery,
    pub target: [f32; 3],
    pub weight: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PfxtCacheStats {
    pub steps: u64,
    pub loss: f32,
    pub records: u32,
    pub queries: u32,
    pub training_paths: u32,
    pub cells_ok: u32,
    pub pad: u32,
}

/// Opaque handles.
#[repr(C)]
pub struct PfxtTrace {
    _private: [u8; 0],
}
#[repr(C)]
pub struct PfxtSceneBlobs {
    _private: [u8; 0],
}
#[repr(C)]
pub struct PfxtCache {
    _private: [u8; 0],
}
#[repr(C)]
pub struct PfxtDenoiser {
    _private: [u8; 0],
}

/// `between(user, milliseconds)` of pfxt_sample_paced.
pub type PfxtBetween = Option<unsafe extern "C" fn(*mut c_void, f64)>;

extern "C" {
    pub fn pfxt_abi_version() -> c_int;
    pub fn pfxt_last_error() -> *const c_char;
    pub fn pfxt_device_count() -> c_int;
    pub fn pfxt_scene_build(scene: *const PfxtScene, settings: *const PfxtSettings, out: *mut *mut PfxtSceneBlobs) -> c_int;
    pub fn pfxt_scene_free(blobs: *mut PfxtSceneBlobs);
    pub fn pfxt_scene_buffers(blobs: *const PfxtSceneBlobs, out: *mut PfxtBuffers) -> c_int;
    pub fn pfxt_scene_order(blobs: *const PfxtSceneBlobs, order: *mut *const u32, count: *mut u32) -> c_int;
    pub fn pfxt_create(buffers: *const PfxtBuffers, view: *const PfxtScene, settings: *const PfxtSettings, width: u32, height: u32, out: *mut *mut PfxtTrace) -> c_int;
    pub fn pfxt_destroy(trace: *mut PfxtTrace);
    pub fn pfxt_set_camera(trace: *mut PfxtTrace, camera: *const PfxtCamera) -> c_int;
    pub fn pfxt_set_lens(trace: *mut PfxtTrace, lens: *const f32) -> c_int;
    pub fn pfxt_set_window(trace: *mut PfxtTrace, full: *const u32, origin: *const u32) -> c_int;
    pub fn pfxt_sample(trace: *mut PfxtTrace, count: u32, seed: u32) -> c_int;
    pub fn pfxt_sample_paced(trace: *mut PfxtTrace, count: u32, seed: u32, between: PfxtBetween, user: *mut c_void, wall_ms: *mut f64) -> c_int;
    pub fn pfxt_samples(trace: *const PfxtTrace) -> u32;
    pub fn pfxt_sample_adaptive(trace: *mut PfxtTrace, adaptive: *const PfxtAdaptive, seed: u32, rounds: *mut PfxtRound, cap: u32, written: *mut u32) -> c_int;
    pub fn pfxt_sample_adaptive_kept(trace: *mut PfxtTrace, adaptive: *const PfxtAdaptive, seed: u32, key: *const c_char, keeper: *const PfxtKeeper, rounds: *mut PfxtRound, cap: u32, written: *mut u32) -> c_int;
    pub fn pfxt_adaptive_measure(trace: *mut PfxtTrace, first: u32) -> c_int;
    pub fn pfxt_adaptive_mark(trace: *mut PfxtTrace, min_samples: u32, threshold: f32, running: *mut u32) -> c_int;
    pub fn pfxt_adaptive_snaps_device(trace: *mut PfxtTrace, snaps: *mut *mut f32) -> c_int;
    pub fn pfxt_set_pixel_mask(trace: *mut PfxtTrace, mask: *const u8) -> c_int;
    pub fn pfxt_adaptive_rounds(adaptive: *const PfxtAdaptive, rounds: *mut u32, cap: u32, written: *mut u32) -> c_int;
    pub fn pfxt_readback(trace: *mut PfxtTrace, color: *mut f32, albedo: *mut f32, normal: *mut f32) -> c_int;
    pub fn pfxt_films_device(trace: *mut PfxtTrace, color: *mut *mut f32, albedo: *mut *mut f32, normal: *mut *mut f32) -> c_int;
    pub fn pfxt_sample_counts(trace: *mut PfxtTrace, counts: *mut u32) -> c_int;
    pub fn pfxt_read_accum(trace: *mut PfxtTrace, accum: *mut f32) -> c_int;
    pub fn pfxt_trace_rays(trace: *mut PfxtTrace, rays: *const PfxtRay, count: u32, hits: *mut PfxtHit) -> c_int;
    pub fn pfxt_occluded(trace: *mut PfxtTrace, rays: *const PfxtRay, count: u32, blocked: *mut u8) -> c_int;
    pub fn pfxt_trace_rays_device(trace: *mut PfxtTrace, rays: *const PfxtRay, count: u32, hits: *mut PfxtHit, stream: *mut c_void) -> c_int;
    pub fn pfxt_occluded_device(trace: *mut PfxtTrace, rays: *const PfxtRay, count: u32, blocked: *mut u32, stream: *mut c_void) -> c_int;
    pub fn pfxt_occluded_noalloc(trace: *mut PfxtTrace, rays: *const PfxtRay, count: u32, blocked: *mut u8, stream: *mut c_void) -> c_int;
    pub fn pfxt_save(trace: *mut PfxtTrace, key: *const c_char, bytes: *mut c_void, capacity: usize, written: *mut usize) -> c_int;
    pub fn pfxt_restore(trace: *mut PfxtTrace, key: *const c_char, bytes: *const c_void, length: usize) -> c_int;
    pub fn pfxt_checkpoint_read(key: *const c_char, bytes: *const c_void, length: usize, out: *mut PfxtCheckpointInfo) -> c_int;
    pub fn pfxt_set_projection(trace: *mut PfxtTrace, projection: u32, ortho: *const f32) -> c_int;
    pub fn pfxt_scene_move_instances(blobs: *mut PfxtSceneBlobs, transforms: *const f32, count: u32, moved: *mut u32) -> c_int;
    pub fn pfxt_scene_builds(blobs: *const PfxtSceneBlobs, bottom: *mut u32, top: *mut u32) -> c_int;
    pub fn pfxt_set_instance_transforms(trace: *mut PfxtTrace, blobs: *mut PfxtSceneBlobs, transforms: *const f32, count: u32, moved: *mut u32) -> c_int;
    pub fn pfxt_finish_tops(trace: *mut PfxtTrace, buffers: *const PfxtBuffers) -> c_int;
    pub fn pfxt_get_tuning(trace: *mut PfxtTrace, out: *mut PfxtTuning) -> c_int;
    pub fn pfxt_set_tuning(trace: *mut PfxtTrace, tuning: *const PfxtTuning) -> c_int;
    pub fn pfxt_autotune(trace: *mut PfxtTrace, passes: u32, out: *mut PfxtTuning) -> c_int;
    pub fn pfxt_cache_defaults(settings: *mut PfxtCacheSettings) -> c_int;
    pub fn pfxt_cache_create(settings: *const PfxtCacheSettings, out: *mut *mut PfxtCache) -> c_int;
    pub fn pfxt_cache_destroy(cache: *mut PfxtCache);
    pub fn pfxt_set_cache(trace: *mut PfxtTrace, cache: *mut PfxtCache) -> c_int;
    pub fn pfxt_cache_get_stats(cache: *mut PfxtCache, stats: *mut PfxtCacheStats) -> c_int;
    pub fn pfxt_cache_infer(cache: *mut PfxtCache, queries: *const PfxtCacheQuery, count: u32, rgb: *mut f32) -> c_int;
    pub fn pfxt_cache_gradients(cache: *mut PfxtCache, records: *const PfxtCacheRecord, count: u32, mlp: *mut f32, table: *mut f32, loss: *mut f32) -> c_int;
    pub fn pfxt_cache_train(cache: *mut PfxtCache, records: *const PfxtCacheRecord, count: u32, loss: *mut f32) -> c_int;
    pub fn pfxt_cache_params(cache: *mut PfxtCache, mlp: *mut f32, table: *mut f32) -> c_int;
    pub fn pfxt_cache_set_params(cache: *mut PfxtCache, mlp: *const f32, table: *const f32) -> c_int;
    pub fn pfxt_cache_encoding(cache: *mut PfxtCache, scales: *mut f32, resolutions: *mut u32, dense: *mut u32) -> c_int;
    pub fn pfxt_cache_set_wait_limit(cache: *mut PfxtCache, polls: u32) -> c_int;
    pub fn pfxt_denoiser_create(tza: *const c_void, bytes: usize, out: *mut *mut PfxtDenoiser) -> c_int;
    pub fn pfxt_denoiser_destroy(denoiser: *mut PfxtDenoiser);
    pub fn pfxt_denoise(denoiser: *mut PfxtDenoiser, width: u32, height: u32, color: *const f32, albedo: *const f32, normal: *const f32, out: *mut f32) -> c_int;
    pub fn pfxt_denoise_device(denoiser: *mut PfxtDenoiser, width: u32, height: u32, color: *const f32, albedo: *const f32, normal: *const f32, out: *mut f32, stream: *mut c_void) -> c_int;
    pub fn pfxt_denoise_trace(denoiser: *mut PfxtDenoiser, trace: *mut PfxtTrace, out_device: *mut f32) -> c_int;
    pub fn pfxt_denoiser_tiles(denoiser: *mut PfxtDenoiser, tile_w: *mut u32, tile_h: *mut u32, count: *mut u32) -> c_int;
    pub fn pfxt_denoiser_last(denoiser: *mut PfxtDenoiser, ms: *mut f32, macs: *mut u64) -> c_int;
    pub fn pfxt_denoiser_set_max_tile_pixels(denoiser: *mut PfxtDenoiser, pixels: u64) -> c_int;
    pub fn pfxt_denoiser_set_wait_limit(denoiser: *mut PfxtDenoiser, polls: u32) -> c_int;
}

// Layout checks against the header's sizes.
const _: () = assert!(std::mem::size_of::<PfxtTriangle>() == 100);
const _: () = assert!(std::mem::size_of::<PfxtInstance>() == 80);
const _: () = assert!(std::mem::size_of::<PfxtMaterial>() == 112);
const _: () = assert!(std::mem::size_of::<PfxtLight>() == 100);
const _: () = assert!(std::mem::size_of::<PfxtRay>() == 32);
const _: () = assert!(std::mem::size_of::<PfxtHit>() == 16);
const _: () = assert!(std::mem::size_of::<PfxtRound>() == 16);
const _: () = assert!(std::mem::size_of::<PfxtCacheRecord>() == 96);
