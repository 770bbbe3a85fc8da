"""ctypes declarations of include/pfxt.h and the loader of libpfxtrace.so.

The library is the product: there is no Python or CPU fallback.  If the shared
library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libpfxtrace.so"

f3 = C.c_float * 3
f4 = C.c_float * 4
u4 = C.c_uint32 * 4


class Triangle(C.Structure):
    _fields_ = [("v", (C.c_float * 3) * 3), ("n", (C.c_float * 3) * 3), ("uv", (C.c_float * 2) * 3),
                ("material", C.c_uint32)]


class Mesh(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("count", C.c_uint32)]


class Instance(C.Structure):
    _fields_ = [("mesh", C.c_uint32), ("shadow_only", C.c_uint32), ("two_sided", C.c_uint32),
                ("casts_shadow", C.c_uint32), ("transform", C.c_float * 16)]


class Material(C.Structure):
    _fields_ = [("base", f3), ("roughness", C.c_float),
                ("metalness", C.c_float), ("specular", C.c_float), ("clearcoat", C.c_float),
                ("clearcoat_roughness", C.c_float),
                ("sheen", C.c_float), ("transmission", C.c_float), ("ior", C.c_float), ("dispersion", C.c_float),
                ("thickness", C.c_float), ("subsurface", C.c_float), ("thin_film", C.c_float),
                ("thin_film_ior", C.c_float),
                ("subsurface_tint", f3), ("absorption", C.c_float),
                ("emission", f3), ("thin_film_amount", C.c_float),
                ("fresnel_power", C.c_float), ("pad", f3)]


LIGHT_POINT, LIGHT_SPOT, LIGHT_RECT, LIGHT_DISC = 0, 1, 2, 3


class Light(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("shadow", C.c_uint32), ("two_sided", C.c_uint32), ("pad", C.c_uint32),
                ("position", f3), ("colour", f3), ("intensity", C.c_float), ("radius", C.c_float),
                ("range", C.c_float), ("direction", f3), ("inner_deg", C.c_float), ("outer_deg", C.c_float),
                ("half_u", f3), ("half_v", f3), ("disc_radius", C.c_float)]


class Camera(C.Structure):
    _fields_ = [("origin", f3), ("forward", f3), ("right", f3), ("up", f3)]


class Sun(C.Structure):
    _fields_ = [("direction", f3), ("color", f3), ("intensity", C.c_float), ("radius_deg", C.c_float)]


class Scene(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("triangle_count", C.c_uint32),
                ("meshes", C.c_void_p), ("mesh_count", C.c_uint32),
                ("instances", C.c_void_p), ("instance_count", C.c_uint32),
                ("materials", C.c_void_p), ("material_count", C.c_uint32),
                ("lights", C.c_void_p), ("light_count", C.c_uint32),
                ("sky", f3), ("sky_width", C.c_uint32), ("sky_height", C.c_uint32), ("pad", C.c_uint32),
                ("camera", Camera), ("sun", Sun)]


SAMPLER_PCG, SAMPLER_SOBOL = 0, 1
PROJECTION_PERSPECTIVE, PROJECTION_ORTHOGRAPHIC, PROJECTION_EQUIRECT = 0, 1, 2


class Settings(C.Structure):
    _fields_ = [("bounces", u4), ("sampler", C.c_uint32), ("sobol_samples", C.c_uint32),
                ("clamp_indirect", C.c_float), ("filter_glossy", C.c_float), ("projection", C.c_uint32),
                ("ortho", C.c_float * 2), ("lens", f4), ("pad", C.c_uint32)]


class Buffers(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("triangles_bytes", C.c_size_t),
                ("nodes", C.c_void_p), ("nodes_bytes", C.c_size_t),
                ("materials", C.c_void_p), ("materials_bytes", C.c_size_t),
                ("uv", C.c_void_p), ("uv_bytes", C.c_size_t),
                ("surfaces", C.c_void_p), ("surfaces_bytes", C.c_size_t),
                ("emitters", C.c_void_p), ("emitters_bytes", C.c_size_t),
                ("emitter_cdf", C.c_void_p), ("emitter_cdf_bytes", C.c_size_t),
                ("lights", C.c_void_p), ("lights_bytes", C.c_size_t),
                ("triangle_count", C.c_uint32), ("shape_count", C.c_uint32), ("emitter_count", C.c_uint32),
                ("light_count", C.c_uint32),
                ("sky_rows", C.c_void_p), ("sky_columns", C.c_void_p),
                ("sky_width", C.c_uint32), ("sky_height", C.c_uint32),
                ("sky_radiance", f3), ("sky_sun_probability", C.c_float),
                ("sobol", C.c_void_p), ("sobol_length", C.c_uint32), ("max_depth", C.c_uint32)]


class Ray(C.Structure):
    _fields_ = [("origin", f3), ("tmax", C.c_float), ("direction", f3), ("pad", C.c_uint32)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("slot", C.c_uint32), ("record", C.c_uint32), ("hit", C.c_uint32)]


class Round(C.Structure):
    _fields_ = [("samples", C.c_uint32), ("pad", C.c_uint32), ("active", C.c_uint64)]


class Adaptive(C.Structure):
    _fields_ = [("threshold", C.c_float), ("min_samples", C.c_uint32), ("max_samples", C.c_uint32),
                ("growth", C.c_float)]


class CheckpointInfo(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("samples", C.c_uint32), ("rounds", C.c_uint32)]


BETWEEN = C.CFUNCTYPE(None, C.c_void_p, C.c_double)
KEEPER_DUE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint32)
KEEPER_KEEP = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t)


class Keeper(C.Structure):
    _fields_ = [("user", C.c_void_p), ("resume", C.c_void_p), ("resume_length", C.c_size_t),
                ("due", KEEPER_DUE), ("keep", KEEPER_KEEP)]


class Tuning(C.Structure):
    _fields_ = [("trace_threads", C.c_uint32), ("sort_shading", C.c_uint32), ("graphs", C.c_uint32),
                ("split_shade", C.c_uint32), ("sort_rays", C.c_uint32), ("pass_ms", C.c_float),
                ("shadow_queue", C.c_uint32), ("short_stack", C.c_uint32), ("from_cache", C.c_uint32),
                ("slot_kernels", C.c_uint32)]


class CacheSettings(C.Structure):
    _fields_ = [("log2_entries", C.c_uint32), ("base_resolution", C.c_uint32), ("max_resolution", C.c_uint32),
                ("batch", C.c_uint32), ("steps", C.c_uint32), ("seed", C.c_uint32), ("query_bounce", C.c_uint32),
                ("record_bounces", C.c_uint32), ("learning_rate", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("epsilon", C.c_float), ("train_fraction", C.c_float),
                ("error_bound", C.c_float), ("min_roughness", C.c_float), ("delay_bounces", C.c_uint32),
                ("lo", f3), ("hi", f3)]


class CacheStats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("loss", C.c_float), ("records", C.c_uint32), ("queries", C.c_uint32),
                ("training_paths", C.c_uint32), ("cells_ok", C.c_uint32), ("pad", C.c_uint32)]


OK, ERR_INVALID, ERR_REFUSED, ERR_CUDA, ERR_DEVICE = 0, 1, 2, 3, 4

# (name, restype, argtypes) of every exported entry point declared in pfxt.h.
PROTOTYPES = [
    ("pfxt_abi_version", C.c_int, []),
    ("pfxt_last_error", C.c_char_p, []),
    ("pfxt_device_count", C.c_int, []),
    ("pfxt_scene_build", C.c_int, [C.POINTER(Scene), C.POINTER(Settings), C.POINTER(C.c_void_p)]),
    ("pfxt_scene_free", None, [C.c_void_p]),
    ("pfxt_scene_buffers", C.c_int, [C.c_void_p, C.POINTER(Buffers)]),
    ("pfxt_scene_order", C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint32)]),
    ("pfxt_create", C.c_int, [C.POINTER(Buffers), C.POINTER(Scene), C.POINTER(Settings), C.c_uint32, C.c_uint32,
                              C.POINTER(C.c_void_p)]),
    ("pfxt_destroy", None, [C.c_void_p]),
    ("pfxt_set_camera", C.c_int, [C.c_void_p, C.POINTER(Camera)]),
    ("pfxt_set_lens", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("pfxt_set_window", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("pfxt_sample", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    ("pfxt_samples", C.c_uint32, [C.c_void_p]),
    ("pfxt_sample_paced", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, BETWEEN, C.c_void_p,
                                    C.POINTER(C.c_double)]),
    ("pfxt_sample_adaptive", C.c_int, [C.c_void_p, C.POINTER(Adaptive), C.c_uint32, C.POINTER(Round), C.c_uint32,
                                       C.POINTER(C.c_uint32)]),
    ("pfxt_sample_adaptive_kept", C.c_int, [C.c_void_p, C.POINTER(Adaptive), C.c_uint32, C.c_char_p,
                                            C.POINTER(Keeper), C.POINTER(Round), C.c_uint32, C.POINTER(C.c_uint32)]),
    ("pfxt_adaptive_rounds", C.c_int, [C.POINTER(Adaptive), C.POINTER(C.c_uint32), C.c_uint32,
                                       C.POINTER(C.c_uint32)]),
    ("pfxt_readback", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pfxt_sample_counts", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pfxt_read_accum", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pfxt_films_device", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_void_p)]),
    ("pfxt_trace_rays", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("pfxt_occluded", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("pfxt_trace_rays_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pfxt_occluded_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pfxt_occluded_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("pfxt_save", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("pfxt_restore", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]),
    ("pfxt_checkpoint_read", C.c_int, [C.c_char_p, C.c_void_p, C.c_size_t, C.POINTER(CheckpointInfo)]),
    ("pfxt_set_projection", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_float)]),
    ("pfxt_scene_move_instances", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    ("pfxt_scene_builds", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("pfxt_finish_tops", C.c_int, [C.c_void_p, C.POINTER(Buffers)]),
    ("pfxt_set_instance_transforms", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                               C.POINTER(C.c_uint32)]),
    ("pfxt_get_tuning", C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    ("pfxt_set_tuning", C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    ("pfxt_autotune", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(Tuning)]),
    ("pfxt_cache_defaults", C.c_int, [C.POINTER(CacheSettings)]),
    ("pfxt_cache_create", C.c_int, [C.POINTER(CacheSettings), C.POINTER(C.c_void_p)]),
    ("pfxt_cache_destroy", None, [C.c_void_p]),
    ("pfxt_set_cache", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pfxt_cache_get_stats", C.c_int, [C.c_void_p, C.POINTER(CacheStats)]),
    ("pfxt_cache_infer", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("pfxt_cache_gradients", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_float)]),
    ("pfxt_cache_train", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_float)]),
    ("pfxt_cache_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pfxt_cache_set_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pfxt_cache_encoding", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]),
    ("pfxt_cache_set_wait_limit", C.c_int, [C.c_void_p, C.c_uint32]),
    ("pfxt_adaptive_measure", C.c_int, [C.c_void_p, C.c_uint32]),
    ("pfxt_adaptive_mark", C.c_int, [C.c_void_p, C.c_uint32, C.c_float, C.POINTER(C.c_uint32)]),
    ("pfxt_adaptive_snaps_device", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("pfxt_set_pixel_mask", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pfxt_denoiser_create", C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)]),
    ("pfxt_denoiser_destroy", None, [C.c_void_p]),
    ("pfxt_denoise", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p]),
    ("pfxt_denoise_device", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]),
    ("pfxt_denoise_trace", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pfxt_denoiser_tiles", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32)]),
    ("pfxt_denoiser_last", C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint64)]),
    ("pfxt_denoiser_set_max_tile_pixels", C.c_int, [C.c_void_p, C.c_uint64]),
    ("pfxt_denoiser_set_wait_limit", C.c_int, [C.c_void_p, C.c_uint32]),
]
NOALLOC_MAX_RAYS = 1 << 20

# Exported beside the header for the measurement harness.
EXTRA = [
    ("pfxt_debug_frame", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pfxt_debug_rays", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pfxt_debug_stream", C.c_void_p, [C.c_void_p]),
    ("pfxt_debug_pixel_mask", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pfxt_debug_sort", C.c_int, [C.c_void_p, C.c_uint32]),
    ("pfxt_debug_graphs", C.c_int, [C.c_void_p, C.c_uint32]),
    ("pfxt_debug_graph_captures", C.c_uint32, [C.c_void_p]),
    ("pfxt_debug_pass_kernels", C.c_uint32, [C.c_void_p]),
    ("pfxt_debug_select_nth", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_int32, C.c_void_p]),
    ("pfxt_debug_gpu_bvh", C.c_int, [C.c_int32]),
    ("pfxt_debug_scene_gpu_builds", C.c_uint32, [C.c_void_p]),
    ("pfxt_debug_denoiser_shape", C.c_int, [C.c_void_p, C.c_uint32]),
    ("pfxt_debug_denoise_plan", C.c_int, [C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("pfxt_trace_counts_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                           C.c_void_p]),
]

_lib = None


def load() -> C.CDLL:
    """Load libpfxtrace.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"libpfxtrace.so is not built ({LIB_PATH}); run pfx_b200/build.py")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_GLOBAL if hasattr(os, "RTLD_GLOBAL") else 0)
    for name, res, args in PROTOTYPES + EXTRA:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class TraceError(RuntimeError):
    """TraceError of the reference (gpu.rs:269-307): a refusal or a setup error."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


def check(code: int) -> None:
    if code != OK:
        msg = load().pfxt_last_error().decode("utf-8", "replace")
        raise TraceError(code, msg)
