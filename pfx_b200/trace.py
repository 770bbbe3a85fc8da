"""Host-side mirror of the reference's `Trace` (crates/trace/src/gpu.rs and
adaptive.rs) over the C ABI of libpfxtrace.

    scene = SceneDesc(...)                       # Scene + Detail
    trace = Trace(scene, Settings(...), w, h)    # Trace::new_detailed
    trace.sample(16, seed=0)                     # Trace::sample
    conv = trace.sample_adaptive(Adaptive(...), seed=0)
    out = trace.readback()                       # Output{color, albedo, normal}

Errors surface as `TraceError` (refusals and setup errors of the reference).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import TraceError, check

TRIANGLE = np.dtype(abi.Triangle)
INSTANCE = np.dtype(abi.Instance)
MATERIAL = np.dtype(abi.Material)
LIGHT = np.dtype(abi.Light)
RAY = np.dtype(abi.Ray)
HIT = np.dtype(abi.Hit)
assert TRIANGLE.itemsize == 100 and RAY.itemsize == 32 and HIT.itemsize == 16


@dataclass
class Camera:
    origin: tuple
    forward: tuple
    right: tuple
    up: tuple

    def c(self) -> abi.Camera:
        return abi.Camera(abi.f3(*self.origin), abi.f3(*self.forward), abi.f3(*self.right), abi.f3(*self.up))


@dataclass
class Sun:
    direction: tuple = (0.0, 1.0, 0.0)
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 0.0
    radius_deg: float = 0.0


@dataclass
class SceneDesc:
    """Scene (gpu.rs:242-249) plus the Detail fields this tracer covers."""
    triangles: np.ndarray                      # TRIANGLE records, world space
    materials: np.ndarray                      # MATERIAL records
    camera: Camera
    lights: np.ndarray = field(default_factory=lambda: np.zeros(0, LIGHT))
    meshes: list = field(default_factory=list)  # list of TRIANGLE arrays
    instances: np.ndarray = field(default_factory=lambda: np.zeros(0, INSTANCE))
    sky: tuple = (0.0, 0.0, 0.0)
    sun: Sun = field(default_factory=Sun)
    sky_width: int = 256
    sky_height: int = 128

    def c(self):
        """ctypes Scene; the returned keep-alive list must outlive the call."""
        keep = []
        tri = np.ascontiguousarray(self.triangles, TRIANGLE)
        mats = np.ascontiguousarray(self.materials, MATERIAL)
        lights = np.ascontiguousarray(self.lights, LIGHT)
        inst = np.ascontiguousarray(self.instances, INSTANCE)
        keep += [tri, mats, lights, inst]
        mesh_arr = (abi.Mesh * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            m = np.ascontiguousarray(m, TRIANGLE)
            keep.append(m)
            mesh_arr[i].triangles = m.ctypes.data
            mesh_arr[i].count = len(m)
        keep.append(mesh_arr)
        s = abi.Scene()
        s.triangles, s.triangle_count = tri.ctypes.data, len(tri)
        s.meshes, s.mesh_count = C.cast(mesh_arr, C.c_void_p), len(self.meshes)
        s.instances, s.instance_count = inst.ctypes.data, len(inst)
        s.materials, s.material_count = mats.ctypes.data, len(mats)
        s.lights, s.light_count = lights.ctypes.data, len(lights)
        s.sky = abi.f3(*self.sky)
        s.sky_width, s.sky_height = self.sky_width, self.sky_height
        s.camera = self.camera.c()
        s.sun = abi.Sun(abi.f3(*self.sun.direction), abi.f3(*self.sun.color), self.sun.intensity,
                        self.sun.radius_deg)
        return s, keep

    @property
    def world_triangle_count(self) -> int:
        return len(self.triangles) + sum(len(self.meshes[int(i["mesh"])]) for i in self.instances)


@dataclass
class Settings:
    """Detail fields that specialise the tracer (detail.rs, gpu.rs:1140-1196)."""
    bounces: tuple = (16, 4, 8, 12)   # Bounces::REFERENCE
    sampler: str = "sobol"            # "sobol" | "pcg"
    sobol_samples: int = 256
    clamp_indirect: float = 0.0
    filter_glossy: float = 0.0
    projection: int = abi.PROJECTION_PERSPECTIVE
    ortho: tuple = (0.0, 0.0)
    lens: tuple = (0.0, 0.0, 0.0, 1.0)

    @staticmethod
    def deep(n: int, **kw) -> "Settings":
        """Bounces::deep(n) (detail.rs:435)."""
        return Settings(bounces=(n, n, n, n), **kw)

    def c(self) -> abi.Settings:
        s = abi.Settings()
        s.bounces = abi.u4(*self.bounces)
        s.sampler = abi.SAMPLER_SOBOL if self.sampler == "sobol" else abi.SAMPLER_PCG
        s.sobol_samples = self.sobol_samples
        s.clamp_indirect = self.clamp_indirect
        s.filter_glossy = self.filter_glossy
        s.projection = self.projection
        s.ortho = (C.c_float * 2)(*self.ortho)
        s.lens = abi.f4(*self.lens)
        return s


@dataclass
class Adaptive:
    """Adaptive (adaptive.rs:10-26)."""
    threshold: float = 0.005
    min_samples: int = 32
    max_samples: int = 1024
    growth: float = 1.5

    def c(self) -> abi.Adaptive:
        return abi.Adaptive(self.threshold, self.min_samples, self.max_samples, self.growth)

    def valid(self) -> bool:
        return (np.isfinite(self.threshold) and self.threshold > 0 and self.min_samples >= 2
                and self.max_samples >= self.min_samples and np.isfinite(self.growth) and self.growth > 1.0)

    def rounds(self) -> list:
        lib = abi.load()
        buf = (C.c_uint32 * 4096)()
        n = C.c_uint32()
        check(lib.pfxt_adaptive_rounds(C.byref(self.c()), buf, 4096, C.byref(n)))
        return list(buf[: n.value])


@dataclass
class Round:
    samples: int
    active: int


@dataclass
class Converged:
    """Converged (adaptive.rs:66-102)."""
    rounds: list
    pixels: int

    def mean_samples(self) -> float:
        if self.pixels == 0:
            return 0.0
        total, before, running = 0.0, 0, self.pixels
        for r in self.rounds:
            total += (r.samples - before) * running
            before, running = r.samples, r.active
        return total / self.pixels

    def converged(self) -> bool:
        return bool(self.rounds) and self.rounds[-1].active == 0


@dataclass
class Stats:
    """Stats (crates/gpu/src/pace.rs:66-70): device milliseconds of each pass and
    the host time of the whole call."""
    milliseconds: list
    wall_ms: float


@dataclass
class Output:
    color: np.ndarray
    albedo: np.ndarray
    normal: np.ndarray


class SceneBuffers:
    """SceneBuffers::build (gpu.rs:566) on the host, through the C ABI."""

    def __init__(self, scene: SceneDesc, settings: Settings):
        self._lib = abi.load()
        s, keep = scene.c()
        st = settings.c()
        h = C.c_void_p()
        check(self._lib.pfxt_scene_build(C.byref(s), C.byref(st), C.byref(h)))
        self._h = h
        self.buffers = abi.Buffers()
        check(self._lib.pfxt_scene_buffers(self._h, C.byref(self.buffers)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.pfxt_scene_free(h)
            self._h = None

    def _bytes(self, ptr, n) -> np.ndarray:
        if not n:
            return np.zeros(0, np.uint8)
        return np.ctypeslib.as_array((C.c_uint8 * n).from_address(ptr)).copy()

    def array(self, name: str) -> np.ndarray:
        b = self.buffers
        return self._bytes(getattr(b, name), getattr(b, name + "_bytes"))

    def order(self) -> np.ndarray:
        p = C.POINTER(C.c_uint32)()
        n = C.c_uint32()
        check(self._lib.pfxt_scene_order(self._h, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, (n.value,)).copy() if n.value else np.zeros(0, np.uint32)

    def move_instances(self, transforms) -> bool:
        """Trace::move_instances (gpu.rs:2433-2530) on these host buffers: new
        column-major 4x4 transforms for the first len(transforms) instances.
        Returns whether any instance moved."""
        t = _transforms(transforms)
        moved = C.c_uint32()
        check(self._lib.pfxt_scene_move_instances(self._h, t.ctypes.data if t.size else None, len(t),
                                                  C.byref(moved)))
        return bool(moved.value)

    def builds(self) -> tuple:
        """Trace::builds (gpu.rs:2356): (bottom-level BVHs built, top-level BVHs laid)."""
        bottom, top = C.c_uint32(), C.c_uint32()
        check(self._lib.pfxt_scene_builds(self._h, C.byref(bottom), C.byref(top)))
        return int(bottom.value), int(top.value)

    def sky(self):
        b = self.buffers
        rows = np.ctypeslib.as_array((C.c_float * b.sky_height).from_address(b.sky_rows)).copy()
        cols = np.ctypeslib.as_array((C.c_float * (b.sky_width * b.sky_height)).from_address(b.sky_columns)).copy()
        return rows, cols

    def sobol(self) -> np.ndarray:
        b = self.buffers
        if not b.sobol:
            return np.zeros((0, 4), np.float32)
        n = b.sobol_length * 256 * 4
        return np.ctypeslib.as_array((C.c_float * n).from_address(b.sobol)).copy().reshape(-1, 4)


class Trace:
    """The tracer handle (Trace, gpu.rs:309-342)."""

    def __init__(self, scene: SceneDesc, settings: Settings, width: int, height: int,
                 buffers: SceneBuffers | None = None):
        self._lib = abi.load()
        self.width, self.height = int(width), int(height)
        self.settings = settings
        self.scene_buffers = buffers if buffers is not None else SceneBuffers(scene, settings)
        s, keep = scene.c()
        st = settings.c()
        h = C.c_void_p()
        check(self._lib.pfxt_create(C.byref(self.scene_buffers.buffers), C.byref(s), C.byref(st),
                                    self.width, self.height, C.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.pfxt_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._h

    # ---------------------------------------------------------- sampling
    def sample(self, count: int, seed: int) -> None:
        check(self._lib.pfxt_sample(self._h, count, seed))

    def sample_paced(self, count: int, seed: int, between=None) -> Stats:
        """Trace::sample_paced (gpu.rs:2951): the samples one pass at a time,
        `between(ms)` after each with its device time; the image equals
        sample(count, seed)'s."""
        ms, failure = [], []

        def hook(_user, t):
            ms.append(float(t))
            if between is not None:
                try:
                    between(float(t))
                except Exception as e:  # noqa: BLE001 - carried back to the caller below
                    failure.append(e)

        wall = C.c_double()
        rc = self._lib.pfxt_sample_paced(self._h, count, seed, abi.BETWEEN(hook), None, C.byref(wall))
        if failure:
            raise failure[0]
        check(rc)
        return Stats(ms, float(wall.value))

    def samples(self) -> int:
        return int(self._lib.pfxt_samples(self._h))

    def sample_adaptive(self, adaptive: Adaptive, seed: int) -> Converged:
        cap = 4096
        rounds = (abi.Round * cap)()
        n = C.c_uint32()
        check(self._lib.pfxt_sample_adaptive(self._h, C.byref(adaptive.c()), seed, rounds, cap, C.byref(n)))
        return Converged([Round(int(rounds[i].samples), int(rounds[i].active)) for i in range(n.value)],
                         self.width * self.height)

    def sample_adaptive_kept(self, adaptive: Adaptive, seed: int, key: str, keeper) -> Converged:
        """Trace::sample_adaptive_kept (adaptive.rs:136-325).  `keeper` mirrors the
        Keeper trait (checkpoint.rs:30-34): keeper.resume() -> checkpoint bytes or
        None, keeper.due(samples) -> bool, keeper.keep(bytes) (raise to refuse).
        Checkpoints are taken under `key` in the layout of Trace.save, with the
        adaptive rounds and snapshots."""
        cap = 4096
        rounds = (abi.Round * cap)()
        n = C.c_uint32()
        resume = keeper.resume()
        failure = []

        def due(_user, samples):
            try:
                return 1 if keeper.due(int(samples)) else 0
            except Exception as e:  # noqa: BLE001 - carried back to the caller below
                failure.append(e)
                return 0

        def keep(_user, ptr, length):
            try:
                keeper.keep(C.string_at(ptr, length))
                return 0
            except Exception as e:  # noqa: BLE001
                failure.append(e)
                return 1

        k = abi.Keeper(None, None, 0, abi.KEEPER_DUE(due), abi.KEEPER_KEEP(keep))
        if resume is not None:
            buf = C.create_string_buffer(bytes(resume), len(resume))
            k.resume, k.resume_length = C.cast(buf, C.c_void_p), len(resume)
        rc = self._lib.pfxt_sample_adaptive_kept(self._h, C.byref(adaptive.c()), seed, key.encode(), C.byref(k),
                                                 rounds, cap, C.byref(n))
        if failure:
            raise failure[0]
        check(rc)
        return Converged([Round(int(rounds[i].samples), int(rounds[i].active)) for i in range(n.value)],
                         self.width * self.height)

    # ---------------------------------------------------------- readback
    def readback(self) -> Output:
        shape = (self.height, self.width, 4)
        c, a, n = (np.empty(shape, np.float32) for _ in range(3))
        check(self._lib.pfxt_readback(self._h, c.ctypes.data, a.ctypes.data, n.ctypes.data))
        return Output(c, a, n)

    def sample_counts(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.uint32)
        check(self._lib.pfxt_sample_counts(self._h, out.ctypes.data))
        return out

    def read_accum(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 12), np.float32)
        check(self._lib.pfxt_read_accum(self._h, out.ctypes.data))
        return out

    # ---------------------------------------------------------- view
    def set_camera(self, camera: Camera) -> None:
        check(self._lib.pfxt_set_camera(self._h, C.byref(camera.c())))

    def set_lens(self, shift=(0.0, 0.0), aperture=0.0, focus_distance=1.0) -> None:
        lens = abi.f4(shift[0], shift[1], aperture, focus_distance)
        check(self._lib.pfxt_set_lens(self._h, lens))

    def set_projection(self, projection: str = "perspective", width: float = 0.0, height: float = 0.0) -> None:
        """Trace::set_projection (gpu.rs:2872): "perspective", "orthographic" (width,
        height) or "equirect"; restarts the accumulation."""
        kind = {"perspective": 0, "orthographic": 1, "equirect": 2}[projection]
        check(self._lib.pfxt_set_projection(self._h, kind, (C.c_float * 2)(width, height)))

    def set_instance_transforms(self, transforms) -> bool:
        """Trace::set_instance_transforms (gpu.rs:2422-2431): new column-major 4x4
        transforms for the first len(transforms) instances; the accumulation
        restarts when any of them moved.  Returns whether any moved."""
        t = _transforms(transforms)
        moved = C.c_uint32()
        check(self._lib.pfxt_set_instance_transforms(self._h, self.scene_buffers._h,
                                                     t.ctypes.data if t.size else None, len(t), C.byref(moved)))
        return bool(moved.value)

    def finish_tops(self, buffers: SceneBuffers | None = None) -> None:
        """Trace::finish_tops (gpu.rs:2533): upload host buffers whose instances
        were moved (SceneBuffers.move_instances) and restart the accumulation."""
        b = buffers if buffers is not None else self.scene_buffers
        check(self._lib.pfxt_finish_tops(self._h, C.byref(b.buffers)))

    def builds(self) -> tuple:
        """Trace::builds (gpu.rs:2356): (bottom-level BVHs built, top-level BVHs laid)."""
        return self.scene_buffers.builds()

    def save(self, key: str) -> bytes:
        """Trace::save + Saved::write_to (checkpoint.rs): the checkpoint bytes."""
        need = C.c_size_t()
        check(self._lib.pfxt_save(self._h, key.encode(), None, 0, C.byref(need)))
        buf = (C.c_uint8 * need.value)()
        check(self._lib.pfxt_save(self._h, key.encode(), buf, need.value, C.byref(need)))
        return bytes(buf)

    def restore(self, key: str, data: bytes) -> None:
        """Saved::read_from + Trace::restore (checkpoint.rs)."""
        check(self._lib.pfxt_restore(self._h, key.encode(), data, len(data)))

    def set_window(self, full, origin) -> None:
        f = (C.c_uint32 * 2)(*full)
        o = (C.c_uint32 * 2)(*origin)
        check(self._lib.pfxt_set_window(self._h, f, o))

    # ---------------------------------------------------------- ray batches
    def trace_rays(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, RAY)
        hits = np.zeros(len(rays), HIT)
        check(self._lib.pfxt_trace_rays(self._h, rays.ctypes.data, len(rays), hits.ctypes.data))
        return hits

    def occluded(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, RAY)
        out = np.zeros(len(rays), np.uint8)
        check(self._lib.pfxt_occluded(self._h, rays.ctypes.data, len(rays), out.ctypes.data))
        return out.astype(bool)

    def trace_rays_device(self, rays_ptr: int, count: int, hits_ptr: int, stream: int = 0) -> None:
        check(self._lib.pfxt_trace_rays_device(self._h, rays_ptr, count, hits_ptr, stream))

    def occluded_device(self, rays_ptr: int, count: int, blocked_ptr: int, stream: int = 0) -> None:
        check(self._lib.pfxt_occluded_device(self._h, rays_ptr, count, blocked_ptr, stream))

    def films_device(self):
        """The colour, albedo and normal films as (H, W, 4) float32 CUDA tensors
        that alias the tracer's own device memory (no copy)."""
        import torch
        ptrs = [C.c_void_p() for _ in range(3)]
        check(self._lib.pfxt_films_device(self._h, *[C.byref(p) for p in ptrs]))

        class _View:
            def __init__(self, ptr, shape):
                self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False),
                                                 "version": 3, "strides": None}

        shape = (self.height, self.width, 4)
        return [torch.as_tensor(_View(p.value, shape), device="cuda") for p in ptrs]

    def tuning(self) -> dict:
        k = abi.Tuning()
        check(self._lib.pfxt_get_tuning(self._h, C.byref(k)))
        return {"trace_threads": k.trace_threads, "sort_shading": bool(k.sort_shading), "graphs": bool(k.graphs),
                "split_shade": bool(k.split_shade), "sort_rays": bool(k.sort_rays), "pass_ms": float(k.pass_ms),
                "shadow_queue": bool(k.shadow_queue), "short_stack": int(k.short_stack),
                "from_cache": bool(k.from_cache), "slot_kernels": bool(k.slot_kernels)}

    def set_tuning(self, trace_threads: int = 128, sort_shading: bool = True, graphs: bool = True,
                   split_shade: bool = True, sort_rays: bool = False, shadow_queue: bool = True,
                   short_stack: int = 0, slot_kernels: bool = True) -> None:
        k = abi.Tuning(trace_threads, int(sort_shading), int(graphs), int(split_shade), int(sort_rays), 0.0,
                       int(shadow_queue), int(short_stack), 0, int(slot_kernels))
        check(self._lib.pfxt_set_tuning(self._h, C.byref(k)))

    def pass_kernels(self) -> int:
        """Kernel launches of the last pass, counted in its captured graph (0
        when passes are not captured)."""
        return int(self._lib.pfxt_debug_pass_kernels(self._h))

    def autotune(self, passes: int = 3) -> dict:
        """Time passes of this scene under each launch choice and keep the
        fastest, or take an earlier tuning of the same scene (restarts the
        accumulation)."""
        k = abi.Tuning()
        check(self._lib.pfxt_autotune(self._h, passes, C.byref(k)))
        out = self.tuning()
        out["from_cache"] = bool(k.from_cache)
        return out

    def set_cache(self, cache) -> None:
        """Attach a pfx_b200.cache.RadianceCache (None detaches): paths then end
        into the cache at its query bounce and a fraction of them train it.
        Restarts the accumulation; the cache's grid takes the scene's bounds."""
        check(self._lib.pfxt_set_cache(self._h, None if cache is None else cache.handle))
        self._cache = cache

    def set_pixel_mask(self, mask) -> None:
        """Sample only the pixels where `mask` (H, W) is true; None lifts it.
        Restarts the accumulation."""
        if mask is None:
            check(self._lib.pfxt_set_pixel_mask(self._h, None))
            return
        m = np.ascontiguousarray(np.asarray(mask, bool).astype(np.uint8).reshape(self.height, self.width))
        check(self._lib.pfxt_set_pixel_mask(self._h, m.ctypes.data))

    # ---------------------------------------------------------- adaptive steps
    def adaptive_measure(self, first: bool) -> None:
        """measure (converge.wgsl:9-31) over the accumulation; `first` starts a
        new adaptive render (clears the snapshots)."""
        check(self._lib.pfxt_adaptive_measure(self._h, 1 if first else 0))

    def adaptive_mark(self, min_samples: int, threshold: float) -> int:
        """mark (converge.wgsl:32-51) on the errors in the snapshots; returns
        this tracer's running count."""
        n = C.c_uint32()
        check(self._lib.pfxt_adaptive_mark(self._h, int(min_samples), float(threshold), C.byref(n)))
        return int(n.value)

    def adaptive_snaps_device(self):
        """The (H, W, 8) float32 snapshots as a CUDA tensor aliasing the
        tracer's memory (the error at [..., 5])."""
        import torch
        p = C.c_void_p()
        check(self._lib.pfxt_adaptive_snaps_device(self._h, C.byref(p)))

        class _View:
            def __init__(self, ptr, shape):
                self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False),
                                                 "version": 3, "strides": None}

        return torch.as_tensor(_View(p.value, (self.height, self.width, 8)), device="cuda")


    def rays_traced(self) -> tuple:
        """(closest-hit, any-hit) queries traced by the sampling passes so far."""
        out = np.zeros(2, np.uint64)
        check(self._lib.pfxt_debug_rays(self._h, out.ctypes.data))
        return int(out[0]), int(out[1])

    def frame(self) -> np.ndarray:
        """The base per-pass uniform (10 x 16 bytes: size, counts, origin, forward,
        right, up, sun_dir, sun_color, lens, window)."""
        out = np.zeros(40, np.uint32)
        check(self._lib.pfxt_debug_frame(self._h, out.ctypes.data))
        return out

    def counts_device(self, rays_ptr: int, count: int, any_hit: bool, counts_ptr: int, stream: int = 0) -> None:
        check(self._lib.pfxt_trace_counts_device(self._h, rays_ptr, count, 1 if any_hit else 0, counts_ptr, stream))


def _transforms(transforms) -> np.ndarray:
    """Transforms as contiguous (n, 16) float32: each a column-major 4x4, given
    either flat (16 values) or as 4 columns of 4 (detail.rs Transform)."""
    t = np.ascontiguousarray(np.asarray(transforms, np.float32).reshape(-1, 16))
    return t


def make_rays(origins: np.ndarray, directions: np.ndarray, tmax) -> np.ndarray:
    rays = np.zeros(len(origins), RAY)
    rays["origin"] = origins
    rays["direction"] = directions
    rays["tmax"] = tmax
    return rays


__all__ = ["SceneDesc", "Settings", "Camera", "Sun", "Adaptive", "Converged", "Round", "Output", "Trace",
           "SceneBuffers", "TraceError", "make_rays", "TRIANGLE", "INSTANCE", "MATERIAL", "LIGHT", "RAY", "HIT"]
