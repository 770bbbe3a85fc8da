"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the B200 tracer.

ctypes bindings of oracle/lib/liboracle.so, a scalar C++ restatement of the
reference tracer (gmrdad82/pfx crates/trace) that tests/ and bench.py's CPU
baseline use as the checker.  The product package (pfx_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "liboracle.so"

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime
                                   for p in [HERE / "oracle.cpp", HERE / "render.cpp", HERE / "pack.cpp",
                                             HERE.parent / "pfx_b200/csrc/pfxt_math.h"]
                                   if p.exists()):
            build()
        L = C.CDLL(str(LIB))
        vp, u32, f32, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_int32
        sig = {
            "orc_bvh_build": (u32, [vp, u32, vp, vp]),
            "orc_bvh_intersect": (i32, [vp, u32, vp, vp, vp, vp, f32]),
            "orc_brute_intersect": (i32, [vp, u32, vp, vp, f32]),
            "orc_trace": (C.c_int, [vp, u32, vp, u32, vp, vp, u32, C.c_int, vp, vp, vp]),
            "orc_hash_uint2": (u32, [u32, u32]),
            "orc_animated_seed": (u32, [u32, u32]),
            "orc_sequence_size": (u32, [u32]),
            "orc_generate_4d": (None, [vp, u32, u32]),
            "orc_automatic_min_samples": (u32, [f32]),
            "orc_adaptive_error": (f32, [vp, f32, vp, f32]),
            "orc_falloff": (f32, [f32, f32, f32, f32]),
            "orc_check_div": (C.c_uint64, [C.c_uint64, C.c_uint64]),
            "orc_math": (None, [C.c_int, vp, vp, vp, C.c_uint64]),
            "orc_scene_build": (vp, [vp]),
            "orc_scene_free": (None, [vp]),
            "orc_scene_blob": (C.c_uint64, [vp, C.c_int, C.POINTER(C.c_void_p)]),
            "orc_scene_counts": (None, [vp, vp]),
            "orc_select_nth": (None, [vp, u32, u32, C.c_int32, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class _InMesh(C.Structure):
    _fields_ = [("tris", C.c_void_p), ("count", C.c_uint32)]


class _InScene(C.Structure):
    _fields_ = [("world", C.c_void_p), ("world_count", C.c_uint32), ("meshes", C.c_void_p),
                ("mesh_count", C.c_uint32), ("instances", C.c_void_p), ("instance_count", C.c_uint32),
                ("materials", C.c_void_p), ("material_count", C.c_uint32), ("lights", C.c_void_p),
                ("light_count", C.c_uint32), ("sky", C.c_float * 3), ("sky_width", C.c_uint32),
                ("sky_height", C.c_uint32), ("sobol", C.c_uint32), ("sobol_samples", C.c_uint32)]


class _Counts:
    pass


class OracleBuffers:
    """The oracle's own SceneBuffers::build (oracle/pack.cpp, a restatement of
    gpu.rs:566-1061, tree.rs, levels.rs, lights.rs, record.rs and sky.rs) for a
    scene description (a pfx_b200.trace.SceneDesc: its input arrays only).
    Offers the blob accessors the oracle's tracer reads (array, order, sky,
    sobol and the counts in .buffers), so the oracle can trace without any
    buffer the product made."""

    NAMES = {"nodes": 0, "triangles": 1, "uv": 2, "surfaces": 3, "materials": 4, "emitters": 5, "emitter_cdf": 6,
             "lights": 7}

    def __init__(self, scene, settings):
        world = np.ascontiguousarray(scene.triangles)
        meshes = [np.ascontiguousarray(m) for m in scene.meshes]
        inst = np.ascontiguousarray(scene.instances)
        mats = np.ascontiguousarray(scene.materials)
        lights = np.ascontiguousarray(scene.lights)
        for a, size in ((world, 100), (inst, 80), (mats, 112), (lights, 100)):
            assert a.dtype.itemsize == size, "input layout"
        mesh_arr = (_InMesh * max(1, len(meshes)))()
        for i, m in enumerate(meshes):
            mesh_arr[i].tris, mesh_arr[i].count = (_p(m) if len(m) else None), len(m)
        s = _InScene()
        s.world, s.world_count = (_p(world) if len(world) else None), len(world)
        s.meshes, s.mesh_count = C.cast(mesh_arr, C.c_void_p), len(meshes)
        s.instances, s.instance_count = (_p(inst) if len(inst) else None), len(inst)
        s.materials, s.material_count = _p(mats), len(mats)
        s.lights, s.light_count = (_p(lights) if len(lights) else None), len(lights)
        s.sky = (C.c_float * 3)(*scene.sky)
        s.sky_width, s.sky_height = scene.sky_width, scene.sky_height
        s.sobol = 1 if settings.sampler == "sobol" else 0
        s.sobol_samples = settings.sobol_samples
        h = lib().orc_scene_build(C.byref(s))
        try:
            self._blobs = {}
            for name, which in list(self.NAMES.items()) + [("order", 8), ("sky_rows", 9), ("sky_columns", 10),
                                                           ("sobol", 11)]:
                ptr = C.c_void_p()
                n = lib().orc_scene_blob(h, which, C.byref(ptr))
                self._blobs[name] = (np.ctypeslib.as_array((C.c_uint8 * n).from_address(ptr.value)).copy()
                                     if n else np.zeros(0, np.uint8))
            counts = np.zeros(7, np.uint32)
            lib().orc_scene_counts(h, _p(counts))
        finally:
            lib().orc_scene_free(h)
        b = _Counts()
        (b.triangle_count, b.emitter_count, b.light_count, b.sky_width, b.sky_height, b.sobol_length,
         b.bottom_builds) = (int(x) for x in counts)
        b.sky_radiance = tuple(float(x) for x in scene.sky)
        b.sky_sun_probability = 0.0
        self.buffers = b

    def array(self, name: str) -> np.ndarray:
        return self._blobs[name].copy()

    def order(self) -> np.ndarray:
        return self._blobs["order"].view(np.uint32).copy()

    def sky(self):
        return self._blobs["sky_rows"].view(np.float32).copy(), self._blobs["sky_columns"].view(np.float32).copy()

    def sobol(self) -> np.ndarray:
        return self._blobs["sobol"].view(np.float32).reshape(-1, 4).copy()


def select_nth(keys, index: int, rounds: int = 16) -> np.ndarray:
    """Rust's select_nth_unstable_by(index, f32::total_cmp) as the light tree
    runs it: the original positions of `keys` in the order it leaves them."""
    k = np.ascontiguousarray(keys, np.float32)
    out = np.zeros(len(k), np.uint32)
    lib().orc_select_nth(_p(k), len(k), index, rounds, _p(out))
    return out


def scene_buffers(scene, settings) -> OracleBuffers:
    """The oracle's own packed buffers of `scene` (see OracleBuffers)."""
    return OracleBuffers(scene, settings)


def bvh_build(vertices: np.ndarray):
    """Bvh::build (bvh.rs:95-266) over (n, 3, 3) float32 vertices -> (nodes bytes, order)."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 9)
    n = len(v)
    nodes = np.zeros(max(1, 2 * n) * 48, np.uint8)
    order = np.zeros(max(1, n), np.uint32)
    count = lib().orc_bvh_build(_p(v), n, _p(nodes), _p(order))
    return nodes[: count * 48].copy(), order[:n].copy()


def bvh_intersect(nodes: np.ndarray, order: np.ndarray, vertices: np.ndarray, o, d, limit=np.inf) -> int:
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 9)
    o = np.asarray(o, np.float32)
    d = np.asarray(d, np.float32)
    return lib().orc_bvh_intersect(_p(nodes), len(nodes) // 48, _p(order), _p(v), _p(o), _p(d), float(limit))


def brute_intersect(vertices: np.ndarray, o, d, limit=np.inf) -> int:
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 9)
    o = np.asarray(o, np.float32)
    d = np.asarray(d, np.float32)
    return lib().orc_brute_intersect(_p(v), len(v), _p(o), _p(d), float(limit))


def trace(buffers, rays: np.ndarray, any_hit: bool = False, counts: bool = False):
    """scene() / occluded() of trace.wgsl over a ray batch on SceneBuffers
    layouts.  `buffers` is a pfx_b200.trace.SceneBuffers (its packed bytes)."""
    from pfx_b200.trace import HIT, RAY
    rays = np.ascontiguousarray(rays, RAY)
    nodes = buffers.array("nodes")
    tris = buffers.array("triangles")
    surf = buffers.array("surfaces")
    hits = np.zeros(len(rays), HIT)
    cnt = np.zeros((len(rays), 2), np.uint32) if counts else None
    overflow = np.zeros(1, np.uint32)
    lib().orc_trace(_p(nodes), len(nodes) // 48, _p(tris), len(tris) // 96, _p(surf), _p(rays), len(rays),
                    1 if any_hit else 0, _p(hits), _p(cnt) if counts else None, _p(overflow))
    return (hits, cnt, int(overflow[0])) if counts else hits


def hash_uint2(kx: int, ky: int) -> int:
    return int(lib().orc_hash_uint2(kx, ky))


def animated_seed(seed: int, frame: int) -> int:
    return int(lib().orc_animated_seed(seed, frame))


def sequence_size(samples: int) -> int:
    return int(lib().orc_sequence_size(samples))


def generate_4d(size: int, seed: int) -> np.ndarray:
    out = np.zeros((size, 4), np.float32)
    lib().orc_generate_4d(_p(out), size, seed)
    return out


def automatic_min_samples(threshold: float) -> int:
    return int(lib().orc_automatic_min_samples(threshold))


def adaptive_error(prior, prior_count, now, count) -> float:
    p = np.asarray(prior, np.float32)
    n = np.asarray(now, np.float32)
    return float(lib().orc_adaptive_error(_p(p), prior_count, _p(n), count))


def falloff(intensity, radius, range_, distance) -> float:
    return float(lib().orc_falloff(intensity, radius, range_, distance))


def check_div(per_family: int, seed: int = 1) -> int:
    """Mismatches between the kernels' correctly-rounded division (div_rn) and IEEE division."""
    return int(lib().orc_check_div(per_family, seed))


MATH_FUNCTIONS = ("sin", "cos", "asin", "acos", "atan2", "exp", "log", "pow")


def math(fn: str, x, y=None) -> np.ndarray:
    """The transcendentals the kernels and the oracle share (pfxt_math.h), on float32 arrays."""
    x = np.ascontiguousarray(x, np.float32)
    yy = None if y is None else np.ascontiguousarray(y, np.float32)
    out = np.empty_like(x)
    lib().orc_math(MATH_FUNCTIONS.index(fn), _p(x), None if yy is None else _p(yy), _p(out), x.size)
    return out


def frame_of(scene, width: int, height: int, tri_count: int, window=None) -> np.ndarray:
    """The per-pass uniform the product computes on the host (gpu.rs:2295-2316)
    for a perspective camera without lens; `window` = (full_w, full_h, x, y)
    renders a tile of a larger frame (Trace::set_window, gpu.rs:2834)."""
    import math
    f = np.zeros(40, np.uint32)
    fl = f.view(np.float32)
    f[0:4] = (width, height, 0, 0)
    f[4:8] = (tri_count, 0, 0, 0)
    fl[8:11] = scene.camera.origin
    fl[12:15] = scene.camera.forward
    fl[16:19] = scene.camera.right
    fl[20:23] = scene.camera.up
    fl[24:27] = scene.sun.direction
    fl[27] = np.float32(math.cos(np.float32(scene.sun.radius_deg) * np.float32(math.pi / 180.0)))
    fl[28:31] = scene.sun.color
    fl[31] = scene.sun.intensity
    fl[32:36] = (0.0, 0.0, 0.0, 1.0)
    f[36:40] = window if window is not None else (width, height, 0, 0)
    return f


class _OrcScene(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("node_count", C.c_uint32), ("tris", C.c_void_p), ("tri_count", C.c_uint32),
                ("surfaces", C.c_void_p), ("materials", C.c_void_p), ("material_rows", C.c_uint32),
                ("emitters", C.c_void_p), ("emitter_cdf", C.c_void_p), ("lights", C.c_void_p),
                ("sky_rows", C.c_void_p), ("sky_columns", C.c_void_p), ("sky_width", C.c_uint32),
                ("sky_height", C.c_uint32), ("sky_radiance", C.c_float * 3), ("sky_sun_probability", C.c_float),
                ("sobol", C.c_void_p), ("sobol_length", C.c_uint32), ("sobol_on", C.c_uint32),
                ("bounces", C.c_uint32 * 4), ("clamp_indirect", C.c_float), ("filter_glossy", C.c_float)]


class Renderer:
    """main()/radiance() of the reference restated on the CPU over one scene's
    packed buffers (a pfx_b200 SceneBuffers) and settings."""

    def __init__(self, buffers, settings):
        L = lib()
        L.orc_render.restype = C.c_int
        L.orc_render.argtypes = [C.c_void_p] * 6
        L.orc_converge.restype = C.c_uint32
        L.orc_converge.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_int]
        L.orc_tree_pick.restype = None
        L.orc_tree_pick.argtypes = [C.c_void_p] * 4 + [C.c_uint32] + [C.c_void_p] * 3
        self.keep = {k: buffers.array(k) for k in ("nodes", "triangles", "surfaces", "materials", "emitters",
                                                   "emitter_cdf", "lights")}
        rows, cols = buffers.sky()
        self.keep["sky_rows"], self.keep["sky_cols"] = rows, cols
        self.keep["sobol"] = np.ascontiguousarray(buffers.sobol(), np.float32)
        b = buffers.buffers
        s = _OrcScene()
        s.nodes, s.node_count = _p(self.keep["nodes"]), len(self.keep["nodes"]) // 48
        s.tris, s.tri_count = _p(self.keep["triangles"]), len(self.keep["triangles"]) // 96
        s.surfaces = _p(self.keep["surfaces"])
        s.materials, s.material_rows = _p(self.keep["materials"]), len(self.keep["materials"]) // 16
        s.emitters = _p(self.keep["emitters"])
        s.emitter_cdf = _p(self.keep["emitter_cdf"]) if len(self.keep["emitter_cdf"]) else None
        s.lights = _p(self.keep["lights"]) if len(self.keep["lights"]) else None
        s.sky_rows, s.sky_columns = _p(rows), _p(cols)
        s.sky_width, s.sky_height = b.sky_width, b.sky_height
        s.sky_radiance = (C.c_float * 3)(*b.sky_radiance)
        s.sky_sun_probability = b.sky_sun_probability
        sob = self.keep["sobol"]
        s.sobol = _p(sob) if len(sob) else None
        s.sobol_length = b.sobol_length
        s.sobol_on = 1 if settings.sampler == "sobol" else 0
        s.bounces = (C.c_uint32 * 4)(*settings.bounces)
        s.clamp_indirect, s.filter_glossy = settings.clamp_indirect, settings.filter_glossy
        self.scene = s

    def render(self, frame: np.ndarray, accum: np.ndarray, accumulated: int, count: int, seed: int, mask=None):
        """One Trace::sample(count, seed) pass on `accum` (H, W, 12 floats,
        updated in place); returns (color, albedo, normal) films.  With `mask`
        (H, W bools) only those pixels are reset and sampled."""
        f = np.array(frame, np.uint32).copy()
        f[2], f[3], f[6] = accumulated, count, seed
        h, w = accum.shape[:2]
        color = np.zeros((h, w, 4), np.float32)
        albedo = np.zeros_like(color)
        normal = np.zeros_like(color)
        if mask is None:
            lib().orc_render(C.byref(self.scene), _p(f), _p(accum), _p(color), _p(albedo), _p(normal))
        else:
            m = np.ascontiguousarray(np.asarray(mask, bool).reshape(h, w).astype(np.uint8))
            L = lib()
            L.orc_render_masked.restype = C.c_int
            L.orc_render_masked.argtypes = [C.c_void_p] * 7
            L.orc_render_masked(C.byref(self.scene), _p(f), _p(accum), _p(color), _p(albedo), _p(normal), _p(m))
        return color, albedo, normal

    @staticmethod
    def ray_counts() -> tuple:
        """(closest, any) queries traced by render() since the last call."""
        L = lib()
        L.orc_ray_counts.restype = None
        L.orc_ray_counts.argtypes = [C.c_void_p]
        out = np.zeros(2, np.uint64)
        L.orc_ray_counts(_p(out))
        return int(out[0]), int(out[1])

    def converge(self, accum: np.ndarray, snaps: np.ndarray, min_samples: int, threshold: float, mark: bool) -> int:
        """measure (converge.wgsl:9-31), then mark (:32-51) when `mark`."""
        h, w = accum.shape[:2]
        return int(lib().orc_converge(_p(accum), _p(snaps), w, h, min_samples, threshold, 1 if mark else 0))

    def measure(self, accum: np.ndarray, snaps: np.ndarray) -> None:
        h, w = accum.shape[:2]
        lib().orc_converge(_p(accum), _p(snaps), w, h, 0, 0.0, 0)

    def mark(self, accum: np.ndarray, snaps: np.ndarray, min_samples: int, threshold: float) -> int:
        """mark alone, on errors already in `snaps`; returns the running count."""
        h, w = accum.shape[:2]
        return int(lib().orc_converge(_p(accum), _p(snaps), w, h, min_samples, threshold, 2))

    def tree_pick(self, points: np.ndarray, normals: np.ndarray, rands: np.ndarray):
        n = len(points)
        pts = np.ascontiguousarray(points, np.float32)
        nrm = np.ascontiguousarray(normals, np.float32)
        r = np.ascontiguousarray(rands, np.float32)
        light = np.zeros(n, np.int32)
        pmf = np.zeros(n, np.float32)
        leaf = np.zeros(n, np.uint32)
        lib().orc_tree_pick(C.byref(self.scene), _p(pts), _p(nrm), _p(r), n, _p(light), _p(pmf), _p(leaf))
        return light, pmf, leaf

    def sample_adaptive(self, frame, width, height, adaptive, seed):
        """Trace::sample_adaptive (adaptive.rs:136-325) on the CPU: returns
        (rounds [(samples, active)], accum, films)."""
        accum = np.zeros((height, width, 12), np.float32)
        snaps = np.zeros((height, width, 8), np.float32)
        samples, rounds, films = 0, [], None
        for step, target in enumerate(adaptive.rounds()):
            count = max(target - samples, 0)
            if count:
                films = self.render(frame, accum, samples, count, seed)
            samples += count
            running = self.converge(accum, snaps, adaptive.min_samples, adaptive.threshold, step > 0)
            active = running if step > 0 else width * height
            rounds.append((target, active))
            if active == 0:
                break
        return rounds, accum, films
