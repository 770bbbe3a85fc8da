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
                                   for p in [HERE / "oracle.cpp", HERE.parent / "pfx_b200/csrc/pfxt_math.h"]
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
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


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
