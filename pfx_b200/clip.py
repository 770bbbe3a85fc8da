"""A clip: the frames of a moving camera rendered back to back.

The batched workload of the tracer: shots over procedural rooms of different
sizes (10k, 100k, 400k and 1M triangles by default), each with a camera that
follows a Catmull-Rom spline through 8 random keys while looking along a second
spline through 8 random points of interest.  Every frame is an independent
still: the camera moves (Trace::set_camera restarts the accumulation) and
`spp` samples are taken with the frame's index as the seed.

On the device a shot is one tracer on one stream: the camera travels in the
pass variables, not in the captured launch parameters, so every frame of a shot
replays the same CUDA graph (one capture per shot).  The launch choices are
autotuned once per shot, and a radiance cache, when asked for, is shared by all
frames of its shot (it learns the scene, not the view).

    python -m pfx_b200.clip [--frames 240] [--spp 16] [--size 1280x720] [--cache]

prints one JSON line: frames per second, Mrays/s and per-shot figures, all
device time measured with CUDA events on the tracers' streams.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import synth
from .trace import Camera, Trace

SCENE_TRIANGLES = (10_000, 100_000, 400_000, 1_000_000)


@dataclass
class Shot:
    """One scene and the camera path through it."""
    workload: synth.Workload
    keys: np.ndarray        # (8, 3) camera positions
    targets: np.ndarray     # (8, 3) points the camera looks at
    frames: int
    first_frame: int = 0    # index of this shot's first frame in the clip (the seed of that frame)
    vfov_deg: float = 60.0


def catmull_rom(points: np.ndarray, t: float) -> np.ndarray:
    """Uniform Catmull-Rom spline through `points` (n, 3) at t in [0, 1]: the
    curve passes through every point (t = k / (n - 1) gives point k) with a
    continuous tangent; the end segments repeat their end points."""
    p = np.asarray(points, np.float64)
    n = len(p)
    if n == 1:
        return p[0].copy()
    x = min(max(float(t), 0.0), 1.0) * (n - 1)
    k = min(int(math.floor(x)), n - 2)
    u = x - k
    p0, p1, p2, p3 = p[max(k - 1, 0)], p[k], p[k + 1], p[min(k + 2, n - 1)]
    return 0.5 * ((2.0 * p1) + (-p0 + p2) * u + (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3) * u * u +
                  (-p0 + 3.0 * p1 - 3.0 * p2 + p3) * u * u * u)


def camera_at(shot: Shot, frame: int) -> Camera:
    """The camera of frame `frame` (0-based within the shot)."""
    t = frame / max(shot.frames - 1, 1)
    eye = catmull_rom(shot.keys, t)
    target = catmull_rom(shot.targets, t)
    w = shot.workload
    return synth.look_at(tuple(eye), tuple(target), shot.vfov_deg, w.width / w.height)


def room_shot(triangles: int, seed: int, size=(1280, 720), frames: int = 60, sampler: str = "sobol") -> Shot:
    """A room of about `triangles` triangles (synth.room_4k's generator: room
    box, shelves, meshes of 1k-20k triangles) and a random camera path inside
    it: keys at eye heights 1.5-6 m within the room, points of interest on the
    floor and shelves."""
    meshes = max(1, int(round(triangles / 5000)))
    w = synth.room_4k(seed=seed, width=size[0], height=size[1], target=triangles, meshes_n=meshes, sampler=sampler)
    w.name = f"room_{triangles // 1000}k"
    rng = np.random.default_rng(seed + 7919)
    keys = np.stack([rng.uniform(-11.0, 11.0, 8), rng.uniform(1.5, 6.0, 8), rng.uniform(-11.0, 11.0, 8)], 1)
    targets = np.stack([rng.uniform(-12.0, 12.0, 8), rng.uniform(0.0, 4.0, 8), rng.uniform(-12.0, 12.0, 8)], 1)
    # never look straight down the path's own position
    close = np.linalg.norm(targets - keys, axis=1) < 1.0
    targets[close, 0] += 3.0
    return Shot(w, keys, targets, frames)


def clip_shots(frames: int = 240, size=(1280, 720), scene_triangles=SCENE_TRIANGLES, seed: int = 5,
               sampler: str = "sobol") -> list[Shot]:
    """The clip: `frames` frames split evenly over one shot per scene size."""
    n = len(scene_triangles)
    per = [frames // n + (1 if i < frames % n else 0) for i in range(n)]
    shots, first = [], 0
    for i, (tris, f) in enumerate(zip(scene_triangles, per)):
        s = room_shot(tris, seed + i, size, f, sampler)
        s.first_frame = first
        first += f
        shots.append(s)
    return shots


@dataclass
class ShotResult:
    name: str
    triangles: int
    frames: int
    device_s: float
    rays: int
    graph_captures: int
    create_s: float
    tuning: dict = field(default_factory=dict)


def render(shots: list[Shot], spp: int = 16, cache_settings=None, autotune: bool = True, on_frame=None,
           timed: bool = True) -> list[ShotResult]:
    """Render every frame of every shot: per frame set_camera, then `spp`
    samples in one sampling call with the clip frame index as the seed.
    `on_frame(index, trace)` is called after each frame (the films are the
    frame's image).  `cache_settings` attaches one RadianceCache per shot."""
    import torch

    from .cache import RadianceCache

    out = []
    for shot in shots:
        w = shot.workload
        t0 = time.perf_counter()
        trace = Trace(w.scene, w.settings, w.width, w.height)
        create_s = time.perf_counter() - t0
        cache = None
        if cache_settings is not None:
            cache = RadianceCache(cache_settings)
            trace.set_cache(cache)
        tuning = trace.autotune(passes=2) if autotune else trace.tuning()
        stream = torch.cuda.ExternalStream(trace._lib.pfxt_debug_stream(trace.handle))
        captures0 = trace._lib.pfxt_debug_graph_captures(trace.handle)
        rays0 = trace.rays_traced()
        device_ms = 0.0
        for f in range(shot.frames):
            trace.set_camera(camera_at(shot, f))
            if timed:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            trace.sample(spp, shot.first_frame + f)
            if timed:
                e1.record(stream)
                e1.synchronize()
                device_ms += e0.elapsed_time(e1)
            if on_frame is not None:
                on_frame(shot.first_frame + f, trace)
        rays1 = trace.rays_traced()
        out.append(ShotResult(w.name, int(w.scene.world_triangle_count), shot.frames, device_ms / 1e3,
                              int((rays1[0] - rays0[0]) + (rays1[1] - rays0[1])),
                              int(trace._lib.pfxt_debug_graph_captures(trace.handle) - captures0), create_s, tuning))
        trace.close()
        if cache is not None:
            cache.close()
    return out


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--frames", type=int, default=240)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--size", default="1280x720")
    ap.add_argument("--cache", action="store_true", help="one radiance cache per shot")
    args = ap.parse_args()
    size = tuple(int(x) for x in args.size.split("x"))
    shots = clip_shots(args.frames, size)
    settings = None
    if args.cache:
        from .cache import CacheSettings
        settings = CacheSettings()
    res = render(shots, args.spp, settings)
    device_s = sum(r.device_s for r in res)
    rays = sum(r.rays for r in res)
    print(json.dumps({
        "workload": f"clip: {args.frames} frames at {size[0]}x{size[1]}, {args.spp} spp per frame, shots over "
                    f"rooms of {', '.join(str(r.triangles) for r in res)} triangles"
                    + (", one radiance cache per shot" if args.cache else ""),
        "frames_per_s": args.frames / device_s, "Mrays_s": rays / device_s / 1e6, "device_s": device_s,
        "shots": [{"name": r.name, "triangles": r.triangles, "frames": r.frames, "device_s": r.device_s,
                   "ms_per_frame": 1e3 * r.device_s / r.frames, "Mrays_s": r.rays / r.device_s / 1e6,
                   "graph_captures": r.graph_captures, "create_s": r.create_s, "tuning": r.tuning} for r in res]}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
