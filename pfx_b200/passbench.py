"""Time sampling passes of one workload on the current GPU.

    python -m pfx_b200.passbench --workload room_4k --passes 3 [--width W --height H]

Prints one JSON line: milliseconds per one-sample pass (CUDA events on the
tracer's own stream), closest-hit and any-hit queries per pass, Mrays/s and
Mpaths/s.  Used for profiling runs; bench.py is the benchmark.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="room_4k")
    ap.add_argument("--passes", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--sampler", default="sobol")
    args = ap.parse_args()

    import torch

    from . import synth
    from .trace import Trace

    w = synth.WORKLOADS[args.workload](sampler=args.sampler)
    if args.width and args.height:
        w = synth.small(args.workload, (args.width, args.height), sampler=args.sampler)
    t0 = time.perf_counter()
    tr = Trace(w.scene, w.settings, w.width, w.height)
    create_s = time.perf_counter() - t0
    lib = tr._lib
    stream = torch.cuda.ExternalStream(lib.pfxt_debug_stream(tr.handle))
    for p in range(args.warmup):
        tr.sample(1, 1000 + p)
    rays = np.zeros(2, np.uint64)
    lib.pfxt_debug_rays(tr.handle, rays.ctypes.data)
    before = rays.copy()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for p in range(args.passes):
        tr.sample(1, p)
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end) / args.passes
    lib.pfxt_debug_rays(tr.handle, rays.ctypes.data)
    d = (rays - before).astype(np.float64) / args.passes
    print(json.dumps({"workload": w.name, "width": w.width, "height": w.height,
                      "triangles": w.scene.world_triangle_count, "create_s": create_s, "ms_per_pass": ms,
                      "closest_per_pass": d[0], "any_per_pass": d[1], "Mrays_s": d.sum() / ms / 1e3,
                      "Mpaths_s": w.width * w.height / ms / 1e3}))
    tr.close()


if __name__ == "__main__":
    main()
