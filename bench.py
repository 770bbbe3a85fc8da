#!/usr/bin/env python
"""Benchmark of the B200 path tracer; prints ONE JSON line on rank 0.

Workload (default): the 4K room scene (3840x2160, 1.19M triangles, 128 lights,
32 materials; pfx_b200.synth.room_4k) and a fixed batch with the ray mix of one
tracing pass: camera rays and cosine bounce rays (closest hit) plus shadow
rays to the lights (any hit).  One step = one closest-hit launch over the
closest batch and one any-hit launch over the shadow batch, inputs resident in
HBM.  The metric is Mrays/s = (closest + any-hit queries) / s.  L2 is flushed
(a 256 MiB write) before every timed step; the per-step device time comes from
CUDA events on the launching stream.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun); every rank traces its own batch
(different seeds), nothing is exchanged on the data path (weak scaling); the
time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0  # profiling recipe's fallback, used only without MEASURED_PEAKS.json


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM traffic of `kernel` from the committed ncu summary
    (profiles/traffic.json), scaled to this workload by the summary's rule."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text()).get(kernel)
    return None if d is None else d


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_workload(args, seed: int):
    from pfx_b200 import synth
    w = synth.room_4k(seed=2) if args.workload == "room_4k" else synth.WORKLOADS[args.workload]()
    return w


def cpu_baseline(trace, closest, shadow, budget_rays: int):
    """The oracle's traversal (the CPU restatement of scene()/occluded()) on a
    bounded sample of the same batches, all host threads."""
    import oracle
    n_c = min(len(closest), budget_rays // 2)
    n_s = min(len(shadow), budget_rays // 2)
    c, s = closest[:n_c], shadow[:n_s]
    oracle.trace(trace.scene_buffers, c[:256])  # warm the library
    t0 = time.perf_counter()
    oracle.trace(trace.scene_buffers, c)
    oracle.trace(trace.scene_buffers, s, any_hit=True)
    dt = time.perf_counter() - t0
    return {"value": (n_c + n_s) / dt / 1e6, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{n_c} closest-hit + {n_s} any-hit rays of the same batch, oracle traversal on all host threads"}


def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    w = build_workload(args, 0)
    from pfx_b200.trace import SceneBuffers
    import oracle
    from pfx_b200 import rays as raymix
    sb = SceneBuffers(w.scene, w.settings)

    class _T:  # ray generation needs closest hits; the oracle provides them here
        scene_buffers = sb

        def trace_rays(self, r):
            return oracle.trace(sb, r)

    per_step = min(args.rays, 1 << 17)
    closest, shadow = raymix.pass_mix(_T(), w.scene, w.width, w.height, per_step, seed=7)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.trace(sb, closest)
        oracle.trace(sb, shadow, any_hit=True)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    rays = (len(closest) + len(shadow)) * len(times)
    value = rays / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_of(args, w, len(closest), len(shadow)),
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{len(closest)} closest + {len(shadow)} any-hit rays per step; the reference's "
                                   "wgpu tracer cannot run on this box (no Rust, no graphics stack), so its CPU "
                                   "restatement (oracle/) runs on all host threads"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


METRIC = "Mrays/s, closest-hit + any-hit traversal of one tracing pass's ray mix (4K room, 1.19M triangles)"


def config_of(args, w, n_closest, n_shadow):
    return {"workload": f"{w.name}: {w.width}x{w.height}, {w.scene.world_triangle_count} triangles, "
                        f"{len(w.scene.lights)} lights, one-pass ray mix",
            "closest_rays_per_step": n_closest, "shadow_rays_per_step": n_shadow,
            "l2": "flushed before every timed step (256 MiB write)", "parallelism": f"replica-free pixel/ray shards x{args.gpus}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="room_4k")
    ap.add_argument("--rays", type=int, default=1 << 22, help="rays per step (closest + shadow)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    from pfx_b200 import rays as raymix
    from pfx_b200.trace import HIT, RAY, Trace

    w = build_workload(args, rank)
    trace = Trace(w.scene, w.settings, w.width, w.height)
    closest, shadow = raymix.pass_mix(trace, w.scene, w.width, w.height, args.rays, seed=7 + rank)
    nc, ns = len(closest), len(shadow)
    dev = torch.device("cuda", local)
    d_closest = torch.from_numpy(closest.view(np.uint8).copy()).to(dev)
    d_shadow = torch.from_numpy(shadow.view(np.uint8).copy()).to(dev)
    d_hits = torch.empty(nc * 16, dtype=torch.uint8, device=dev)
    d_blocked = torch.empty(ns * 4, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    # algorithmic bytes per query: 32 per box test, 36 per triangle test, 48 per ray (in + out)
    counts_c = torch.empty(nc * 2, dtype=torch.int32, device=dev)
    counts_s = torch.empty(ns * 2, dtype=torch.int32, device=dev)
    trace.counts_device(d_closest.data_ptr(), nc, False, counts_c.data_ptr(), sh)
    trace.counts_device(d_shadow.data_ptr(), ns, True, counts_s.data_ptr(), sh)
    torch.cuda.synchronize()
    cc = counts_c.view(-1, 2).double().sum(0).cpu().numpy()
    cs = counts_s.view(-1, 2).double().sum(0).cpu().numpy()
    bytes_closest = 32 * cc[0] + 36 * cc[1] + 48 * nc
    bytes_shadow = 32 * cs[0] + 36 * cs[1] + 48 * ns

    def step():
        trace.trace_rays_device(d_closest.data_ptr(), nc, d_hits.data_ptr(), sh)
        trace.occluded_device(d_shadow.data_ptr(), ns, d_blocked.data_ptr(), sh)

    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        for e0, e1, e2 in ev:
            flush.fill_(1)
            e0.record(stream)
            trace.trace_rays_device(d_closest.data_ptr(), nc, d_hits.data_ptr(), sh)
            e1.record(stream)
            trace.occluded_device(d_shadow.data_ptr(), ns, d_blocked.data_ptr(), sh)
            e2.record(stream)
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(c) for a, _, c in ev]
    closest_ms = [a.elapsed_time(b) for a, b, _ in ev]
    total_ms = sum(step_ms)
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
        pg.barrier()
    rays_per_step = nc + ns
    value = rays_per_step * world * args.steps / (total_ms / 1e3) / 1e6

    # end to end through the host-buffer entry points (pinned host memory,
    # copies in and results out inside the timed region)
    h_closest = torch.from_numpy(closest.view(np.uint8).copy()).pin_memory()
    h_shadow = torch.from_numpy(shadow.view(np.uint8).copy()).pin_memory()
    h_hits = torch.empty(nc * 16, dtype=torch.uint8).pin_memory()
    h_blocked = torch.empty(ns, dtype=torch.uint8).pin_memory()
    lib = trace._lib
    e2e_steps = max(3, args.steps // 2)
    lib.pfxt_trace_rays(trace.handle, h_closest.data_ptr(), nc, h_hits.data_ptr())
    lib.pfxt_occluded(trace.handle, h_shadow.data_ptr(), ns, h_blocked.data_ptr())
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        rc = lib.pfxt_trace_rays(trace.handle, h_closest.data_ptr(), nc, h_hits.data_ptr())
        rc |= lib.pfxt_occluded(trace.handle, h_shadow.data_ptr(), ns, h_blocked.data_ptr())
        assert rc == 0, lib.pfxt_last_error()
    e2e_s = time.perf_counter() - t0
    if pg:
        t = torch.tensor([e2e_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = rays_per_step * world * e2e_steps / e2e_s / 1e6

    if rank == 0:
        peak, peak_kind = peaks()
        closest_s = statistics.mean(closest_ms) / 1e3
        achieved = bytes_closest / closest_s / 1e9
        traffic = ncu_traffic("k_trace<0>")
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(args, w, nc, ns),
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": int((nc + ns) * 32),
                    "d2h_bytes_per_step": int(nc * 16 + ns)},
            "gpu_launches": 2 * args.steps,
            "roofline": {"bound": "hbm", "kernel": "k_trace<0> (closest-hit traversal)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": bytes_closest,
                         "bytes_per_ray": bytes_closest / nc,
                         "box_tests_per_ray": cc[0] / nc, "triangle_tests_per_ray": cc[1] / nc},
            "closest_ms_per_launch": statistics.mean(closest_ms),
            "clocks": clk.summary(),
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(trace, closest, shadow, 1 << 18)
        print(json.dumps(line))
    trace.close()
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
