#!/usr/bin/env python
"""Benchmark of the B200 path tracer; prints ONE JSON line on rank 0.

Workload: the 4K room (3840x2160, 1.19M triangles, 32 materials with glass and
metals, 128 point/spot lights through the light tree, depth 8, Sobol sampler;
pfx_b200.synth.room_4k), synthetic and seeded.  One step = one sampling pass
(one sample for all 8.3M pixels) through the wavefront tracer, scene resident
in HBM; L2 is flushed before every timed step.  Device time comes from CUDA
events recorded on the tracer's own stream.

  value            Mrays/s = closest-hit + any-hit queries traced per second
  time_to_relmse   seconds of sampling passes until relMSE <= 0.01, relMSE =
                   mean over pixels and channels of (I-R)^2 / (R^2 + 0.01), R a
                   4096-spp reference accumulated in FP64 over every 8th pixel
                   in x and y (a stratified 480x270 subset of the 4K frame);
                   the error is followed on those pixels alone (their values do
                   not depend on the other pixels) and the time is spp x the
                   full-frame pass time measured above.  The cached tracer
                   (radiance cache at vertex 1, trained online from an untrained
                   start) runs full-frame passes; its time is the sum of their
                   event-timed durations, training included, L2 flushed before
                   each; relMSE evaluation is outside the timed regions
  roofline         the closest-hit traversal kernel on a batch with the ray mix
                   of one pass (the same traversal code as the tracer's extend
                   kernel): algorithmic bytes 32*box + 36*tri + 48 per ray over
                   its event-timed launch
  e2e              Trace::sample(1) + Trace::readback(colour) through the C ABI
                   per step, host wall clock, film copied into pinned memory

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun); every rank renders the full frame
with its own seed, nothing is exchanged (weak scaling); time = max over ranks.
The relMSE measurement runs at N=1 only.
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

FALLBACK_HBM_GBS = 6650.0  # used only when MEASURED_PEAKS.json is absent
METRIC = "time to relMSE 0.01 at 4K, cached vs plain tracer on one B200; Mrays/s"
TARGET_RELMSE = 0.01


FALLBACK_BF16_TFLOPS = 1590.0  # dense bf16 burst, used only when MEASURED_PEAKS.json is absent


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def tensor_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return FALLBACK_BF16_TFLOPS, "fallback"


def ncu_traffic(kernel: str, rays: int):
    """DRAM bytes (read + write) of one launch of `kernel` over `rays` rays: the
    committed ncu capture's bytes scaled linearly by rays (an upper bound: the
    scene's L2 misses do not grow with the ray count)."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    e = json.loads(p.read_text()).get(kernel)
    if not e:
        return None
    return e["dram_bytes"] * rays / e["captured_rays"]


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device, self.proc, self.file = device_index, None, None

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
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(rank: int) -> int:
    """First pass seed of a rank: every rank renders its own frame (weak scaling)."""
    return 1000 * (rank + 1)


def combine_ranks(pg, elapsed: float, units: float, device):
    """(max of `elapsed` over ranks, sum of `units` over ranks): the job's time is
    its slowest rank's, its work every rank's.  `pg` is torch.distributed or None."""
    if pg is None:
        return elapsed, units
    import torch
    t = torch.tensor([elapsed, units], dtype=torch.float64, device=device)
    tmax = t.clone()
    pg.all_reduce(tmax, op=pg.ReduceOp.MAX)
    tsum = t.clone()
    pg.all_reduce(tsum, op=pg.ReduceOp.SUM)
    return float(tmax[0].item()), float(tsum[1].item())


def workload(name: str):
    from pfx_b200 import synth
    return synth.WORKLOADS[name]()


def config_of(w, args, extra=None):
    c = {"workload": f"{w.name}: {w.width}x{w.height}, {w.scene.world_triangle_count} triangles, "
                     f"{len(w.scene.lights)} point/spot lights (light tree), {len(w.scene.materials)} materials "
                     f"(2 glass IOR 1.5, metals), depth {w.settings.bounces[0]}, {w.settings.sampler} sampler, "
                     f"filter_glossy {w.settings.filter_glossy:g}, clamp_indirect {w.settings.clamp_indirect:g}; "
                     f"fixed 1 spp per step, not adaptive",
         "step": "one sampling pass (1 spp, every pixel; adaptive stopping off)",
         "l2": "flushed before every timed step (256 MiB write)",
         "parallelism": f"independent frames x{args.gpus} (no collective on the data path)"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ reference
def run_reference(args):
    """The reference's path on the host cores: the oracle (a C++ restatement of
    crates/trace's main()/radiance()) on a bounded window of the same frame.
    The reference's own wgpu tracer cannot run here (no Rust toolchain, no
    graphics stack)."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    w = workload(args.workload)
    sb = oracle.scene_buffers(w.scene, w.settings)  # the oracle's own packing: no product code on this arm
    r = oracle.Renderer(sb, w.settings)
    ww, wh = 160, 90
    x0, y0 = (w.width - ww) // 2, (w.height - wh) // 2
    frame = oracle.frame_of(w.scene, ww, wh, sb.buffers.triangle_count, window=(w.width, w.height, x0, y0))
    accum = np.zeros((wh, ww, 12), np.float32)
    times, rays = [], 0
    for i in range(args.warmup + args.steps):
        oracle.Renderer.ray_counts()
        t0 = time.perf_counter()
        r.render(frame, accum, 0, 1, i)
        dt = time.perf_counter() - t0
        c = oracle.Renderer.ray_counts()
        if i >= args.warmup:
            times.append(dt)
            rays += c[0] + c[1]
    value = rays / sum(times) / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_of(w, args),
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"each step a {ww}x{wh} centre window of the {w.width}x{w.height} frame at 1 spp "
                                   "(the same scene, settings and pixels' samples as the full frame), oracle path "
                                   "tracer on its own scene packing, all host threads; the reference's wgpu tracer "
                                   "is unavailable on this box"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


# ------------------------------------------------------------------ ours
def relmse(img, ref):
    """mean over pixels and channels of (I-R)^2 / (R^2 + 0.01), in FP64."""
    d = img.double() - ref
    return float((d * d / (ref * ref + 0.01)).mean())


def masked_trace(w, mask):
    from pfx_b200.trace import Trace
    t = Trace(w.scene, w.settings, w.width, w.height)
    t.set_pixel_mask(mask)
    return t


def reference_image(w, args, mask, mask_idx):
    """The reference over the masked pixels: args.ref_spp samples accumulated in
    FP64 on the device, in chunks of 64 with their own seeds."""
    import torch
    ref_trace = masked_trace(w, mask)
    chunk = 64
    total = torch.zeros((len(mask_idx), 3), dtype=torch.float64, device="cuda")
    chunks = max(1, args.ref_spp // chunk)
    t0 = time.perf_counter()
    for c in range(chunks):
        ref_trace.set_camera(w.scene.camera)  # restarts the accumulation
        ref_trace.sample(chunk, 100_000 + c)
        color = ref_trace.films_device()[0].reshape(-1, 4)
        total += color[mask_idx, :3].double()
    ref = total / chunks
    ref_trace.close()
    return ref, time.perf_counter() - t0


def plain_convergence(w, mask, mask_idx, ref, max_spp):
    """Samples per pixel the plain tracer needs to reach the target relMSE.

    A pixel's samples depend only on the pixel, the sample index and the pass
    seed, never on which other pixels are traced, so a pass over the masked
    pixels gives exactly the values a full-frame pass gives there; the time to
    the target is then the spp count times the full-frame pass time."""
    t = masked_trace(w, mask)
    color = t.films_device()[0].reshape(-1, 4)
    curve = []
    for p in range(max_spp):
        t.sample(1, 50_000 + p)
        err = relmse(color[mask_idx, :3], ref)
        curve.append((p + 1, err))
        if err <= TARGET_RELMSE:
            break
    t.close()
    reached = curve[-1][1] <= TARGET_RELMSE
    return (curve[-1][0] if reached else None), curve


def cache_settings(args):
    """The radiance cache of the 4K workload: 16 levels x 2^19 entries, 64-wide
    MLP, 2^16 records per step, 4 steps per pass, paths end at vertex 1 (the first scattering vertex after the
    camera hit), glossy vertices delaying that by up to two."""
    from pfx_b200.cache import CacheSettings
    s = CacheSettings()
    if args.cache_error_bound is not None:
        s.error_bound = args.cache_error_bound
    if args.cache_min_roughness is not None:
        s.min_roughness = args.cache_min_roughness
    if args.cache_query_bounce is not None:
        s.query_bounce = args.cache_query_bounce
    if args.cache_delay_bounces is not None:
        s.delay_bounces = args.cache_delay_bounces
    if args.cache_train_fraction is not None:
        s.train_fraction = args.cache_train_fraction
    return s


def cached_convergence(trace, w, mask_idx, ref, stream, flush, max_spp, cache_settings):
    """The cached tracer on the full frame from an untrained cache: device time
    of every sampling pass (online training included, L2 flushed before each),
    summed until the masked pixels reach the target relMSE."""
    import torch
    from pfx_b200.cache import RadianceCache
    # the launch choices of the cached pass, tuned on a cache that is then dropped
    scratch = RadianceCache(cache_settings)
    trace.set_cache(scratch)
    tuning = trace.autotune(passes=3)
    trace.set_cache(None)
    scratch.close()
    cache = RadianceCache(cache_settings)
    trace.set_cache(cache)  # restarts the accumulation
    color = trace.films_device()[0].reshape(-1, 4)
    elapsed, curve, pass_ms = 0.0, [], []
    reached = None
    for p in range(max_spp):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        trace.sample(1, 50_000 + p)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        pass_ms.append(ms)
        elapsed += ms / 1e3
        err = relmse(color[mask_idx, :3], ref)
        curve.append((p + 1, round(elapsed, 3), err))
        if err <= TARGET_RELMSE:
            reached = p + 1
            break
    stats = cache.stats()
    trace.set_cache(None)
    cache.close()
    stats["tuning"] = tuning
    return reached, elapsed, statistics.median(pass_ms), curve, stats


def traversal_roofline(trace, w, dev, stream, flush):
    """Closest-hit kernel on a one-pass ray mix, timed with events on its stream."""
    import torch
    from pfx_b200 import rays as raymix
    closest, _ = raymix.pass_mix(trace, w.scene, w.width, w.height, 1 << 22, seed=7)
    n = len(closest)
    d_rays = torch.from_numpy(closest.view(np.uint8).copy()).to(dev)
    d_hits = torch.empty(n * 16, dtype=torch.uint8, device=dev)
    counts = torch.empty(n * 2, dtype=torch.int32, device=dev)
    sh = stream.cuda_stream
    trace.counts_device(d_rays.data_ptr(), n, False, counts.data_ptr(), sh)
    torch.cuda.synchronize()
    c = counts.view(-1, 2).double().sum(0).cpu().numpy()
    algorithmic = 32 * c[0] + 36 * c[1] + 48 * n
    for _ in range(3):
        trace.trace_rays_device(d_rays.data_ptr(), n, d_hits.data_ptr(), sh)
    ms = []
    for _ in range(5):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        trace.trace_rays_device(d_rays.data_ptr(), n, d_hits.data_ptr(), sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    launch_s = statistics.mean(ms) / 1e3
    peak, kind = peaks()
    achieved = algorithmic / launch_s / 1e9
    return {"bound": "hbm", "kernel": "k_trace<0>: closest-hit traversal (the extend kernel's walk)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": kind,
            "traffic": ncu_traffic("k_trace<0>", n), "algorithmic_bytes_per_launch": algorithmic,
            "rays_per_launch": n, "box_tests_per_ray": c[0] / n, "triangle_tests_per_ray": c[1] / n,
            "launch_ms": statistics.mean(ms), "Mrays_s": n / launch_s / 1e6}


def cpu_baseline(w, budget_s=12.0):
    """The oracle path tracer on a window of the same frame, all host threads."""
    import oracle
    sb = oracle.scene_buffers(w.scene, w.settings)
    r = oracle.Renderer(sb, w.settings)
    ww, wh = 160, 90
    x0, y0 = (w.width - ww) // 2, (w.height - wh) // 2
    frame = oracle.frame_of(w.scene, ww, wh, sb.buffers.triangle_count, window=(w.width, w.height, x0, y0))
    accum = np.zeros((wh, ww, 12), np.float32)
    oracle.Renderer.ray_counts()
    t0, spp = time.perf_counter(), 0
    while time.perf_counter() - t0 < budget_s or spp == 0:
        r.render(frame, accum, 0, 1, spp)
        spp += 1
    dt = time.perf_counter() - t0
    c = oracle.Renderer.ray_counts()
    return {"value": (c[0] + c[1]) / dt / 1e6, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{ww}x{wh} centre window of the 4K frame, {spp} x 1 spp, oracle path tracer on all host threads"}


def denoise_line(trace, w, stream):
    """The denoiser on the 4K frame's films (after the timed passes): device
    time of the whole filter (exposure, both tiles' 16 convolutions, input and
    output processing) with CUDA events, 3 warm-up runs then the median of 5;
    end to end through the host-buffer call (three images up, one down); the
    convolutions' FLOPs (2 x multiply-adds at the padded channel counts, once:
    the hi/lo split doubles the tensor-core work, not the algorithm's) against
    the dense FP16/BF16 tensor peak.  OIDN's weights when fetched, else seeded
    FP16 weights of the same shapes (the same work)."""
    import statistics

    import torch

    from pfx_b200.denoise import DEFAULT_WEIGHTS, Denoiser, write_tza
    if DEFAULT_WEIGHTS.exists():
        den, weights = Denoiser(), "OIDN 2.5.1 rt_hdr_alb_nrm.tza"
    else:
        rng = np.random.default_rng(0)
        shapes = [("enc_conv0", 32, 9), ("enc_conv1", 32, 32), ("enc_conv2", 48, 32), ("enc_conv3", 64, 48),
                  ("enc_conv4", 80, 64), ("enc_conv5a", 96, 80), ("enc_conv5b", 96, 96), ("dec_conv4a", 112, 160),
                  ("dec_conv4b", 112, 112), ("dec_conv3a", 96, 160), ("dec_conv3b", 96, 96),
                  ("dec_conv2a", 64, 128), ("dec_conv2b", 64, 64), ("dec_conv1a", 64, 73),
                  ("dec_conv1b", 32, 64), ("dec_conv0", 3, 32)]
        t = {}
        for name, o, i in shapes:
            t[f"{name}.weight"] = rng.normal(0, np.sqrt(2.0 / (9 * i)), (o, i, 3, 3)).astype(np.float16)
            t[f"{name}.bias"] = np.zeros(o, np.float16)
        den, weights = Denoiser(write_tza(t)), "seeded FP16 weights of OIDN's shapes (OIDN's not fetched)"
    color, albedo, normal = (f.data_ptr() for f in trace.films_device())
    out = torch.empty((w.height, w.width, 4), dtype=torch.float32, device="cuda")
    ms = []
    for k in range(8):
        den.denoise_device(w.width, w.height, color, albedo, normal, out.data_ptr(), stream.cuda_stream)
        m, macs = den.last()
        if k >= 3:
            ms.append(m)
    device_ms = statistics.median(ms)
    films = trace.readback()
    den.denoise(films.color, films.albedo, films.normal)  # untimed: allocates the pinned staging
    e2e = []
    for _ in range(3):
        t0 = time.perf_counter()
        den.denoise(films.color, films.albedo, films.normal)
        e2e.append((time.perf_counter() - t0) * 1e3)
    peak, source = tensor_peak()
    tflops = 2.0 * macs / (device_ms * 1e-3) / 1e12
    tiles = den.tiles()
    den.close()
    return {"workload": f"OIDN RT filter on the {w.width}x{w.height} frame's colour/albedo/normal films, "
                        f"{tiles[2]} tiles of {tiles[0]}x{tiles[1]}", "weights": weights,
            "device_ms": round(device_ms, 3), "frames_per_s": round(1e3 / device_ms, 2),
            "e2e_ms": round(statistics.median(e2e), 3),
            "e2e": {"h2d_bytes": 3 * w.width * w.height * 16, "d2h_bytes": w.width * w.height * 16},
            "roofline": {"bound": "tensor", "kernel": "k_conv (16 layers x tiles)",
                         "achieved": round(tflops, 1), "peak": peak, "unit": "TFLOP/s",
                         "frac": round(tflops / peak, 4), "peak_source": source,
                         "flops_per_frame": 2 * macs},
            "reference": "274 ms on an RX 9060 XT, textures in and out (docs/denoise.md:63-67)"}


def clip_line(frames: int):
    """The batched clip workload (1280x720, 16 spp per frame, shots over rooms
    of 10k/100k/400k/1M triangles, the camera moving every frame): `frames`
    frames split evenly over the four shots, device time of the sampling calls."""
    from pfx_b200 import clip
    shots = clip.clip_shots(frames, (1280, 720))
    res = clip.render(shots, spp=16)
    device_s = sum(r.device_s for r in res)
    rays = sum(r.rays for r in res)
    return {"workload": f"clip: 1280x720, 16 spp per frame, {frames} frames over shots of "
                        f"{', '.join(str(r.triangles) for r in res)} triangles (the 240-frame clip's shots, "
                        f"{frames // len(res)} frames each)",
            "frames_per_s": frames / device_s, "Mrays_s": rays / device_s / 1e6, "device_s": device_s,
            "ms_per_frame": [round(1e3 * r.device_s / r.frames, 2) for r in res],
            "graph_captures": [r.graph_captures for r in res]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="room_4k")
    ap.add_argument("--ref-spp", type=int, default=4096)
    ap.add_argument("--stride", type=int, default=8)
    ap.add_argument("--max-spp", type=int, default=2048)
    ap.add_argument("--max-cached-spp", type=int, default=1024)
    ap.add_argument("--cache-error-bound", type=float, default=None)
    ap.add_argument("--cache-min-roughness", type=float, default=None)
    ap.add_argument("--cache-query-bounce", type=int, default=None)
    ap.add_argument("--cache-delay-bounces", type=int, default=None)
    ap.add_argument("--cache-train-fraction", type=float, default=None)
    ap.add_argument("--no-relmse", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-denoise", action="store_true")
    ap.add_argument("--clip-frames", type=int, default=48, help="frames of the clip line (0: none)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180), device_id=torch.device("cuda", local))
        pg = dist
    from pfx_b200.trace import Trace

    dev = torch.device("cuda", local)
    w = workload(args.workload)
    t0 = time.perf_counter()
    trace = Trace(w.scene, w.settings, w.width, w.height)
    create_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tuning = trace.autotune(passes=3) if not args.no_autotune else trace.tuning()
    autotune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(trace._lib.pfxt_debug_stream(trace.handle), device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    seed0 = rank_seed(rank)

    for i in range(args.warmup):
        trace.sample(1, seed0 + i)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    before = trace.rays_traced()
    step_ms = []
    with Clocks(local) as clk:
        for i in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            trace.sample(1, seed0 + 100 + i)
            e1.record(stream)
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
    after = trace.rays_traced()
    rays = (after[0] - before[0]) + (after[1] - before[1])
    total_ms, rays_all = combine_ranks(pg, sum(step_ms), float(rays), dev)
    value = rays_all / (total_ms / 1e3) / 1e6

    # e2e: sample + readback of the colour film through the host-buffer API
    film = torch.empty((w.height, w.width, 4), dtype=torch.float32).pin_memory()
    lib = trace._lib
    e2e_steps = max(3, args.steps // 2)
    r0 = trace.rays_traced()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        rc = lib.pfxt_sample(trace.handle, 1, seed0 + 500 + i)
        rc |= lib.pfxt_readback(trace.handle, film.data_ptr(), None, None)
        assert rc == 0, lib.pfxt_last_error()
    e2e_s = time.perf_counter() - t0
    r1 = trace.rays_traced()
    e2e_s, e2e_rays = combine_ranks(pg, e2e_s, float((r1[0] - r0[0]) + (r1[1] - r0[1])), dev)
    e2e_value = e2e_rays / e2e_s / 1e6

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(w, args), "rays_per_step": rays / args.steps,
            "Mpaths_s": w.width * w.height * world * args.steps / (total_ms / 1e3) / 1e6,
            "create_s": create_s, "autotune": {**tuning, "seconds": autotune_s},
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(w.width * w.height * 16),
                    "note": "scene uploaded once by Trace::new (create_s); per step one pass and the colour film"},
            # the kernel nodes of the pass's captured graph, one pass per step
            "gpu_launches": args.steps * trace.pass_kernels(),
            "clocks": clk.summary(),
        }
        line["roofline"] = traversal_roofline(trace, w, dev, stream, flush)
        if world == 1 and not args.no_relmse:
            mask = np.zeros((w.height, w.width), bool)
            s = args.stride
            mask[s // 2::s, s // 2::s] = True
            mask_idx = torch.from_numpy(np.flatnonzero(mask.reshape(-1))).to(dev)
            ref, ref_s = reference_image(w, args, mask, mask_idx)
            spp_plain, curve = plain_convergence(w, mask, mask_idx, ref, args.max_spp)
            pass_s = total_ms / args.steps / 1e3
            settings = cache_settings(args)
            spp_c, t_c, pass_c, curve_c, stats = cached_convergence(trace, w, mask_idx, ref, stream, flush,
                                                                    args.max_cached_spp, settings)
            plain_s = None if spp_plain is None else spp_plain * pass_s
            line["time_to_relmse"] = {
                "target": TARGET_RELMSE, "plain_spp": spp_plain, "plain_s": plain_s, "pass_s": pass_s,
                "cached_spp": spp_c, "cached_s": t_c if spp_c else None, "cached_pass_s": pass_c / 1e3,
                "speedup": (plain_s / t_c) if (plain_s and spp_c) else None,
                "reference": f"{args.ref_spp} spp accumulated in FP64 over every {s}th pixel in x and y "
                             f"({int(mask.sum())} pixels), {ref_s:.1f} s",
                "cache": {k: v for k, v in settings.__dict__.items() if k not in ("lo", "hi")},
                "cache_stats": stats,
                "plain_curve": [(n, round(e, 5)) for n, e in curve[:: max(1, len(curve) // 12)] + curve[-1:]],
                "cached_curve": [(n, t, round(e, 5)) for n, t, e in
                                 curve_c[:: max(1, len(curve_c) // 12)] + curve_c[-1:]]}
        if world == 1 and not args.no_denoise:
            line["denoise"] = denoise_line(trace, w, stream)
        if world == 1 and args.clip_frames > 0:
            line["clip"] = clip_line(args.clip_frames)
        if world == 1 and not args.no_cpu_baseline:  # the host baseline is timed at N=1 only
            line["cpu_baseline"] = cpu_baseline(w)
        print(json.dumps(line))
    trace.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
