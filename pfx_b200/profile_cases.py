"""Small, self-contained launches of the hot kernels for profiler captures.

    python -m pfx_b200.profile_cases traverse   # closest-hit traversal, 2^20 rays of a 4K pass mix
    python -m pfx_b200.profile_cases infer      # radiance-cache inference, 2^20 queries
    python -m pfx_b200.profile_cases train      # radiance-cache training, 2 steps of 2^16 records
    python -m pfx_b200.profile_cases shade      # two 960x540 passes of the 4K room (all pass kernels)
    python -m pfx_b200.profile_cases pass-plain # three 4K passes, plain
    python -m pfx_b200.profile_cases pass-cached# eight 4K passes with the radiance cache
    python -m pfx_b200.profile_cases denoise    # two denoises of a 1024x544 frame (one tile, 16 convolutions each)

Each case runs its kernel a few times on inputs larger than L2 where the
kernel's input allows, and holds a few GB on the device at most, so that a
capture of one or a few launches ends within a minute or two.  Prints "ok".
"""
from __future__ import annotations

import sys

import numpy as np


def traverse() -> None:
    import torch

    from . import rays, synth
    from .trace import Trace

    w = synth.room_4k()
    t = Trace(w.scene, w.settings, 64, 36)
    closest, _ = rays.pass_mix(t, w.scene, w.width, w.height, 1 << 21, seed=7)
    d_rays = torch.from_numpy(closest.view(np.uint8).copy()).cuda()
    d_hits = torch.empty(len(closest) * 16, dtype=torch.uint8, device="cuda")
    for _ in range(3):
        t.trace_rays_device(d_rays.data_ptr(), len(closest), d_hits.data_ptr(), 0)
    torch.cuda.synchronize()


def _cache():
    from .cache import CacheSettings, RadianceCache

    return RadianceCache(CacheSettings(lo=(-10.0, -1.0, -10.0), hi=(10.0, 10.0, 10.0)))


def infer() -> None:
    from .cache import random_queries

    c = _cache()
    q = random_queries(1 << 20, np.random.default_rng(1), (-10, -1, -10), (10, 10, 10))
    for _ in range(3):
        c.infer(q)


def train() -> None:
    from .cache import RECORD, random_queries

    c = _cache()
    rng = np.random.default_rng(2)
    r = np.zeros(2 << 16, RECORD)
    r["query"] = random_queries(len(r), rng, (-10, -1, -10), (10, 10, 10))
    r["target"] = rng.uniform(0, 2, (len(r), 3)).astype(np.float32)
    r["weight"] = 1.0
    c.train(r)


def shade() -> None:
    from . import synth
    from .trace import Trace

    w = synth.room_4k()
    t = Trace(w.scene, w.settings, 960, 540)
    for s in range(2):
        t.sample(1, s)


def passes(cached: bool) -> None:
    from . import synth
    from .cache import RadianceCache
    from .trace import Trace

    w = synth.room_4k()
    t = Trace(w.scene, w.settings, w.width, w.height)
    # the launch choices the autotuner makes for this scene (bench.py reports them)
    t.set_tuning(trace_threads=64, sort_shading=False)
    n = 3
    if cached:
        c = RadianceCache()
        t.set_cache(c)
        t.set_tuning(trace_threads=64, sort_shading=False)
        n = 8
    for s in range(n):
        t.sample(1, s)


def denoise() -> None:
    import torch

    from .denoise import DEFAULT_WEIGHTS, Denoiser, write_tza

    if DEFAULT_WEIGHTS.exists():
        den = Denoiser()
    else:  # seeded FP16 weights of the same shapes: the same work
        rng = np.random.default_rng(0)
        t = {}
        for name, o, i in [("enc_conv0", 32, 9), ("enc_conv1", 32, 32), ("enc_conv2", 48, 32), ("enc_conv3", 64, 48),
                           ("enc_conv4", 80, 64), ("enc_conv5a", 96, 80), ("enc_conv5b", 96, 96),
                           ("dec_conv4a", 112, 160), ("dec_conv4b", 112, 112), ("dec_conv3a", 96, 160),
                           ("dec_conv3b", 96, 96), ("dec_conv2a", 64, 128), ("dec_conv2b", 64, 64),
                           ("dec_conv1a", 64, 73), ("dec_conv1b", 32, 64), ("dec_conv0", 3, 32)]:
            t[f"{name}.weight"] = rng.normal(0, np.sqrt(2.0 / (9 * i)), (o, i, 3, 3)).astype(np.float16)
            t[f"{name}.bias"] = np.zeros(o, np.float16)
        den = Denoiser(write_tza(t))
    h, w = 544, 1024
    rng = np.random.default_rng(1)
    imgs = [torch.from_numpy(rng.uniform(0, 1, (h, w, 4)).astype(np.float32)).cuda() for _ in range(3)]
    out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
    for _ in range(2):
        den.denoise_device(w, h, *(x.data_ptr() for x in imgs), out.data_ptr(), 0)
        den.last()


def main() -> None:
    case = sys.argv[1] if len(sys.argv) > 1 else "traverse"
    {"traverse": traverse, "infer": infer, "train": train, "shade": shade,
     "pass-plain": lambda: passes(False), "pass-cached": lambda: passes(True), "denoise": denoise}[case]()
    print("ok", case)


if __name__ == "__main__":
    main()
