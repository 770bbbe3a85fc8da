"""The tracer with the radiance cache attached.

* With every fallback cell closed (error bound 0) no path ends into the cache:
  the image must be the plain tracer's bit for bit, while the training paths
  still feed the cache (training paths are plain paths that also record).
* With the cache open, paths end into it at the query bounce and the image
  stays finite and close to the plain one."""
import numpy as np
import pytest

from pfx_b200 import synth
from pfx_b200.cache import CacheSettings, RadianceCache
from pfx_b200.trace import Trace

pytestmark = pytest.mark.gpu


def small_cache(**kw):
    base = dict(log2_entries=14, base_resolution=8, max_resolution=512, batch=256, steps=2, train_fraction=0.05)
    base.update(kw)
    return RadianceCache(CacheSettings(**base))


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_closed_cells_render_the_plain_image(gpu, sampler):
    w = synth.small("room_4k", (64, 40), sampler=sampler)
    plain = Trace(w.scene, w.settings, w.width, w.height)
    cached = Trace(w.scene, w.settings, w.width, w.height)
    cache = small_cache(error_bound=0.0)
    cached.set_cache(cache)
    for seed in range(4):
        plain.sample(2, seed)
        cached.sample(2, seed)
    assert np.array_equal(plain.read_accum(), cached.read_accum())
    st = cache.stats()
    assert st["queries"] == 0 and st["records"] > 0 and st["training_paths"] > 0
    assert st["steps"] >= 4


def test_open_cache_ends_paths(gpu):
    w = synth.small("room_4k", (64, 40), sampler="sobol")
    trace = Trace(w.scene, w.settings, w.width, w.height)
    cache = small_cache(error_bound=1e30, train_fraction=0.5, batch=1024, steps=4)
    trace.set_cache(cache)
    for seed in range(24):
        trace.sample(1, seed)
    st = cache.stats()
    assert st["cells_ok"] > 0 and st["queries"] > 0
    out = trace.readback()
    assert np.isfinite(out.color).all()
    trace.set_cache(None)
    trace.sample(1, 99)
    assert cache.stats()["queries"] == st["queries"]  # detached: nothing more asked of it


def test_the_cache_lowers_the_error_at_equal_device_time(gpu):
    """What the trained network gains over the tracer without it: on the
    reduced room (60 k triangles) at 1920x1080 with the default cache, both
    tracers given the same device time (CUDA events on each tracer's stream;
    the cache starts untrained and trains online inside its passes), the
    cached image's relMSE against a 128-spp plain reference is lower than the
    plain image's.  At a few hundred pixels a pass is launch-bound and the
    cache's fixed cost per pass (inference and training launches) buys
    nothing; the film here is large enough for the pass to be bandwidth-bound,
    as at the full 4K frame."""
    import torch

    from pfx_b200.trace import Settings

    w = synth.small("room_4k", (1920, 1080), sampler="sobol")
    w.settings = Settings.deep(8, sampler="sobol", sobol_samples=256, filter_glossy=0.25, clamp_indirect=4.0)

    def stream_of(t):
        return torch.cuda.ExternalStream(t._lib.pfxt_debug_stream(t.handle))

    def timed_pass(t, seed):
        s = stream_of(t)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        t.sample(1, seed)
        b.record(s)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    reference = Trace(w.scene, w.settings, w.width, w.height)
    reference.sample(128, 9000)
    ref = reference.readback().color[..., :3].astype(np.float64)
    reference.close()

    def relmse(t):
        img = t.readback().color[..., :3].astype(np.float64)
        return float(np.mean((img - ref) ** 2 / (ref * ref + 0.01)))

    cached = Trace(w.scene, w.settings, w.width, w.height)
    cache = RadianceCache(CacheSettings())
    cached.set_cache(cache)
    budget = sum(timed_pass(cached, seed) for seed in range(32))
    cached_err = relmse(cached)

    plain = Trace(w.scene, w.settings, w.width, w.height)
    spent, passes = 0.0, 0
    while spent < budget and passes < 512:
        spent += timed_pass(plain, passes)
        passes += 1
    plain_err = relmse(plain)
    print(f"equal device time {budget:.1f} ms: cached relMSE {cached_err:.5f} (32 passes), "
          f"plain {plain_err:.5f} ({passes} passes)")
    assert cache.stats()["queries"] > 0
    assert cached_err < plain_err, (cached_err, plain_err, passes, budget)
