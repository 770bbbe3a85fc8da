"""One frame split over tracers (pfx_b200.shard) on one GPU.

  * contiguous bands, each traced by its own tracer through Trace::set_window
    (gpu.rs:2836), are the rows of the whole frame's render bit for bit;
  * golden-ratio strips, each rank's sampled by its own full-frame tracer
    through pfxt_set_pixel_mask, are the whole frame's rows bit for bit;
  * an adaptive render split over three strip tracers with the one-row error
    halo written between measure and mark (pfxt_adaptive_measure,
    pfxt_adaptive_snaps_device, pfxt_adaptive_mark) has the rounds and the
    accumulation of one tracer's Trace::sample_adaptive.  The three tracers
    run one after another on this GPU; between GPUs the same steps run with
    one all-gather and one all-reduce per round (shard.sample_adaptive)."""
import numpy as np
import pytest

from pfx_b200 import shard, synth
from pfx_b200.trace import Adaptive, Settings, Trace

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ranks", [2, 3])
def test_bands_are_the_rows_of_the_frame(gpu, ranks):
    w = synth.small("instanced_1080", (48, 23), sampler="sobol")
    whole = Trace(w.scene, w.settings, w.width, w.height)
    whole.sample(2, 5)
    accum, color = whole.read_accum(), whole.readback().color
    for r in range(ranks):
        t, (first, rows) = shard.render_band(w.scene, w.settings, w.width, w.height, r, ranks, 2, 5)
        assert np.array_equal(t.read_accum().view(np.uint32), accum[first:first + rows].view(np.uint32))
        assert np.array_equal(t.readback().color.view(np.uint32), color[first:first + rows].view(np.uint32))


@pytest.mark.parametrize("ranks", [2, 3])
def test_strips_are_the_rows_of_the_frame(gpu, ranks):
    w = synth.small("room_4k", (48, 40), sampler="sobol")
    whole = Trace(w.scene, w.settings, w.width, w.height)
    whole.sample(2, 6)
    accum = whole.read_accum()
    seen = np.zeros(w.height, bool)
    for r in range(ranks):
        t = shard.render_strips(w.scene, w.settings, w.width, w.height, r, ranks, 2, 6)
        rows = t.rows()
        mine = t.trace.read_accum()
        assert np.array_equal(mine[rows].view(np.uint32), accum[rows].view(np.uint32))
        others = np.setdiff1d(np.arange(w.height), rows)
        assert not mine[others].any()  # other ranks' strips are not sampled here
        seen[rows] = True
    assert seen.all()


def test_adaptive_strips_with_the_halo_render_the_whole_frame(gpu):
    import torch

    w = synth.small("instanced_1080", (40, 30), sampler="sobol")
    w.settings = Settings.deep(8, sampler="sobol", sobol_samples=64)
    adaptive = Adaptive(threshold=0.05, min_samples=8, max_samples=32, growth=1.5)
    whole = Trace(w.scene, w.settings, w.width, w.height)
    want = whole.sample_adaptive(adaptive, 11)
    want_accum = whole.read_accum()

    ranks = 3
    ts = [shard.StripTracer(Trace(w.scene, w.settings, w.width, w.height), r, ranks) for r in range(ranks)]
    samples, rounds = 0, []
    for step, target in enumerate(adaptive.rounds()):
        count = max(target - samples, 0)
        for t in ts:
            if count:
                t.sample(count, 11)
        samples += count
        for t in ts:
            t.measure(step == 0)
        if step == 0:
            active = w.width * w.height
        else:
            for t in ts:  # the halo: rows next to t's strips, from the edge rows of their owners
                for o in ts:
                    if o is not t:
                        rows = np.intersect1d(shard.halo_rows(w.height, t.blocks), o.rows())
                        if len(rows):
                            t.set_errors(rows, o.errors(rows))
            torch.cuda.synchronize()
            active = sum(t.mark(adaptive.min_samples, adaptive.threshold) for t in ts)
        rounds.append((target, active))
        if active == 0:
            break
    assert rounds == [(x.samples, x.active) for x in want.rounds]
    got = np.zeros_like(want_accum)
    for t in ts:
        got[t.rows()] = t.trace.read_accum()[t.rows()]
    assert np.array_equal(got.view(np.uint32), want_accum.view(np.uint32))
