"""Moving instances of a live tracer on the GPU (Trace::set_instance_transforms,
crates/trace/src/gpu.rs:2422-2546), on the stage of the reference's own
crates/trace/tests/instances.rs:

* moved_instances_trace_as_a_fresh_stage (instances.rs:214-254): a tracer
  whose instances moved renders the image of a tracer built with the moved
  transforms, bit for bit; the bottom levels are kept and one more top is laid.
* a_camera_move_keeps_the_trace_and_builds_nothing (instances.rs:256-273):
  the same transforms move nothing and keep the accumulation; a prefix moves;
  more transforms than instances is an error.
* With the radiance cache attached, a move keeps the cache working."""
import numpy as np
import pytest

from pfx_b200 import synth
from pfx_b200.cache import CacheSettings, RadianceCache
from pfx_b200.trace import Trace, TraceError

pytestmark = pytest.mark.gpu


def staged(moved, **kw):
    w = synth.staged(synth.staged_poses(moved), **kw)
    return Trace(w.scene, w.settings, w.width, w.height)


def traced(trace):
    trace.sample(8, 11)
    return trace.readback().color


@pytest.mark.parametrize("world, empty, route", [(False, False, "trace"), (True, True, "trace"),
                                                 (True, False, "buffers")])
def test_moved_instances_trace_as_a_fresh_stage(gpu, world, empty, route):
    kept = staged(False, world=world, empty=empty)
    before = traced(kept)
    if route == "trace":
        assert kept.set_instance_transforms(synth.staged_poses(True))
    else:  # a host that moves its own buffers, then uploads them
        assert kept.scene_buffers.move_instances(synth.staged_poses(True))
        kept.finish_tops()
    assert kept.samples() == 0
    moved = traced(kept)
    fresh = staged(True, world=world, empty=empty)
    expected = traced(fresh)
    assert not np.array_equal(before, moved), "the move changed nothing"
    assert np.array_equal(moved.view(np.uint32), expected.view(np.uint32))
    assert np.array_equal(kept.read_accum(), fresh.read_accum())
    assert kept.builds() == (3 + int(world), 2) and fresh.builds() == (3 + int(world), 1)


def test_a_camera_move_keeps_the_trace(gpu):
    trace = staged(False)
    assert trace.builds() == (3, 1)
    first = traced(trace)
    trace.set_camera(synth.look_at((1.5, 2.0, 4.0), (0.0, 0.4, 0.0), 53.13010235415598, 96 / 64))
    turned = traced(trace)
    assert not np.array_equal(first, turned)
    assert trace.builds() == (3, 1)
    trace.sample(2, 12)
    assert not trace.set_instance_transforms(synth.staged_poses(False))
    assert trace.samples() == 10 and trace.builds() == (3, 1)
    assert trace.set_instance_transforms(synth.staged_poses(True)[:2])
    assert trace.samples() == 0 and trace.builds() == (3, 2)
    with pytest.raises(TraceError, match="4 instances and 5 transforms"):
        trace.set_instance_transforms([synth.IDENTITY] * 5)
    # the tracer still samples after the refused call
    assert np.isfinite(traced(trace)).all()


def test_a_move_under_the_radiance_cache(gpu):
    trace = staged(False)
    cache = RadianceCache(CacheSettings(log2_entries=14, base_resolution=8, max_resolution=512, batch=256, steps=2,
                                        train_fraction=0.5, error_bound=1e30))
    trace.set_cache(cache)
    for seed in range(4):
        trace.sample(1, seed)
    assert trace.set_instance_transforms(synth.staged_poses(True))
    for seed in range(4):
        trace.sample(1, 10 + seed)
    assert trace.samples() == 4
    assert np.isfinite(trace.readback().color).all()
    assert cache.stats()["steps"] >= 8


def test_the_reference_stage_moves_like_a_fresh_stage(gpu):
    """moved_instances_trace_as_a_fresh_stage (instances.rs:214-254) on the
    reference's own stage built with pfx_b200.stage (indexed meshes, one ball
    mesh placed with two materials), 96 x 64, 8 samples with seed 11."""
    from test_stage import staged as reference_stage
    kept = reference_stage(synth.staged_poses(False)).trace(96, 64)
    before = traced(kept)
    assert kept.set_instance_transforms(synth.staged_poses(True))
    moved = traced(kept)
    expected = traced(reference_stage(synth.staged_poses(True)).trace(96, 64))
    assert not np.array_equal(before, moved)
    assert np.array_equal(moved.view(np.uint32), expected.view(np.uint32))
    assert kept.builds() == (3, 2)
