"""Checkpoints and projections through the C ABI on the GPU.

* pfxt_save / pfxt_restore round-trip the accumulation and films; a render
  saved, restored into a new tracer and continued equals the uninterrupted one
  bit for bit (Trace::save/restore, checkpoint.rs:161-203).
* A checkpoint written byte by byte in the reference's layout restores those
  exact bytes; one of another size is refused with the reference's message.
* Trace::set_projection (gpu.rs:2872) gives the image of a tracer created with
  that projection.
* Trace::sample_adaptive_kept with a keeper: checkpoints with the adaptive
  rounds and snapshots, and a render resumed from one ends as the
  uninterrupted render does."""
import dataclasses

import numpy as np
import pytest

from pfx_b200 import abi, synth
from pfx_b200.trace import Adaptive, Trace, TraceError
from test_checkpoint import info as checkpoint_info
from test_checkpoint import write_to

pytestmark = pytest.mark.gpu


def small():
    return synth.small("room_4k", (40, 24), sampler="sobol")


def test_resume_from_a_checkpoint_equals_the_uninterrupted_render(gpu):
    w = small()
    whole = Trace(w.scene, w.settings, w.width, w.height)
    whole.sample(2, 1)
    whole.sample(2, 2)
    first = Trace(w.scene, w.settings, w.width, w.height)
    first.sample(2, 1)
    data = first.save("still 1")
    resumed = Trace(w.scene, w.settings, w.width, w.height)
    resumed.restore("still 1", data)
    assert resumed.samples() == 2
    assert np.array_equal(resumed.read_accum(), first.read_accum())
    assert np.array_equal(resumed.readback().color, first.readback().color)
    resumed.sample(2, 2)
    assert np.array_equal(resumed.read_accum(), whole.read_accum())
    with pytest.raises(TraceError, match="another render"):
        resumed.restore("still 2", data)


def test_restore_takes_the_reference_layout_byte_for_byte(gpu):
    w = small()
    t = Trace(w.scene, w.settings, w.width, w.height)
    data = write_to("k", size=(w.width, w.height), samples=7, adaptive=True)
    t.restore("k", data)
    assert t.samples() == 7
    pixels = w.width * w.height
    head = 8 + 8 + 1 + 12
    accum = np.frombuffer(data[head:head + 48 * pixels], np.float32).reshape(w.height, w.width, 12)
    assert np.array_equal(t.read_accum().view(np.uint32), accum.view(np.uint32))
    color = np.frombuffer(data[head + 48 * pixels:head + 64 * pixels], np.float32).reshape(w.height, w.width, 4)
    assert np.array_equal(t.readback().color.view(np.uint32), color.view(np.uint32))
    # a save writes the same layout back (without the adaptive part)
    again = t.save("k")
    assert again[:head + 96 * pixels] == data[:head + 96 * pixels] and again[-4:] == b"\xff\xff\xff\xff"
    with pytest.raises(TraceError, match="the checkpoint is 3x2 and the trace"):
        t.restore("k", write_to("k"))


def test_set_projection_matches_a_tracer_made_with_it(gpu):
    w = small()
    ortho = dataclasses.replace(w.settings, projection=abi.PROJECTION_ORTHOGRAPHIC, ortho=(8.0, 4.8))
    made = Trace(w.scene, ortho, w.width, w.height)
    moved = Trace(w.scene, w.settings, w.width, w.height)
    moved.sample(1, 5)
    moved.set_projection("orthographic", 8.0, 4.8)
    assert moved.samples() == 0
    for t in (made, moved):
        t.sample(2, 3)
    assert np.array_equal(made.read_accum(), moved.read_accum())
    with pytest.raises(TraceError, match="invalid projection"):
        moved.set_projection("orthographic", 0.0, 1.0)


class ListKeeper:
    """A Keeper (checkpoint.rs:30-34) that keeps every checkpoint in a list."""

    def __init__(self, every: int, resume: bytes | None = None):
        self.every, self._resume, self.kept = every, resume, []

    def resume(self):
        return self._resume

    def due(self, samples: int) -> bool:
        return samples % self.every == 0

    def keep(self, data: bytes) -> None:
        self.kept.append(data)


def rounds_of(converged):
    return [(r.samples, r.active) for r in converged.rounds]


def test_kept_adaptive_render_resumes_to_the_same_image(gpu):
    """sample_adaptive_kept (adaptive.rs:136-325): checkpoints taken every few
    samples change nothing, and a fresh tracer resumed from one of them ends
    with the same rounds and the same accumulation as the uninterrupted render."""
    w = small()
    a = Adaptive(threshold=0.05, min_samples=4, max_samples=24, growth=1.5)
    plain = Trace(w.scene, w.settings, w.width, w.height)
    whole = plain.sample_adaptive(a, 9)
    kept = Trace(w.scene, w.settings, w.width, w.height)
    keeper = ListKeeper(4)
    assert rounds_of(kept.sample_adaptive_kept(a, 9, "still 1", keeper)) == rounds_of(whole)
    assert np.array_equal(kept.read_accum(), plain.read_accum())
    assert len(keeper.kept) >= 2
    mid = keeper.kept[1]
    rc, _, info = checkpoint_info("still 1", mid)
    assert rc == abi.OK and info.samples == 8 and info.rounds != 0xFFFFFFFF
    resumed = Trace(w.scene, w.settings, w.width, w.height)
    back = resumed.sample_adaptive_kept(a, 9, "still 1", ListKeeper(1000, resume=mid))
    assert rounds_of(back) == rounds_of(whole)
    assert np.array_equal(resumed.read_accum(), plain.read_accum())
    with pytest.raises(TraceError, match="no adaptive rounds"):
        Trace(w.scene, w.settings, w.width, w.height).sample_adaptive_kept(
            a, 9, "still 1", ListKeeper(1000, resume=plain.save("still 1")))
    with pytest.raises(TraceError, match="another render"):
        Trace(w.scene, w.settings, w.width, w.height).sample_adaptive_kept(
            a, 9, "still 2", ListKeeper(1000, resume=mid))
