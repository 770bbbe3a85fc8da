"""One frame split into bands (pfx_b200.shard) on one GPU: the bands, each
traced by its own tracer through Trace::set_window (gpu.rs:2836), are the rows
of the whole frame's render bit for bit, so ranks that each trace one band and
gather them render the frame the whole tracer renders."""
import numpy as np
import pytest

from pfx_b200 import shard, synth
from pfx_b200.trace import Trace

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
