"""The clip workload on the GPU (pfx_b200.clip).

* Every frame of a clip equals a still rendered by a fresh tracer with that
  frame's camera and seed, bit for bit: moving the camera restarts the
  accumulation and nothing of the previous frame leaks into the next.
* A shot replays one CUDA graph for all its frames (the camera travels in the
  pass variables, not in the captured launch parameters).
* With a radiance cache per shot, the frames stay finite and the cache trains
  across the shot's frames."""
import numpy as np
import pytest

from pfx_b200 import clip
from pfx_b200.cache import CacheSettings
from pfx_b200.trace import Trace

pytestmark = pytest.mark.gpu


def small_shots():
    return clip.clip_shots(frames=6, size=(64, 36), scene_triangles=(3000, 6000), sampler="pcg")


def test_clip_frames_equal_fresh_stills(gpu):
    shots = small_shots()
    frames = {}
    res = clip.render(shots, spp=2, on_frame=lambda i, t: frames.__setitem__(i, t.read_accum()), timed=False)
    assert sorted(frames) == list(range(6))
    assert [r.graph_captures for r in res] == [1, 1]
    for shot in shots:
        w = shot.workload
        for f in range(shot.frames):
            i = shot.first_frame + f
            still = Trace(w.scene, w.settings, w.width, w.height)
            still.set_camera(clip.camera_at(shot, f))
            still.sample(2, i)
            assert np.array_equal(still.read_accum().view(np.uint32), frames[i].view(np.uint32)), i
    # consecutive frames see different views
    assert not np.array_equal(frames[0], frames[1])


def test_clip_with_a_cache_per_shot(gpu):
    shots = small_shots()
    settings = CacheSettings(log2_entries=14, base_resolution=8, max_resolution=512, batch=256, steps=2,
                             train_fraction=0.5, error_bound=1e30)
    colours = []
    res = clip.render(shots, spp=2, cache_settings=settings,
                      on_frame=lambda i, t: colours.append(t.readback().color))
    assert len(colours) == 6 and all(np.isfinite(c).all() for c in colours)
    assert [r.graph_captures for r in res] == [1, 1]
    assert all(r.device_s > 0.0 and r.rays > 0 for r in res)
