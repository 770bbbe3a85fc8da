"""The clip workload's host side: the camera spline and the shots."""
import numpy as np

from pfx_b200 import clip


def test_catmull_rom_passes_through_its_keys_smoothly():
    rng = np.random.default_rng(3)
    keys = rng.uniform(-5, 5, (8, 3))
    for k in range(8):
        assert np.allclose(clip.catmull_rom(keys, k / 7), keys[k], atol=1e-12)
    eps = 1e-7
    for k in range(1, 7):  # continuous position and tangent at the inner keys
        t = k / 7
        left = (clip.catmull_rom(keys, t) - clip.catmull_rom(keys, t - eps)) / eps
        right = (clip.catmull_rom(keys, t + eps) - clip.catmull_rom(keys, t)) / eps
        assert np.allclose(left, right, rtol=1e-4, atol=1e-4)


def test_shots_split_the_clip_and_cameras_are_orthogonal():
    shots = clip.clip_shots(frames=10, size=(64, 36), scene_triangles=(2000, 3000, 4000))
    assert [s.frames for s in shots] == [4, 3, 3]
    assert [s.first_frame for s in shots] == [0, 4, 7]
    for s in shots:
        for f in range(s.frames):
            c = clip.camera_at(s, f)
            fwd, right, up = (np.asarray(v) for v in (c.forward, c.right, c.up))
            assert abs(np.linalg.norm(fwd) - 1.0) < 1e-6
            assert abs(fwd @ right) < 1e-6 and abs(fwd @ up) < 1e-6
            assert np.all(np.abs(c.origin) < 15.0)  # inside the 30 m room


def test_room_sizes_follow_their_targets():
    for tris in (10_000, 100_000):
        s = clip.room_shot(tris, seed=5, size=(64, 36), frames=2)
        n = s.workload.scene.world_triangle_count
        assert 0.8 * tris <= n <= 1.2 * tris, n
