"""Moving instances on the host buffers (Trace::move_instances,
crates/trace/src/gpu.rs:2433-2530; Levels::top, levels.rs:426-470), on the
stage of the reference's own test crates/trace/tests/instances.rs.

Moving every instance of a built scene to new transforms leaves the buffers
bit for bit equal to a scene built with those transforms; moving nothing
changes nothing; a partial list moves only its prefix; the reference's error
cases keep their messages."""
import dataclasses

import numpy as np
import pytest

from pfx_b200 import synth
from pfx_b200.trace import SceneBuffers, TraceError

MOVED = ["nodes", "surfaces", "emitters", "emitter_cdf"]
KEPT = ["triangles", "uv", "materials", "lights"]


def built(poses, **kw):
    w = synth.staged(poses, **kw)
    return SceneBuffers(w.scene, w.settings)


def arrays(b):
    return {n: b.array(n) for n in MOVED + KEPT}


@pytest.mark.parametrize("world, empty", [(False, False), (True, True)])
def test_moved_buffers_equal_a_fresh_build(world, empty):
    kept = built(synth.staged_poses(False), world=world, empty=empty)
    fresh = built(synth.staged_poses(True), world=world, empty=empty)
    before = arrays(kept)
    # the emissive panel moves too, so its emitter rows change with the nodes
    assert all(not np.array_equal(before[n], fresh.array(n)) for n in MOVED)
    assert kept.builds() == fresh.builds() == (3 + int(world), 1)
    assert kept.move_instances(synth.staged_poses(True))
    after = arrays(kept)
    for n in MOVED + KEPT:
        assert np.array_equal(after[n], fresh.array(n)), n
    # Trace::builds: the bottom levels are kept, one more top (instances.rs:245-246)
    assert kept.builds() == (3 + int(world), 2)


def test_the_same_transforms_move_nothing():
    kept = built(synth.staged_poses(False), empty=True)
    before = arrays(kept)
    assert not kept.move_instances(synth.staged_poses(False))
    assert not kept.move_instances([])
    # an empty mesh's instance is never placed, so its transform is ignored
    assert not kept.move_instances(synth.staged_poses(False) + [synth.placed((5, 5, 5), 1.0, 2.0)])
    after = arrays(kept)
    assert all(np.array_equal(before[n], after[n]) for n in before)
    assert kept.builds() == (3, 1)


def test_a_prefix_moves_only_its_instances():
    """set_instance_transforms(&pose(true)[..2]) (instances.rs:267-270)."""
    kept = built(synth.staged_poses(False))
    mixed = synth.staged_poses(True)[:2] + synth.staged_poses(False)[2:]
    fresh = built(mixed)
    assert kept.move_instances(synth.staged_poses(True)[:2])
    for n in MOVED:
        assert np.array_equal(kept.array(n), fresh.array(n)), n
    assert kept.builds() == (3, 2)


def test_reference_errors():
    kept = built(synth.staged_poses(False))
    with pytest.raises(TraceError, match="the trace has 4 instances and 5 transforms were given"):
        kept.move_instances([synth.IDENTITY] * 5)
    bad = synth.staged_poses(True)
    bad[3] = bad[3].copy()
    bad[3][3, 0] = np.inf
    before = arrays(kept)
    with pytest.raises(TraceError, match="instance transform is not finite"):
        kept.move_instances(bad)
    # nothing moved on an error, even the instances before the bad transform
    assert all(np.array_equal(before[n], kept.array(n)) for n in before)
    plain = synth.small("plain_512", (16, 16))
    lone = SceneBuffers(plain.scene, plain.settings)
    assert not lone.move_instances([])
    with pytest.raises(TraceError, match="this trace has no instances to move"):
        lone.move_instances([synth.IDENTITY])


@pytest.mark.parametrize("seed", [1, 2])
def test_many_random_moves_equal_fresh_builds(seed):
    """The instanced workload (boxes and icospheres from 8 clusters): moving
    every instance to a random pose gives a fresh build's buffers, bit for bit."""
    rng = np.random.default_rng(seed)
    w = synth.instanced_1080(target=20_000)
    n = len(w.scene.instances)
    poses = np.stack([synth.transform_matrix(float(rng.uniform(0.2, 5.0)), synth.random_rotation(rng),
                                             rng.uniform(-60, 60, 3)) for _ in range(n)])
    kept = SceneBuffers(w.scene, w.settings)
    assert kept.move_instances(poses)
    moved = w.scene.instances.copy()
    moved["transform"] = poses
    fresh_scene = dataclasses.replace(w.scene, instances=moved)
    fresh = SceneBuffers(fresh_scene, w.settings)
    for name in MOVED + KEPT:
        assert np.array_equal(kept.array(name), fresh.array(name)), name
    assert kept.builds() == (fresh.builds()[0], 2)


def test_a_move_keeps_the_emitter_list_a_fresh_build_would_shrink():
    """move_instances rewrites the vertices of the emitter candidates it built
    with and keeps the list (gpu.rs:2484-2499): an emissive panel shrunk below
    the 1e-12 area cutoff stays an emitter, where a fresh build would drop it."""
    kept = built(synth.staged_poses(False))
    count = kept.buffers.emitter_count
    poses = synth.staged_poses(False)
    poses[3] = synth.placed((0.0, 1.8, -0.8), 0.0, 1e-7)
    assert kept.move_instances(poses)
    assert kept.buffers.emitter_count == count
    assert np.frombuffer(kept.array("emitters")[:4].tobytes(), np.float32)[0] == count  # the header's count
    assert built(poses).buffers.emitter_count < count


def test_pose_checks_of_the_reference():
    """a_tiny_scaled_instance_keeps_its_normals_and_only_a_flat_one_is_refused
    (detail.rs:653-688) and Pose::new's refusals (detail.rs:190-221), through
    moving an instance of the stage: tiny rotations and scales are accepted,
    flat, zero, non-affine and non-finite transforms are refused."""
    kept = built(synth.staged_poses(False))
    for s in (1e-2, 1e-4, 1e-6):
        m = np.array([[s, 0, 0, 0], [0, 0, s, 0], [0, -s, 0, 0], [0, 0, 0, 1]], np.float32)
        assert kept.move_instances([synth.IDENTITY, m])
    flat = np.array([[1, 0, 0, 0], [1, 1e-9, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], np.float32)
    zero = flat.copy()
    zero[1] = 0.0
    skew = synth.IDENTITY.copy()
    skew[0, 3] = 0.5
    bad = synth.IDENTITY.copy()
    bad[3, 0] = np.nan
    for m, message in ((flat, "singular"), (zero, "singular"), (skew, "not affine"), (bad, "not finite")):
        with pytest.raises(TraceError, match=message):
            kept.move_instances([synth.IDENTITY, m])


def test_instance_records_transform_positions_and_normals():
    """transforms_instance_positions_and_normals (detail.rs:692-717) read from the
    instance's surface record: its forward rows take the origin to (3, 4, 5) and
    its inverse rows take the normal (1, 1, 0) to x = 0.4472136 once normalised."""
    from pfx_b200.trace import INSTANCE, TRIANGLE, Camera, SceneDesc, Settings
    tri = np.zeros(1, TRIANGLE)
    tri["v"] = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]  # a non-empty triangle; vertex 0 at the origin
    tri["n"] = [[1, 1, 0]] * 3
    inst = np.zeros(1, INSTANCE)
    inst["transform"] = np.array([[2, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [3, 4, 5, 1]], np.float32).reshape(16)
    inst["two_sided"], inst["casts_shadow"] = 1, 1
    cam = Camera((0.0, 0.0, 5.0), (0.0, 0.0, -1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    sb = SceneBuffers(SceneDesc(np.zeros(0, TRIANGLE), synth.material(), cam, meshes=[tri], instances=inst),
                      Settings())
    rec = sb.array("surfaces").view(np.float32).reshape(-1, 44)[1]
    forward, inverse = rec[20:32].reshape(3, 4), rec[32:44].reshape(3, 4)
    assert np.array_equal(forward @ np.array([0, 0, 0, 1], np.float32), [3.0, 4.0, 5.0])
    n = inverse[:, :3].T.astype(np.float64) @ np.array([1.0, 1.0, 0.0])
    assert abs(n[0] / np.linalg.norm(n) - 0.4472136) < 1e-6
