"""Parity on the full-size workloads the bench measures, not reduced copies:
the 4K room (1.19 M triangles, 300 meshes, 128 lights through the light tree)
and the instanced scene at its full 200 k triangles.

  * traversal on 2^18-ray batches with the mix of one pass (camera, bounce and
    shadow rays): hit flag, slot, record and distance bit for bit against the
    oracle's walk, the same box and triangle tests per ray, and the any-hit
    flags (trace.wgsl:999-1168);
  * images of a window of the full 4K frame (Trace::set_window keeps the
    full-frame pixel coordinates, so the window's samples are the full
    frame's): accumulation and films within 1e-4 relative, PCG and Sobol."""
import numpy as np
import pytest

import oracle
from pfx_b200 import rays as raymix
from pfx_b200 import synth
from pfx_b200.trace import Settings, Trace

from test_gpu_render import render_both
from test_gpu_traverse import compare_any, compare_closest, device_counts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def room():
    return synth.room_4k()


@pytest.mark.parametrize("name", ["room_4k", "instanced_1080"])
def test_traversal_on_the_full_scene(gpu, room, name):
    w = room if name == "room_4k" else synth.instanced_1080()
    assert w.scene.world_triangle_count > (1_000_000 if name == "room_4k" else 200_000)
    trace = Trace(w.scene, w.settings, 64, 36)
    ref = oracle.scene_buffers(w.scene, w.settings)
    closest, shadow = raymix.pass_mix(trace, w.scene, w.width, w.height, 1 << 18, seed=17)
    got, counts = compare_closest(trace, closest, ref)
    assert got["hit"].mean() > 0.5
    hit = got["hit"] == 1
    if len(w.scene.instances):
        # slots of instanced meshes are indices into the shared mesh's triangles:
        # hits spread over many placed records instead
        assert len(np.unique(got["record"][hit])) > 100
    else:
        assert int(got["slot"][hit].max()) > w.scene.world_triangle_count // 2
    blocked = compare_any(trace, shadow, ref)
    assert 0.02 < blocked.mean() < 0.98
    assert np.array_equal(device_counts(trace, closest, False), counts)
    _, scounts, overflow = oracle.trace(ref, shadow, any_hit=True, counts=True)
    assert overflow == 0
    assert np.array_equal(device_counts(trace, shadow, True), scounts)
    # deep walks: the batch reaches far into the traversal stack
    assert counts[:, 0].max() > 200
    trace.close()


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_image_of_a_window_of_the_full_4k_room(gpu, room, sampler):
    w = synth.Workload(room.name, room.scene, Settings.deep(8, sampler=sampler, sobol_samples=64,
                                                            filter_glossy=0.25, clamp_indirect=4.0), 96, 54)
    # a window below the frame's centre: shelves, glass and metal spheres
    got, exact = render_both(w, 2, [31, 32], window=((3840, 2160), (1700, 1300)))
    assert got[..., :3].mean() > 0.0
    assert exact > 0.99


@pytest.mark.parametrize("name", ["room_4k", "instanced_1080", "clip_1m"])
def test_gpu_bvh_build_equals_the_host_build(gpu, room, name):
    """The binned-SAH build on the GPU (bvh_gpu.cu) gives the host build's and
    the oracle's nodes and triangle order byte for byte (bvh.rs:95-266), and
    the whole packed scene is unchanged."""
    import time

    from pfx_b200 import abi, clip
    from pfx_b200.trace import SceneBuffers
    if name == "room_4k":
        w = room
    elif name == "instanced_1080":
        w = synth.instanced_1080()
    else:
        w = clip.room_shot(1_000_000, 9).workload
    lib = abi.load()
    t0 = time.perf_counter()
    gpu = SceneBuffers(w.scene, w.settings)
    gpu_s = time.perf_counter() - t0
    lib.pfxt_debug_gpu_bvh(0)
    try:
        t0 = time.perf_counter()
        host = SceneBuffers(w.scene, w.settings)
        host_s = time.perf_counter() - t0
    finally:
        lib.pfxt_debug_gpu_bvh(1)
    big = len(w.scene.triangles) >= (1 << 16)
    assert lib.pfxt_debug_scene_gpu_builds(gpu._h) == (1 if big else 0)
    assert lib.pfxt_debug_scene_gpu_builds(host._h) == 0
    for blob in ("nodes", "triangles", "uv", "surfaces", "emitters", "lights"):
        assert np.array_equal(gpu.array(blob), host.array(blob)), blob
    assert np.array_equal(gpu.order(), host.order())
    if big:
        nodes, order = oracle.bvh_build(w.scene.triangles["v"])
        if not len(w.scene.instances):
            assert np.array_equal(gpu.array("nodes"), nodes)
        assert np.array_equal(gpu.order(), order)
        print(f"{name}: scene build {gpu_s:.2f} s with the GPU BVH, {host_s:.2f} s on the host")
