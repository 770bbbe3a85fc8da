"""Traversal kernels against the oracle on identical ray batches: hit slot,
record and distance bit for bit (closest hit), blocked flag and first blocker
(any hit), and the same number of box and triangle tests per ray."""
import numpy as np
import pytest

import oracle
from pfx_b200 import rays as raymix
from pfx_b200 import synth
from pfx_b200.trace import SceneDesc, Settings, Trace, make_rays

pytestmark = pytest.mark.gpu


def compare_closest(trace, batch, ref):
    """`ref`: the oracle's own buffers of the traced scene (oracle.scene_buffers)."""
    got = trace.trace_rays(batch)
    want, counts, overflow = oracle.trace(ref, batch, any_hit=False, counts=True)
    assert overflow == 0
    assert np.array_equal(got["hit"], want["hit"])
    h = want["hit"] == 1
    assert np.array_equal(got["slot"][h], want["slot"][h])
    assert np.array_equal(got["record"][h], want["record"][h])
    assert np.array_equal(got["t"].view(np.uint32), want["t"].view(np.uint32))
    return got, counts


def compare_any(trace, batch, ref):
    got = trace.occluded(batch)
    want = oracle.trace(ref, batch, any_hit=True)
    assert np.array_equal(got, want["hit"] == 1)
    return got


def device_counts(trace, batch, any_hit):
    import torch
    r = torch.from_numpy(batch.view(np.uint8).copy()).cuda()
    c = torch.zeros(len(batch) * 2, dtype=torch.int32, device="cuda")
    trace.counts_device(r.data_ptr(), len(batch), any_hit, c.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return c.cpu().numpy().view(np.uint32).reshape(-1, 2)


def test_lcg_fixture(gpu):
    verts, rays = synth.lcg_triangles()
    tris = synth.triangles(verts)
    scene = SceneDesc(tris, synth.material(), synth.look_at((0, 0, 10), (0, 0, 0), 45, 1.0))
    trace = Trace(scene, Settings(), 8, 8)
    ref = oracle.scene_buffers(scene, Settings())
    batch = make_rays(np.array([o for o, _ in rays], np.float32), np.array([d for _, d in rays], np.float32), 1e20)
    got, _ = compare_closest(trace, batch, ref)
    assert got["hit"].sum() > 50
    compare_any(trace, make_rays(batch["origin"], batch["direction"], 3.0), ref)


@pytest.mark.parametrize("name", ["plain_512", "instanced_1080"])
def test_pass_mix(gpu, name):
    w = synth.WORKLOADS[name](**({"target": 40_000} if name == "instanced_1080" else {}))
    trace = Trace(w.scene, w.settings, w.width, w.height)
    ref = oracle.scene_buffers(w.scene, w.settings)
    closest, shadow = raymix.pass_mix(trace, w.scene, w.width, w.height, 1 << 16, seed=3)
    got, counts = compare_closest(trace, closest, ref)
    assert got["hit"].mean() > 0.2
    blocked = compare_any(trace, shadow, ref)
    assert 0.02 < blocked.mean() < 0.98
    # the kernel does exactly the reference's box and triangle tests
    assert np.array_equal(device_counts(trace, closest, False), counts)
    _, scounts, _ = oracle.trace(ref, shadow, any_hit=True, counts=True)
    assert np.array_equal(device_counts(trace, shadow, True), scounts)


def test_random_rays_inside_the_sphere_cloud(gpu):
    w = synth.plain_512()
    trace = Trace(w.scene, w.settings, 64, 64)
    ref = oracle.scene_buffers(w.scene, w.settings)
    rng = np.random.default_rng(11)
    batch = synth.random_rays((-12, 0.01, -12), (12, 21, 12), 50_000, rng)
    compare_closest(trace, batch, ref)
    limited = batch.copy()
    limited["tmax"] = rng.uniform(0.01, 8.0, len(batch)).astype(np.float32)
    compare_closest(trace, limited, ref)
    compare_any(trace, limited, ref)


def test_empty_and_degenerate_batches(gpu):
    w = synth.plain_512()
    trace = Trace(w.scene, w.settings, 16, 16)
    ref = oracle.scene_buffers(w.scene, w.settings)
    assert len(trace.trace_rays(np.zeros(0, dtype=make_rays(np.zeros((1, 3)), np.zeros((1, 3)), 1).dtype))) == 0
    # axis-aligned directions exercise the degenerate-slab branch (|d| < 1e-12)
    o = np.array([[0, 5, 30], [3, 25, 0], [0.5, 0.5, -30], [-30, 1, 0.25]], np.float32)
    d = np.array([[0, 0, -1], [0, -1, 0], [0, 0, 1], [1, 0, 0]], np.float32)
    compare_closest(trace, make_rays(o, d, 1e20), ref)
    compare_any(trace, make_rays(o, d, 1e20), ref)


@pytest.mark.parametrize("scale", [1e-3, 40.0, 1e6, 1e7])
def test_unnormalised_directions(gpu, scale):
    """Direction components above 2^20, origins beyond 2^79 or tiny nonzero
    origin components make a ray unbounded: it is walked again with IEEE
    division.  Bounded rays use the unchecked Markstein quotients.  Both equal
    the oracle's divisions bit for bit."""
    w = synth.plain_512()
    trace = Trace(w.scene, w.settings, 64, 64)
    ref = oracle.scene_buffers(w.scene, w.settings)
    rng = np.random.default_rng(12)
    batch = synth.random_rays((-12, 0.01, -12), (12, 21, 12), 20_000, rng)
    batch["direction"] = batch["direction"] * np.float32(scale)
    compare_closest(trace, batch, ref)
    compare_any(trace, make_rays(batch["origin"], batch["direction"], 2.0 / scale), ref)
    far = batch[:64].copy()
    far["origin"] = far["origin"] + np.float32(1e24)
    compare_closest(trace, far, ref)
    tiny = batch[:256].copy()  # an origin component below 2^-70 (but not 0)
    tiny["origin"][:, 0] = np.float32(1e-25)
    compare_closest(trace, tiny, ref)
