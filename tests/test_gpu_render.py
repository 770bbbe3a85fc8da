"""The wavefront tracer against the oracle's restatement of main()/radiance():
with the reference's random sequence reproduced (PCG and Sobol), every pixel of
the accumulation and of the films must match within 1e-4 relative in FP32 (the
tolerance of the parity contract); in practice the images are bit-identical.
The oracle renders from its own packing of the scene (oracle.scene_buffers),
never from the buffers the product built.
Also the reference's furnace and determinism pins, and adaptive sampling
rounds against the oracle."""
import numpy as np
import pytest

import oracle
from pfx_b200 import synth
from pfx_b200.trace import Adaptive, Settings, Trace

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-4, 1e-6


def assert_close(got, want, what):
    bad = ~np.isclose(got, want, rtol=RTOL, atol=ATOL)
    assert not bad.any(), f"{what}: {bad.sum()} of {bad.size} values differ, e.g. {got[bad][:4]} vs {want[bad][:4]}"
    return float(np.mean(got.view(np.uint32) == want.view(np.uint32)))


def render_both(w, spp, seeds, window=None):
    """Trace::sample passes of `w` on the GPU and in the oracle; `window` =
    ((full width, full height), (x, y)) renders that tile of a larger frame."""
    trace = Trace(w.scene, w.settings, w.width, w.height)
    r = oracle.Renderer(oracle.scene_buffers(w.scene, w.settings), w.settings)
    if window is not None:
        trace.set_window(*window)
    frame = trace.frame()
    accum = np.zeros((w.height, w.width, 12), np.float32)
    samples = 0
    films = None
    for seed in seeds:
        trace.sample(spp, seed)
        films = r.render(frame, accum, samples, spp, seed)
        samples += spp
    got = trace.read_accum()
    out = trace.readback()
    exact = assert_close(got, accum, "accumulation")
    assert_close(out.color, films[0], "colour film")
    assert_close(out.albedo, films[1], "albedo film")
    assert_close(out.normal, films[2], "normal film")
    assert np.isfinite(got).all()
    assert trace.samples() == samples
    return got, exact


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_sphere_cloud_with_rect_lights(gpu, sampler):
    w = synth.small("plain_512", (48, 40), sampler=sampler)
    w.settings = Settings.deep(4, sampler=sampler, sobol_samples=16)
    got, exact = render_both(w, 4, [0, 1])
    assert got[..., :3].mean() > 0.0
    assert exact > 0.99


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_instances_and_light_tree(gpu, sampler):
    w = synth.small("instanced_1080", (48, 32), sampler=sampler)
    w.settings = Settings.deep(8, sampler=sampler, sobol_samples=64)
    got, exact = render_both(w, 4, [3])
    assert got[..., :3].mean() > 0.0
    assert exact > 0.99


def test_room_with_glass_and_metals(gpu):
    w = synth.small("room_4k", (48, 32), sampler="sobol")
    w.settings = Settings.deep(8, sampler="sobol", sobol_samples=64)
    got, exact = render_both(w, 4, [9])
    assert exact > 0.99


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_firefly_controls(gpu, sampler):
    # CLAMP_INDIRECT and FILTER_GLOSSY (trace.wgsl:1872-1875, 2377-2379)
    w = synth.small("room_4k", (40, 24), sampler=sampler)
    w.settings = Settings.deep(8, sampler=sampler, sobol_samples=64, filter_glossy=0.25, clamp_indirect=2.0)
    got, exact = render_both(w, 4, [21])
    assert exact > 0.99


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_masked_pixels_match_the_full_frame(gpu, sampler):
    # a pixel's samples depend on the pixel, the sample index and the seed only
    w = synth.small("room_4k", (64, 40), sampler=sampler)
    full = Trace(w.scene, w.settings, w.width, w.height)
    part = Trace(w.scene, w.settings, w.width, w.height)
    mask = np.zeros((w.height, w.width), bool)
    mask[3::5, 2::7] = True
    part.set_pixel_mask(mask)
    for seed in (5, 6, 7):
        full.sample(2, seed)
        part.sample(2, seed)
    a, b = full.read_accum(), part.read_accum()
    assert np.array_equal(a[mask], b[mask])
    assert not b[~mask].any()


def test_material_sort_keeps_the_image(gpu):
    # the shade queue's order is free: sorting it by material changes no value
    w = synth.small("room_4k", (64, 40), sampler="sobol")
    a = Trace(w.scene, w.settings, w.width, w.height)
    b = Trace(w.scene, w.settings, w.width, w.height)
    b._lib.pfxt_debug_sort(b.handle, 0)
    for seed in (3, 4):
        a.sample(2, seed)
        b.sample(2, seed)
    assert np.array_equal(a.read_accum(), b.read_accum())


@pytest.mark.parametrize("name", ["room_4k", "instanced_1080"])
def test_split_shade_matches_the_fused_kernel(gpu, name):
    w = synth.small(name, (64, 40), sampler="sobol")
    a = Trace(w.scene, w.settings, w.width, w.height)
    b = Trace(w.scene, w.settings, w.width, w.height)
    b.set_tuning(split_shade=False, sort_rays=True)
    for t in (a, b):
        t.sample(2, 7)
        t.sample(1, 8)
    assert np.array_equal(a.read_accum(), b.read_accum())


def test_graph_replay_matches_launches(gpu):
    # a captured pass replays with each pass's seed and sample offset
    w = synth.small("plain_512", (48, 40), sampler="sobol")
    w.settings = Settings.deep(4, sampler="sobol", sobol_samples=16)
    a = Trace(w.scene, w.settings, w.width, w.height)
    b = Trace(w.scene, w.settings, w.width, w.height)
    b._lib.pfxt_debug_graphs(b.handle, 0)
    for t in (a, b):
        for seed, count in ((1, 1), (2, 1), (3, 2), (4, 1)):
            t.sample(count, seed)
    assert np.array_equal(a.read_accum(), b.read_accum())
    assert a._lib.pfxt_debug_graph_captures(a.handle) == 2  # one graph per sample count
    cam = w.scene.camera
    moved = type(cam)(tuple(np.asarray(cam.origin) + 0.25), cam.forward, cam.right, cam.up)
    for t in (a, b):
        t.set_camera(moved)
        t.sample(1, 9)
        t.sample(1, 10)
    assert np.array_equal(a.read_accum(), b.read_accum())
    assert a.samples() == 2


def test_autotune_keeps_the_image(gpu):
    w = synth.small("room_4k", (64, 40), sampler="sobol")
    a = Trace(w.scene, w.settings, w.width, w.height)
    b = Trace(w.scene, w.settings, w.width, w.height)
    k = a.autotune(passes=2)
    assert k["trace_threads"] in (64, 128, 256) and k["pass_ms"] > 0 and k["short_stack"] in (0, 8)
    assert a.samples() == 0  # the trial passes are not part of the image
    images = []
    for threads, queue, short in ((64, True, 8), (256, False, 0), (128, False, 8)):
        b.set_tuning(trace_threads=threads, sort_shading=threads == 64, graphs=threads == 256, shadow_queue=queue,
                     short_stack=short)
        b.set_camera(w.scene.camera)
        b.sample(2, 5)
        images.append(b.read_accum())
    a.sample(2, 5)
    for img in images:  # block size, sorts, shadow queue and shared stack change no value
        assert np.array_equal(a.read_accum(), img)
    with pytest.raises(Exception):
        b.set_tuning(trace_threads=96)
    with pytest.raises(Exception):
        b.set_tuning(short_stack=4)
    # the same scene, film and settings again: the choice comes from the first tuning
    c = Trace(w.scene, w.settings, w.width, w.height)
    again = c.autotune(passes=2)
    assert again["from_cache"] and not k["from_cache"]
    assert {x: again[x] for x in ("trace_threads", "short_stack", "shadow_queue")} == \
        {x: k[x] for x in ("trace_threads", "short_stack", "shadow_queue")}
    other = Trace(w.scene, w.settings, w.width + 8, w.height)  # another film: tuned anew
    assert not other.autotune(passes=2)["from_cache"]


def test_furnace_and_determinism(gpu):
    # gpu.rs:3787-3830
    scene = synth.furnace()
    settings = Settings(sampler="pcg")
    a = Trace(scene, settings, 16, 16)
    b = Trace(scene, settings, 16, 16)
    for p in range(32):
        a.sample(4, 73 + p)
        b.sample(4, 73 + p)
    ca, cb = a.readback(), b.readback()
    assert np.array_equal(ca.color, cb.color) and np.array_equal(ca.normal, cb.normal)
    mid = ca.color[8, 8, :3]
    assert np.all(np.abs(mid - 1.0) < 0.12), mid


def test_adaptive_rounds_match_the_oracle(gpu):
    w = synth.small("instanced_1080", (40, 30), sampler="sobol")
    w.settings = Settings.deep(8, sampler="sobol", sobol_samples=64)
    adaptive = Adaptive(threshold=0.05, min_samples=8, max_samples=32, growth=1.5)
    trace = Trace(w.scene, w.settings, w.width, w.height)
    conv = trace.sample_adaptive(adaptive, 11)
    r = oracle.Renderer(oracle.scene_buffers(w.scene, w.settings), w.settings)
    rounds, accum, _ = r.sample_adaptive(trace.frame(), w.width, w.height, adaptive, 11)
    assert [(x.samples, x.active) for x in conv.rounds] == rounds
    got = trace.read_accum()
    assert_close(got, accum, "adaptive accumulation")
    counts = trace.sample_counts()
    assert counts.max() <= adaptive.max_samples and counts.min() >= 1
    assert 0 < conv.mean_samples() <= adaptive.max_samples


def test_paced_sampling_equals_one_call(gpu):
    """Trace::sample_paced (gpu.rs:2951): one pass per sample, `between` told
    each pass's device time; the image equals sample(count)'s bit for bit."""
    w = synth.small("plain_512", (48, 32), sampler="sobol")
    whole = Trace(w.scene, w.settings, w.width, w.height)
    whole.sample(3, 17)
    paced = Trace(w.scene, w.settings, w.width, w.height)
    seen = []
    stats = paced.sample_paced(3, 17, seen.append)
    assert len(seen) == 3 and stats.milliseconds == seen and all(m > 0.0 for m in seen)
    assert stats.wall_ms > 0.0 and paced.samples() == 3
    assert np.array_equal(paced.read_accum(), whole.read_accum())


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_emissive_instances_through_the_emitter_list(gpu, sampler):
    """An emissive panel placed as an instance, a dim sky and a sun
    (crates/trace/tests/instances.rs:159-197): emitter_candidate,
    find_emitter and emitter_weight (lights.wgsl:12-44, 103-144) against the
    oracle, with and without world triangles beside the instances."""
    for world in (False, True):
        w = synth.staged(synth.staged_poses(False), size=(48, 32), world=world)
        w.settings = Settings.deep(4, sampler=sampler, sobol_samples=16)
        got, exact = render_both(w, 4, [2, 3])
        assert got[..., :3].mean() > 0.0
        assert exact > 0.99


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_emissive_world_triangles_and_a_uniform_sky(gpu, sampler):
    """Emissive world triangles (two of the spheres glow) beside the rect
    lights, under a non-black uniform sky: the emitter CDF, the sky's CDF
    sampling and the miss MIS weight (sky.rs:441-480, trace.wgsl:2228-2236)."""
    w = synth.small("plain_512", (48, 40), sampler=sampler)
    mats = w.scene.materials.copy()
    mats["emission"][5] = (4.0, 3.0, 2.0)
    mats["emission"][9] = (0.5, 2.0, 6.0)
    w.scene.materials = mats
    w.scene.sky = (0.3, 0.4, 0.5)
    w.settings = Settings.deep(4, sampler=sampler, sobol_samples=16)
    trace = Trace(w.scene, w.settings, w.width, w.height)
    head = trace.scene_buffers.array("emitters").view(np.float32)[:4]
    assert head[0] > 100  # the glowing spheres' triangles are in the emitter list
    got, exact = render_both(w, 4, [4, 5])
    assert got[..., :3].mean() > 0.0
    assert exact > 0.99


@pytest.mark.parametrize("sampler", ["pcg", "sobol"])
def test_slot_kernels_equal_the_one_kernel_slots(gpu, sampler):
    """The light slots one kind per launch (k_tree_pick, k_light_slot) against
    every slot of a path in one kernel (k_shade_lights): a scene with every
    slot kind live (a soft sun, a uniform sky, emissive world triangles, three
    looped rect lights and a light tree over point and spot lights) gives the
    same accumulation bit for bit, and the same image as the oracle."""
    from pfx_b200.trace import Sun

    w = synth.small("plain_512", (48, 40), sampler=sampler)
    mats = w.scene.materials.copy()
    mats["emission"][5] = (4.0, 3.0, 2.0)
    w.scene.materials = mats
    w.scene.sky = (0.2, 0.25, 0.3)
    w.scene.sun = Sun((0.3, 1.0, 0.2), (1.0, 0.9, 0.8), 1.5, radius_deg=2.0)  # soft: two draws
    street = []
    for k in range(24):
        p = (-8.0 + (k % 6) * 3.2, 14.0 + (k % 3), -8.0 + (k // 6) * 5.0)
        if k % 3 == 0:
            street.append(synth.spot_light(p, (0.0, -1.0, 0.1), 30.0, 50.0, 30.0, (1.0, 0.8, 0.6), rng_range=30.0))
        else:
            street.append(synth.point_light(p, 20.0, (0.6, 0.8, 1.0), radius=0.2, rng_range=30.0))
    w.scene.lights = np.concatenate([w.scene.lights, *street])
    w.settings = Settings.deep(4, sampler=sampler, sobol_samples=16)
    images, kernels = [], []
    for slot_kernels in (True, False):
        t = Trace(w.scene, w.settings, w.width, w.height)
        t.set_tuning(trace_threads=128, sort_shading=False, slot_kernels=slot_kernels)
        for s in range(3):
            t.sample(1, 40 + s)
        images.append(t.read_accum())
        kernels.append(t.pass_kernels())
        t.close()
    assert images[0][..., :3].mean() > 0.0
    assert np.array_equal(images[0].view(np.uint32), images[1].view(np.uint32))
    # per bounce: sun, sky, emitters, three looped lights, the tree's descent and its
    # slot, against one kernel
    extra = kernels[0] - kernels[1]
    assert kernels[1] > 0 and extra > 0 and extra % 7 == 0
    got, exact = render_both(w, 1, [40, 41, 42])
    assert exact > 0.99
