"""The oracle's restatement of the path integrator against the reference's
own statistical pins (crates/trace/src/gpu.rs GPU tests, run here on the CPU)."""
import numpy as np

import oracle
from pfx_b200 import synth
from pfx_b200.trace import SceneBuffers, Settings

# The frame the product computes on the host (gpu.rs:2295-2316) for a
# perspective camera without lens, sun or window offset: size, counts,
# origin..lens, window.
def frame_of(scene, settings, w, h, tri_count):
    f = np.zeros(40, np.uint32)
    fl = f.view(np.float32)
    f[0:4] = (w, h, 0, 0)
    f[4:8] = (tri_count, 0, 0, 0)
    fl[8:11] = scene.camera.origin
    fl[12:15] = scene.camera.forward
    fl[16:19] = scene.camera.right
    fl[20:23] = scene.camera.up
    fl[24:27] = scene.sun.direction
    fl[27] = 1.0  # cos(0 degrees)
    fl[28:31] = scene.sun.color
    fl[31] = scene.sun.intensity
    fl[32:36] = (0.0, 0.0, 0.0, 1.0)
    f[36:40] = (w, h, 0, 0)
    return f


def test_furnace_on_the_oracle():
    # gpu.rs:3787-3830: 32 passes of 4 samples (seeds 73..104), centre pixel 1 +- 0.12
    scene = synth.furnace()
    settings = Settings(sampler="pcg")
    sb = SceneBuffers(scene, settings)
    r = oracle.Renderer(sb, settings)
    f = frame_of(scene, settings, 16, 16, sb.buffers.triangle_count)
    accum = np.zeros((16, 16, 12), np.float32)
    accum2 = np.zeros_like(accum)
    samples = 0
    for p in range(32):
        color, _, _ = r.render(f, accum, samples, 4, 73 + p)
        color2, _, _ = r.render(f, accum2, samples, 4, 73 + p)
        samples += 4
    assert np.array_equal(accum, accum2)  # same seeds, same bytes
    mid = color[8, 8, :3]
    assert np.all(np.abs(mid - 1.0) < 0.12), mid


def test_sobol_and_pcg_agree_on_the_mean():
    # gpu.rs:5660-5685: the mean of an image differs by < 2 % between samplers
    w = synth.small("plain_512", (32, 32), sampler="pcg")
    means = []
    for sampler in ("pcg", "sobol"):
        settings = Settings.deep(4, sampler=sampler, sobol_samples=64)
        sb = SceneBuffers(w.scene, settings)
        r = oracle.Renderer(sb, settings)
        f = frame_of(w.scene, settings, 32, 32, sb.buffers.triangle_count)
        accum = np.zeros((32, 32, 12), np.float32)
        color, _, _ = r.render(f, accum, 0, 64, 5)
        means.append(float(color[..., :3].mean()))
    assert abs(means[0] - means[1]) / means[1] < 0.02, means
