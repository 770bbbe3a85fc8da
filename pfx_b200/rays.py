"""Ray batches with the mix of one tracing pass: camera rays, bounce rays
from their hit points (cosine-weighted around the geometric normal) and shadow
rays from the same points to the lights (limit = distance*0.9999 - 0.0002, as
shadow_ray in lights.wgsl:95-102)."""
from __future__ import annotations

import numpy as np

from .synth import camera_rays
from .trace import make_rays

F32 = np.float32


def geometric_normals(buffers, slots: np.ndarray, records: np.ndarray, instances=None, hit=None) -> np.ndarray:
    """World-space geometric normals of hit triangles (slot order records).
    Rows where `hit` is false (missed rays, whose slot and record mean nothing)
    get +z."""
    if hit is not None:
        out = np.zeros((len(slots), 3), F32)
        out[:, 2] = 1.0
        if hit.any():
            out[hit] = geometric_normals(buffers, slots[hit], records[hit], instances)
        return out
    tri = buffers.array("triangles").view(np.float32).reshape(-1, 24)[slots]
    a, b, c = tri[:, 0:3], tri[:, 4:7], tri[:, 8:11]
    n = np.cross(b - a, c - a)
    if instances is not None and len(instances):
        surf = buffers.array("surfaces").view(np.float32).reshape(-1, 44)
        inv = surf[records][:, 32:44].reshape(-1, 3, 4)[:, :, :3]  # inverse rows
        # normals transform with the inverse transpose: n_world = inv^T n
        n = np.where(records[:, None] > 0, np.einsum("kji,kj->ki", inv, n), n)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-20)
    return n.astype(F32)


def pixel_rays(cam, width: int, height: int, n: int, rng, tmax: float = 1e20) -> np.ndarray:
    """Camera rays for n consecutive pixels in scanline order (wrapping), one
    jittered sample each, as one pass of the tracer generates them."""
    start = int(rng.integers(0, width * height))
    pix = (start + np.arange(n)) % (width * height)
    px = (pix % width).astype(F32) + rng.uniform(0, 1, n).astype(F32)
    py = (pix // width).astype(F32) + rng.uniform(0, 1, n).astype(F32)
    ndc_x = px / F32(width) * F32(2) - F32(1)
    ndc_y = py / F32(height) * F32(2) - F32(1)
    f, r, u = (np.asarray(x, F32) for x in (cam.forward, cam.right, cam.up))
    d = f[None] + r[None] * ndc_x[:, None] + u[None] * (-ndc_y)[:, None]
    d = d / np.sqrt((d * d).sum(-1))[:, None]
    o = np.broadcast_to(np.asarray(cam.origin, F32), d.shape)
    return make_rays(o, d.astype(F32), tmax)


def pass_mix(trace, scene, width, height, n: int, seed: int = 0):
    """(closest-hit rays, any-hit rays): n/2 camera + bounce rays traced for the
    closest hit, and up to n/2 shadow rays; uses the tracer itself to find the
    camera rays' hit points."""
    rng = np.random.default_rng(seed)
    half = n // 2
    cam = pixel_rays(scene.camera, width, height, half, rng)
    hits = trace.trace_rays(cam)
    ok = hits["hit"] == 1
    p = cam["origin"] + cam["direction"] * np.where(ok, hits["t"], F32(0.0))[:, None]
    nrm = geometric_normals(trace.scene_buffers, hits["slot"], hits["record"].astype(np.int64), scene.instances,
                            hit=ok)
    nrm = np.where((nrm * cam["direction"]).sum(1, keepdims=True) > 0, -nrm, nrm)
    origin = (p + nrm * F32(1e-3) * np.maximum(1.0, np.abs(p).max(1, keepdims=True))).astype(F32)
    # cosine-weighted bounce directions
    u1, u2 = rng.uniform(size=half), rng.uniform(size=half)
    r, phi = np.sqrt(u2), 2 * np.pi * u1
    local = np.stack([r * np.cos(phi), r * np.sin(phi), np.sqrt(1 - u2)], 1)
    helper = np.where(np.abs(nrm[:, 1:2]) > 0.9, [[1.0, 0, 0]], [[0, 1.0, 0]])
    t = np.cross(helper, nrm)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    bt = np.cross(nrm, t)
    d = (t * local[:, :1] + bt * local[:, 1:2] + nrm * local[:, 2:3]).astype(F32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    bounce = make_rays(origin[ok], d[ok], 1e20)
    closest = np.concatenate([cam, bounce])[:half + half // 2]
    # shadow rays toward random lights (or random points above the scene)
    lights = scene.lights
    if len(lights):
        pos = lights["position"][rng.integers(0, len(lights), half)]
    else:
        pos = origin + rng.normal(size=(half, 3)) * 10
    to = (pos - origin).astype(F32)
    dist = np.linalg.norm(to, axis=1)
    sd = (to / np.maximum(dist, 1e-20)[:, None]).astype(F32)
    limit = (dist * F32(0.9999) - F32(0.0002)).astype(F32)
    keep = ok & (limit > 0)
    shadow = make_rays(origin[keep], sd[keep], limit[keep])
    return closest, shadow
