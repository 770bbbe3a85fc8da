"""Seeded synthetic scenes with the shapes, sizes and value distributions of the
tracer workloads (there is no scene file or dataset on this path; the
reference's benchmark scenes are not reproduced).

  plain_512      512x512, ground quad + 64 UV spheres (~20k triangles), 3 rect
                 lights (key/fill/rim, radiance log-uniform 1-50), Lambert+GGX,
                 roughness U(0.05,1), albedo U(0.1,0.9), 16 spp, depth 4
  instanced_1080 1920x1080, ~200k instanced triangles (boxes and icospheres,
                 scales log-uniform 0.1-10, 8 Gaussian clusters), 128 point and
                 spot lights through the light tree, adaptive to 64, depth 8
  room_4k        3840x2160, ~1.2M triangles (room, shelves, 300 meshes of
                 1k-20k triangles), 32 materials incl. glass IOR 1.5 and metals,
                 128 lights, adaptive to 64, depth 8

Everything is float32, generated with numpy's PCG64 from the given seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import abi
from .trace import INSTANCE, LIGHT, MATERIAL, TRIANGLE, Adaptive, Camera, SceneDesc, Settings, Sun

F32 = np.float32


# ----------------------------------------------------------------- geometry
def triangles(v: np.ndarray, n: np.ndarray | None = None, material=0, uv: np.ndarray | None = None) -> np.ndarray:
    """TRIANGLE records; without normals, the flat normal of each triangle
    (TriangleDetail::flat, crates/trace/src/detail.rs:16-26)."""
    v = np.asarray(v, F32).reshape(-1, 3, 3)
    out = np.zeros(len(v), TRIANGLE)
    out["v"] = v
    if n is None:
        c = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]).astype(F32)
        ln = np.sqrt((c * c).sum(-1)).astype(F32)
        good = ln > F32(1e-12)
        flat = np.zeros_like(c)
        flat[good] = c[good] * (F32(1.0) / ln[good])[:, None]
        flat[~good] = (0.0, 0.0, 1.0)
        out["n"] = flat[:, None, :]
    else:
        out["n"] = np.asarray(n, F32).reshape(-1, 3, 3)
    if uv is not None:
        out["uv"] = np.asarray(uv, F32).reshape(-1, 3, 2)
    out["material"] = material
    return out


def quad(center, half_u, half_v, material=0) -> np.ndarray:
    c, u, w = (np.asarray(x, F32) for x in (center, half_u, half_v))
    p = [c - u - w, c + u - w, c + u + w, c - u + w]
    return triangles([[p[0], p[1], p[2]], [p[0], p[2], p[3]]], material=material)


def box(lo, hi, material=0, inward=False) -> np.ndarray:
    lo, hi = np.asarray(lo, F32), np.asarray(hi, F32)
    c = [np.array([hi[0] if i & 1 else lo[0], hi[1] if i & 2 else lo[1], hi[2] if i & 4 else lo[2]], F32)
         for i in range(8)]
    faces = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    tris = []
    for a, b, cc, d in faces:
        if inward:
            a, b, cc, d = a, d, cc, b
        tris += [[c[a], c[b], c[cc]], [c[a], c[cc], c[d]]]
    return triangles(tris, material=material)


def uv_sphere(center, radius, slices, stacks, material=0, wobble=None) -> np.ndarray:
    """UV sphere with smooth normals: 2*slices*(stacks-1) triangles."""
    th = np.linspace(0.0, math.pi, stacks + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, slices + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1)
    r = np.full(T.shape, radius, np.float64)
    if wobble is not None:
        r = r * wobble(d)
    p = (np.asarray(center, np.float64) + d * r[..., None]).astype(F32)
    d = d.astype(F32)
    i, j = np.meshgrid(np.arange(stacks), np.arange(slices), indexing="ij")
    a, b, c, e = (i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)
    # per quad: [a, b, e] except on the top row, [e, b, c] except on the bottom row
    first = np.stack([p[a], p[b], p[e]], 2)[1:].reshape(-1, 3, 3)
    first_n = np.stack([d[a], d[b], d[e]], 2)[1:].reshape(-1, 3, 3)
    second = np.stack([p[e], p[b], p[c]], 2)[:-1].reshape(-1, 3, 3)
    second_n = np.stack([d[e], d[b], d[c]], 2)[:-1].reshape(-1, 3, 3)
    return triangles(np.concatenate([first, second]), np.concatenate([first_n, second_n]), material=material)


def icosphere(subdivisions: int, material=0) -> np.ndarray:
    """Unit icosphere: 20 * 4^subdivisions triangles, smooth normals."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache, new = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new
    V = np.array(verts, np.float64)
    F = np.array(faces)
    p = V[F].astype(F32)
    return triangles(p, p.copy(), material=material)


def transform_matrix(scale, rotation: np.ndarray, translation) -> np.ndarray:
    """Column-major 4x4 affine (detail.rs Transform): column c, row r at [c*4+r]."""
    m = np.eye(4)
    m[:3, :3] = rotation @ np.diag(np.broadcast_to(scale, 3))
    m[:3, 3] = translation
    return m.T.reshape(-1).astype(F32)  # transpose: column-major flattening


def random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


# ----------------------------------------------------------------- materials
def material(base=(0.8, 0.8, 0.8), roughness=0.5, metalness=0.0, specular=0.04, transmission=0.0, ior=1.5,
             emission=(0.0, 0.0, 0.0), clearcoat=0.0, clearcoat_roughness=0.03, dispersion=0.0) -> np.ndarray:
    m = np.zeros(1, MATERIAL)
    m["base"] = base
    m["roughness"] = roughness
    m["metalness"] = metalness
    m["specular"] = specular
    m["clearcoat"] = clearcoat
    m["clearcoat_roughness"] = clearcoat_roughness
    m["transmission"] = transmission
    m["ior"] = ior
    m["dispersion"] = dispersion
    m["subsurface_tint"] = (1.0, 1.0, 1.0)
    m["emission"] = emission
    m["thin_film_ior"] = 1.3
    return m


# ----------------------------------------------------------------- lights
def rect_light(center, half_u, half_v, radiance, colour=(1.0, 1.0, 1.0)) -> np.ndarray:
    """LocalLight::rect with intensity = radiance x area (lights.rs:54-74, 212-215)."""
    l = np.zeros(1, LIGHT)
    hu, hv = np.asarray(half_u, F32), np.asarray(half_v, F32)
    area = F32(4.0) * np.linalg.norm(np.cross(hu, hv)).astype(F32)
    l["shape"] = abi.LIGHT_RECT
    l["shadow"] = 1
    l["position"] = center
    l["colour"] = colour
    l["intensity"] = F32(radiance) * area
    l["range"] = np.finfo(F32).max
    l["half_u"] = hu
    l["half_v"] = hv
    return l


def point_light(position, intensity, colour=(1.0, 1.0, 1.0), radius=0.0, rng_range=None) -> np.ndarray:
    l = np.zeros(1, LIGHT)
    l["shape"] = abi.LIGHT_POINT
    l["shadow"] = 1
    l["position"] = position
    l["colour"] = colour
    l["intensity"] = intensity
    l["radius"] = radius
    l["range"] = np.finfo(F32).max if rng_range is None else rng_range
    return l


def spot_light(position, direction, intensity, outer_deg, inner_deg, colour=(1.0, 1.0, 1.0), radius=0.0,
               rng_range=None) -> np.ndarray:
    l = point_light(position, intensity, colour, radius, rng_range)
    l["shape"] = abi.LIGHT_SPOT
    l["direction"] = direction
    l["outer_deg"] = outer_deg
    l["inner_deg"] = inner_deg
    return l


def look_at(eye, target, vfov_deg, aspect, world_up=(0.0, 1.0, 0.0)) -> Camera:
    eye, target = np.asarray(eye, np.float64), np.asarray(target, np.float64)
    f = target - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, world_up)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    h = math.tan(math.radians(vfov_deg) / 2.0)
    return Camera(tuple(map(float, eye)), tuple(map(float, f)), tuple(map(float, r * h * aspect)),
                  tuple(map(float, u * h)))


def _log_uniform(rng, lo, hi, n=None):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), n))


# ----------------------------------------------------------------- configs
@dataclass
class Workload:
    name: str
    scene: SceneDesc
    settings: Settings
    width: int
    height: int
    spp: int = 16
    adaptive: Adaptive | None = None


def plain_512(seed: int = 0, size: int = 512, sampler: str = "sobol") -> Workload:
    rng = np.random.default_rng(seed)
    mats = [material((0.5, 0.5, 0.5), 0.8)]
    tris = [quad((0, 0, 0), (20, 0, 0), (0, 0, -20), 0)]
    for i in range(64):
        r = rng.uniform(0.2, 1.0)
        c = rng.uniform((-10, 0, -10), (10, 20, 10))
        mats.append(material(tuple(rng.uniform(0.1, 0.9, 3)), rng.uniform(0.05, 1.0)))
        tris.append(uv_sphere(c, r, 13, 13, material=len(mats) - 1))
    lights = []
    # key (upper left front), fill (right), rim (behind): normals face the scene centre
    for center, toward in [((-12, 22, 14), (0, 8, 0)), ((16, 10, 10), (0, 8, 0)), ((0, 18, -18), (0, 8, 0))]:
        c = np.asarray(center, np.float64)
        nrm = np.asarray(toward, np.float64) - c
        nrm /= np.linalg.norm(nrm)
        a = np.cross(nrm, (0.0, 1.0, 0.0))
        if np.linalg.norm(a) < 1e-6:
            a = np.cross(nrm, (1.0, 0.0, 0.0))
        a /= np.linalg.norm(a)
        b = np.cross(nrm, a)  # cross(a, b) = nrm
        b = -b
        if np.dot(np.cross(a, b), nrm) < 0:
            b = -b
        lights.append(rect_light(center, a * 1.5, b * 1.5, _log_uniform(rng, 1.0, 50.0)))
    scene = SceneDesc(np.concatenate(tris), np.concatenate(mats), look_at((0, 9, 34), (0, 8, 0), 45.0, 1.0),
                      lights=np.concatenate(lights))
    return Workload("plain_512", scene, Settings.deep(4, sampler=sampler, sobol_samples=16), size, size, spp=16)


def instanced_1080(seed: int = 1, width: int = 1920, height: int = 1080, target: int = 200_000,
                   sampler: str = "sobol") -> Workload:
    rng = np.random.default_rng(seed)
    mats = [material((0.45, 0.45, 0.45), 0.9)]
    for _ in range(15):
        mats.append(material(tuple(rng.uniform(0.1, 0.9, 3)), rng.uniform(0.05, 1.0),
                             metalness=float(rng.uniform() < 0.25)))
    cube = box((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), 0)
    ico = icosphere(3, 0)  # 1280 triangles
    meshes = [cube, ico]
    clusters = rng.uniform((-60, 5, -60), (60, 40, 60), (8, 3))
    inst, total = [], 0
    while total < target:
        k = int(rng.integers(0, 2))
        s = float(_log_uniform(rng, 0.1, 10.0))
        c = clusters[rng.integers(0, 8)] + rng.normal(0.0, 12.0, 3)
        rec = np.zeros(1, INSTANCE)
        rec["mesh"] = k
        rec["two_sided"] = 1
        rec["casts_shadow"] = 1
        rec["transform"] = transform_matrix(s, random_rotation(rng), c)
        inst.append(rec)
        total += len(meshes[k])
    # one material per mesh (all instances of a mesh share its triangles)
    meshes[0]["material"] = 1 + int(rng.integers(0, 15))
    meshes[1]["material"] = 1 + int(rng.integers(0, 15))
    world = quad((0, 0, 0), (150, 0, 0), (0, 0, -150), 0)
    lights = []
    for i in range(128):
        p = clusters[rng.integers(0, 8)] + rng.normal(0.0, 15.0, 3)
        p[1] = abs(p[1]) + 2.0
        inten = float(_log_uniform(rng, 1.0, 1000.0))
        col = tuple(rng.uniform(0.6, 1.0, 3))
        if i % 2 == 0:
            lights.append(point_light(p, inten, col))
        else:
            d = rng.normal(size=3)
            d[1] = -abs(d[1]) - 0.5
            outer = float(rng.uniform(10.0, 60.0))
            lights.append(spot_light(p, d / np.linalg.norm(d), inten, outer, 0.8 * outer, col))
    scene = SceneDesc(world, np.concatenate(mats), look_at((0, 35, 130), (0, 15, 0), 50.0, width / height),
                      lights=np.concatenate(lights), meshes=meshes, instances=np.concatenate(inst))
    return Workload("instanced_1080", scene, Settings.deep(8, sampler=sampler, sobol_samples=64), width, height,
                    spp=64, adaptive=Adaptive(threshold=0.01, min_samples=16, max_samples=64, growth=1.5))


def room_4k(seed: int = 2, width: int = 3840, height: int = 2160, target: int = 1_200_000, meshes_n: int = 300,
            sampler: str = "sobol", light_radius=(0.1, 0.3), light_scale: float = 0.05, light_height=(6.0, 9.6),
            light_seed=None) -> Workload:
    """Lights are soft (bulb radius U(0.1, 0.3) m) and hang in the upper part of
    the room, as ceiling fixtures do."""
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(32):
        kind = i % 3
        if i in (30, 31):  # glass, IOR 1.5
            mats.append(material((1.0, 1.0, 1.0), 0.02, transmission=1.0, ior=1.5))
        elif kind == 0:  # diffuse
            mats.append(material(tuple(rng.uniform(0.1, 0.9, 3)), float(rng.uniform(0.5, 1.0))))
        elif kind == 1:  # metal
            mats.append(material(tuple(rng.uniform(0.5, 0.95, 3)), float(rng.uniform(0.05, 0.6)), metalness=1.0))
        else:  # glossy dielectric with a clear coat on some
            mats.append(material(tuple(rng.uniform(0.1, 0.9, 3)), float(rng.uniform(0.05, 0.4)), specular=0.5,
                                 clearcoat=float(rng.uniform() < 0.3)))
    W, H, D = 30.0, 10.0, 30.0
    parts = [box((-W / 2, 0, -D / 2), (W / 2, H, D / 2), 0, inward=True)]
    shelves = []
    for k in range(6):  # shelves along the back and side walls
        y = 1.5 + 1.6 * (k % 3)
        if k < 3:
            shelves.append(box((-12, y, -14.6), (12, y + 0.08, -12.8), 3))
        else:
            shelves.append(box((-14.6, y, -10), (-12.8, y + 0.08, 10), 3))
    parts += shelves
    n_tri = rng.uniform(math.log(1000), math.log(20000), meshes_n)
    counts = np.exp(n_tri)
    counts = np.clip(counts * ((target - 300) / counts.sum()), 1000, 20000).astype(int)
    for i in range(meshes_n):
        n = int(counts[i])
        slices = max(6, int(round(math.sqrt(n))))
        stacks = max(3, n // (2 * slices) + 1)
        radius = float(rng.uniform(0.15, 0.9))
        freq = rng.uniform(1.0, 5.0, 3)
        amp = float(rng.uniform(0.0, 0.3))
        phase = rng.uniform(0, 6.28, 3)

        def wobble(d, freq=freq, amp=amp, phase=phase):
            return 1.0 + amp * np.sin(freq[0] * d[..., 0] + phase[0]) * np.sin(freq[1] * d[..., 1] + phase[1]) \
                * np.cos(freq[2] * d[..., 2] + phase[2])

        c = rng.uniform((-13, radius, -13), (13, 8.5, 13))
        m = int(rng.integers(0, 32))
        parts.append(uv_sphere(c, radius, slices, stacks, material=m, wobble=wobble))
    tris = np.concatenate(parts)
    lights = []
    lrng = np.random.default_rng(seed + 100) if light_seed is None else np.random.default_rng(light_seed)
    for i in range(128):
        p = lrng.uniform((-14, light_height[0], -14), (14, light_height[1], 14))
        inten = float(_log_uniform(lrng, 1.0, 1000.0)) * light_scale
        col = tuple(lrng.uniform(0.6, 1.0, 3))
        radius = float(lrng.uniform(*light_radius))
        if i % 2 == 0:
            lights.append(point_light(p, inten, col, radius=radius))
        else:
            d = lrng.normal(size=3)
            d[1] = -abs(d[1]) - 0.3
            outer = float(lrng.uniform(10.0, 60.0))
            lights.append(spot_light(p, d / np.linalg.norm(d), inten, outer, 0.8 * outer, col, radius=radius))
    scene = SceneDesc(tris, np.concatenate(mats), look_at((0, 5, 14.5), (0, 4, 0), 60.0, width / height),
                      lights=np.concatenate(lights))
    # the reference's firefly controls, at the values its own firefly test
    # renders with (crates/trace/tests/fireflies.rs:21-22)
    settings = Settings.deep(8, sampler=sampler, sobol_samples=64, filter_glossy=0.25, clamp_indirect=4.0)
    return Workload("room_4k", scene, settings, width, height, spp=64,
                    adaptive=Adaptive(threshold=0.01, min_samples=16, max_samples=64, growth=1.5))


def lcg_triangles():
    """The fixture of the reference's BVH test (crates/trace/src/bvh.rs:330-381):
    120 triangles and 2000 rays from an LCG seeded with 17."""
    state = [17]

    def random():
        state[0] = (state[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return F32((state[0] >> 8)) / F32(1 << 24)

    verts = []
    for _ in range(120):
        x = random() * F32(8.0) - F32(4.0)
        y = random() * F32(8.0) - F32(4.0)
        z = random() * F32(8.0) - F32(4.0)
        a = [x, y, z]
        b = [x + random() + F32(0.1), y, z]
        c = [x, y + random() + F32(0.1), z]
        verts.append([a, b, c])
    rays = []
    for _ in range(2000):
        o = [random() * F32(12.0) - F32(6.0), random() * F32(12.0) - F32(6.0), random() * F32(12.0) - F32(6.0)]
        d = np.array([random() * F32(2.0) - F32(1.0), random() * F32(2.0) - F32(1.0),
                      random() * F32(2.0) - F32(1.0)], F32)
        ln = np.sqrt(np.dot(d, d)).astype(F32)
        d = d * (F32(1.0) / ln) if ln > F32(1e-12) else np.array([0, 0, 1], F32)
        rays.append((o, d))
    return np.array(verts, F32), rays


def camera_rays(cam: Camera, width: int, height: int, n: int, rng, tmax: float = 1e20) -> np.ndarray:
    """Primary rays through random pixel positions (trace.wgsl:2538-2552 with
    the lens shift at zero)."""
    from .trace import make_rays
    px = rng.uniform(0, width, n).astype(F32)
    py = rng.uniform(0, height, n).astype(F32)
    ndc_x = px / F32(width) * F32(2) - F32(1)
    ndc_y = py / F32(height) * F32(2) - F32(1)
    f, r, u = (np.asarray(x, F32) for x in (cam.forward, cam.right, cam.up))
    d = f[None] + r[None] * ndc_x[:, None] + u[None] * (-ndc_y)[:, None]
    d = d / np.sqrt((d * d).sum(-1))[:, None]
    o = np.broadcast_to(np.asarray(cam.origin, F32), d.shape)
    return make_rays(o, d.astype(F32), tmax)


def random_rays(lo, hi, n: int, rng, tmax: float = 1e20) -> np.ndarray:
    from .trace import make_rays
    o = rng.uniform(lo, hi, (n, 3)).astype(F32)
    d = rng.normal(size=(n, 3)).astype(F32)
    d = d / np.sqrt((d * d).sum(-1))[:, None]
    return make_rays(o, d.astype(F32), tmax)


WORKLOADS = {"plain_512": plain_512, "instanced_1080": instanced_1080, "room_4k": room_4k}


def furnace() -> SceneDesc:
    """The reference's furnace scene (crates/trace/src/gpu.rs:3787-3830): a white
    diffuse unit sphere three units in front of the camera under a uniform white
    sky; an icosphere stands in for the analytic ellipsoid."""
    ico = icosphere(4, 0)
    ico["v"] = ico["v"] + np.array([0.0, 0.0, -3.0], F32)
    cam = Camera((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    return SceneDesc(ico, material((1.0, 1.0, 1.0), 1.0, specular=0.0), cam, sky=(1.0, 1.0, 1.0))


IDENTITY = np.eye(4, dtype=F32)


def placed(at, turn: float, scale: float) -> np.ndarray:
    """A turn about +y, a uniform scale and a translation as a column-major 4x4
    (the `placed` helper of crates/trace/tests/instances.rs:89-97)."""
    s, c = math.sin(turn), math.cos(turn)
    return np.array([[c * scale, 0.0, -s * scale, 0.0], [0.0, scale, 0.0, 0.0], [s * scale, 0.0, c * scale, 0.0],
                     [at[0], at[1], at[2], 1.0]], F32)


def staged_poses(moved: bool) -> list:
    """The two sets of placements of crates/trace/tests/instances.rs:137-157:
    floor, two balls and an emissive panel."""
    if moved:
        return [IDENTITY, placed((0.5, 0.45, -0.2), 0.9, 0.9), placed((-0.9, 0.35, 0.6), -0.4, 0.7),
                placed((-0.3, 1.6, -0.5), 0.6, 1.0)]
    return [IDENTITY, placed((-0.4, 0.5, 0.0), 0.0, 1.0), placed((0.8, 0.5, 0.4), 0.3, 1.0),
            placed((0.0, 1.8, -0.8), 0.0, 1.0)]


def staged(transforms, size=(96, 64), world: bool = False, empty: bool = False) -> Workload:
    """The instanced stage of crates/trace/tests/instances.rs:159-197: a floor,
    one ball mesh placed twice (red and grey), an emissive panel, a dim sky and
    a sun.  `world` adds a back wall as world triangles; `empty` appends an
    instance of an empty mesh (never placed)."""
    lambert = lambda base: material(base, 1.0, specular=0.0)  # noqa: E731
    mats = np.concatenate([lambert((0.6, 0.6, 0.6)), lambert((0.8, 0.2, 0.1)),
                           material((0.0, 0.0, 0.0), 1.0, specular=0.0, emission=(6.0, 5.0, 4.0))])
    floor = quad((0, 0, 0), (3, 0, 0), (0, 0, 3), 0)
    panel = quad((0, 0, 0), (0.4, 0, 0), (0, 0, 0.4), 2)
    meshes = [floor, uv_sphere((0, 0, 0), 0.5, 32, 16, 1), uv_sphere((0, 0, 0), 0.5, 32, 16, 0), panel,
              np.zeros(0, TRIANGLE)]
    inst = np.zeros(4 + int(empty), INSTANCE)
    inst["mesh"][:4] = [0, 1, 2, 3]
    if empty:
        inst["mesh"][4] = 4
        inst["transform"][4] = IDENTITY.reshape(16)
    inst["two_sided"] = 1
    inst["casts_shadow"] = 1
    for i, t in enumerate(transforms[:4]):
        inst["transform"][i] = np.asarray(t, F32).reshape(16)
    wall = quad((0, 1.5, -3), (3, 0, 0), (0, 1.5, 0), 0) if world else np.zeros(0, TRIANGLE)
    w, h = size
    cam = look_at((0.0, 2.0, 4.0), (0.0, 0.4, 0.0), 2.0 * math.degrees(math.atan(0.5)), w / h)
    d = np.array([0.4, 1.0, 0.3])
    scene = SceneDesc(wall, mats, cam, meshes=meshes, instances=inst, sky=(0.08, 0.09, 0.1),
                      sun=Sun(tuple(map(float, d / np.linalg.norm(d))), (1.0, 0.95, 0.9), 2.0))
    return Workload("staged", scene, Settings.deep(4, sampler="pcg"), w, h, spp=8)


def small(name: str, size=(64, 48), sampler: str = "pcg") -> Workload:
    """A reduced-resolution copy of a workload for parity tests (same scene
    generator, smaller film, fewer triangles where the generator allows)."""
    if name == "plain_512":
        w = plain_512(sampler=sampler)
    elif name == "instanced_1080":
        w = instanced_1080(target=20_000, sampler=sampler)
    else:
        w = room_4k(target=60_000, meshes_n=30, sampler=sampler)
    w.width, w.height = size
    cam = w.scene.camera
    aspect = size[0] / size[1]
    scale = aspect / (np.linalg.norm(cam.right) / np.linalg.norm(cam.up))
    w.scene.camera = Camera(cam.origin, cam.forward, tuple(np.asarray(cam.right) * scale), cam.up)
    return w
