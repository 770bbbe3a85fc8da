"""Stage (crates/trace/src/stage.rs:28-386): a scene described as indexed
meshes placed by instances, turned into the tracer's scene.

    staged = Stage(meshes=[...], instances=[Placement(0, model, material)],
                   materials=..., sky=Sky(1, 1, [[r, g, b, 1]]), sun=Sun(...),
                   camera=Camera(...)).build()        # Stage::build
    trace = staged.trace(width, height)               # Staged::trace

As in the reference, every placement becomes an instance whose triangles carry
the placement's material; placements of the same mesh with the same material
share one triangle list (and so one bottom-level BVH), and the staged scene has
no world triangles.  Vertex alpha below a placement's cutoff is cut out of the
geometry as the reference cuts it.  The parts of a stage this tracer does not
render (clip planes, content images and text, motion, image-based skies) are
refused with an error instead of being dropped.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import TraceError
from .trace import INSTANCE, TRIANGLE, Camera, SceneDesc, Settings, Sun, Trace

ALPHA_CUTOFF = 0.5


def _invalid(message: str) -> TraceError:
    """The reference's Stage::build errors, as the C ABI's invalid-argument errors."""
    return TraceError(abi.ERR_INVALID, message)


@dataclass
class Mesh:
    """stage.rs Mesh: per-vertex attributes and triangle indices."""
    positions: np.ndarray            # (n, 3)
    normals: np.ndarray              # (n, 3)
    tangents: np.ndarray             # (n, 4), checked for its length only
    uvs: np.ndarray                  # (n, 2)
    indices: np.ndarray              # (3 m,)
    uvs1: np.ndarray | None = None   # (n, 2)
    alpha: np.ndarray | None = None  # (n,)


@dataclass
class Placement:
    """stage.rs Placement (Placement::new's defaults)."""
    mesh: int
    model: np.ndarray                # column-major 4x4 (detail.rs Transform)
    material: int
    casts_shadow: bool = True
    shadow_only: bool = False
    two_sided: bool = True
    alpha_cutoff: float = ALPHA_CUTOFF
    clip: np.ndarray = field(default_factory=lambda: np.zeros((2, 4), np.float32))
    content: object = None
    motion: object = None


@dataclass
class Sky:
    """pfx_load::Sky: an environment image of width x height RGBA texels."""
    width: int
    height: int
    texels: np.ndarray               # (width * height, 4)

    def radiance(self) -> tuple:
        t = np.asarray(self.texels, np.float32).reshape(-1, 4)
        if self.width * self.height != len(t) or len(t) == 0:
            raise _invalid("staged sky has the wrong texel count")
        if not np.all(t[:, :3] == t[0, :3]):
            raise _invalid("image-based skies are outside this tracer's scope (a uniform sky is supported)")
        return tuple(float(x) for x in t[0, :3])


@dataclass
class Staged:
    """stage.rs Staged: the scene and the detail settings."""
    scene: SceneDesc
    settings: Settings

    def trace(self, width: int, height: int) -> Trace:
        """Staged::trace (stage.rs:383): Trace::new_detailed of the staged scene."""
        return Trace(self.scene, self.settings, width, height)


def _check_mesh(mesh: Mesh) -> None:
    """check_mesh (stage.rs:717-734)."""
    count = len(mesh.positions)
    indices = np.asarray(mesh.indices).reshape(-1)
    if count == 0 or len(indices) == 0 or len(indices) % 3 != 0:
        raise _invalid("mesh needs vertices and triangle indices")
    if (len(mesh.normals) != count or len(mesh.tangents) != count or len(mesh.uvs) != count
            or (mesh.uvs1 is not None and len(mesh.uvs1) != count)
            or (mesh.alpha is not None and len(mesh.alpha) != count)):
        raise _invalid("mesh attributes have different vertex counts")
    if np.any(indices.astype(np.int64) >= count) or np.any(indices.astype(np.int64) < 0):
        raise _invalid("mesh index is outside the vertex buffer")


def _cut(corners: list, cutoff: np.float32) -> list:
    """cut / cut_at (stage.rs:770-820): the corners of a triangle clipped to
    where the vertex alpha is at least `cutoff` (interpolated linearly along
    each edge, in f32 as the reference does); all three kept when all pass."""
    if all(c[3] >= cutoff for c in corners):
        return corners
    kept = []
    for k in range(3):
        a, b = corners[k], corners[(k + 1) % 3]
        inside_a, inside_b = a[3] >= cutoff, b[3] >= cutoff
        if inside_a:
            kept.append(a)
        if inside_a != inside_b:
            t = (cutoff - a[3]) / (b[3] - a[3])
            kept.append(tuple([x + (y - x) * t for x, y in zip(a[:3], b[:3])]) + (cutoff,))
    return kept


def _triangles(mesh: Mesh, material: int, cutoff: float) -> np.ndarray:
    """triangles (stage.rs:736-768): one triangle per index triple, corners in
    index order, with the placement's material; where vertex alpha is given,
    each triangle is first clipped to alpha >= cutoff and the kept polygon
    fanned from its first corner."""
    _check_mesh(mesh)
    f = np.asarray(mesh.indices, np.int64).reshape(-1, 3)
    pos = np.asarray(mesh.positions, np.float32)
    nrm = np.asarray(mesh.normals, np.float32)
    uvs = np.asarray(mesh.uvs, np.float32)
    if mesh.alpha is None or np.all(np.asarray(mesh.alpha, np.float32) >= np.float32(cutoff)):
        out = np.zeros(len(f), TRIANGLE)
        out["v"], out["n"], out["uv"] = pos[f], nrm[f], uvs[f]
        out["material"] = material
        return out
    alpha = np.asarray(mesh.alpha, np.float32)
    c32 = np.float32(cutoff)
    tris = []
    for face in f:
        # a corner: (position, normal, uv, alpha) with float32 components
        corners = [(pos[i], nrm[i], uvs[i], alpha[i]) for i in face]
        kept = _cut(corners, c32)
        for k in range(1, len(kept) - 1):
            tris.append((kept[0], kept[k], kept[k + 1]))
    out = np.zeros(len(tris), TRIANGLE)
    for i, corners in enumerate(tris):
        out[i]["v"] = [c[0] for c in corners]
        out[i]["n"] = [c[1] for c in corners]
        out[i]["uv"] = [c[2] for c in corners]
    out["material"] = material
    return out


@dataclass
class Stage:
    """stage.rs Stage."""
    meshes: list
    instances: list
    materials: np.ndarray            # MATERIAL records
    sky: Sky
    sun: Sun
    camera: Camera
    projection: object = "perspective"  # "perspective", ("orthographic", width, height) or "equirect"
    lens: tuple = (0.0, 0.0, 0.0, 1.0)  # shift x, shift y, aperture, focus distance
    detail: Settings = field(default_factory=Settings)

    def _projection(self):
        p = self.projection
        if p == "perspective":
            return abi.PROJECTION_PERSPECTIVE, (0.0, 0.0)
        if p == "equirect":
            return abi.PROJECTION_EQUIRECT, (0.0, 0.0)
        if isinstance(p, tuple) and len(p) == 3 and p[0] == "orthographic":
            w, h = float(p[1]), float(p[2])
            if np.isfinite(w) and np.isfinite(h) and w > 0 and h > 0:
                return abi.PROJECTION_ORTHOGRAPHIC, (w, h)
        raise _invalid("staged camera has an invalid projection or lens")

    def build(self) -> Staged:
        """Stage::build (stage.rs:211-381)."""
        if len(self.materials) == 0:
            raise _invalid("staged scene needs at least one material")
        kind, ortho = self._projection()
        lens = tuple(float(x) for x in self.lens)
        if len(lens) != 4 or not all(np.isfinite(lens)) or lens[2] < 0.0 or lens[3] <= 0.0:
            raise _invalid("staged camera has an invalid projection or lens")
        for mesh in self.meshes:
            _check_mesh(mesh)
        dressed: dict = {}
        meshes, inst = [], np.zeros(len(self.instances), INSTANCE)
        for i, p in enumerate(self.instances):
            if not (0.0 <= p.alpha_cutoff <= 1.0):
                raise _invalid("staged alpha cutoff must be a fraction from 0 to 1")
            clip = np.asarray(p.clip, np.float32)
            if not np.all(np.isfinite(clip)):
                raise _invalid("staged clip plane is not finite")
            if not (0 <= p.mesh < len(self.meshes)):
                raise _invalid("staged instance names a missing mesh")
            if not (0 <= p.material < len(self.materials)):
                raise _invalid("staged instance names a missing material")
            if p.content is not None:
                raise _invalid("content images and text are outside this tracer's scope")
            if p.motion is not None:
                raise _invalid("motion blur is outside this tracer's scope")
            if np.any(clip != 0.0):
                raise _invalid("clip planes are outside this tracer's scope")
            key = (p.mesh, np.float32(p.alpha_cutoff).view(np.uint32).item(), p.material)
            if key not in dressed:  # one triangle list per (mesh, cutoff, material), as `dressed`
                dressed[key] = len(meshes)
                meshes.append(_triangles(self.meshes[p.mesh], p.material, p.alpha_cutoff))
            inst[i]["mesh"] = dressed[key]
            inst[i]["transform"] = np.asarray(p.model, np.float32).reshape(16)
            inst[i]["casts_shadow"] = 1 if p.casts_shadow else 0
            inst[i]["shadow_only"] = 1 if p.shadow_only else 0
            inst[i]["two_sided"] = 1 if p.two_sided else 0
        scene = SceneDesc(np.zeros(0, TRIANGLE), np.asarray(self.materials), self.camera, meshes=meshes,
                          instances=inst, sky=self.sky.radiance(), sun=self.sun)
        d = self.detail
        settings = Settings(bounces=d.bounces, sampler=d.sampler, sobol_samples=d.sobol_samples,
                            clamp_indirect=d.clamp_indirect, filter_glossy=d.filter_glossy, projection=kind,
                            ortho=ortho, lens=lens)
        return Staged(scene, settings)
