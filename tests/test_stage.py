"""Stage::build (crates/trace/src/stage.rs:211-381) on the host: the stage of
the reference's own test crates/trace/tests/instances.rs (a floor, one ball
mesh placed twice with two materials, an emissive panel), its build counts
and the reference's refusals."""
import math

import numpy as np
import pytest

from pfx_b200 import synth
from pfx_b200.stage import Mesh, Placement, Sky, Stage
from pfx_b200.trace import SceneBuffers, Settings, Sun, TraceError


def quad(half):
    """Arrays::quad (instances.rs:40-53)."""
    p = np.array([[-half, 0, -half], [half, 0, -half], [half, 0, half], [-half, 0, half]], np.float32)
    return Mesh(p, np.tile([0, 1, 0], (4, 1)).astype(np.float32), np.tile([1, 0, 0, 1], (4, 1)).astype(np.float32),
                np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32), np.array([0, 2, 1, 0, 3, 2], np.uint32))


def sphere(radius):
    """Arrays::sphere (instances.rs:55-87): 16 rings, 32 segments."""
    rings, segments = 16, 32
    normals, uvs = [], []
    for ring in range(rings + 1):
        theta = math.pi * ring / rings
        for segment in range(segments + 1):
            phi = 2 * math.pi * segment / segments
            normals.append([math.sin(theta) * math.cos(phi), math.cos(theta), math.sin(theta) * math.sin(phi)])
            uvs.append([segment / segments, ring / rings])
    row, indices = segments + 1, []
    for ring in range(rings):
        for segment in range(segments):
            a = ring * row + segment
            b = a + row
            indices += [a, a + 1, b, a + 1, b + 1, b]
    n = np.array(normals, np.float32)
    return Mesh(n * np.float32(radius), n, np.tile([1, 0, 0, 1], (len(n), 1)).astype(np.float32),
                np.array(uvs, np.float32), np.array(indices, np.uint32))


def materials():
    """instances.rs:99-117: two Lambert colours and an emitter."""
    lambert = lambda base: synth.material(base, 1.0, specular=0.0)  # noqa: E731
    return np.concatenate([lambert((0.6, 0.6, 0.6)), lambert((0.8, 0.2, 0.1)),
                           synth.material((0.0, 0.0, 0.0), 1.0, specular=0.0, emission=(6.0, 5.0, 4.0))])


def staged(poses, **kw):
    placements = [Placement(0, poses[0], 0), Placement(1, poses[1], 1), Placement(1, poses[2], 0),
                  Placement(2, poses[3], 2)]
    cam = synth.look_at((0.0, 2.0, 4.0), (0.0, 0.4, 0.0), 53.13, 96 / 64)
    d = np.array([0.4, 1.0, 0.3])
    stage = Stage([quad(3.0), sphere(0.5), quad(0.4)], placements, materials(),
                  Sky(1, 1, np.array([[0.08, 0.09, 0.1, 1.0]], np.float32)),
                  Sun(tuple(d / np.linalg.norm(d)), (1.0, 0.95, 0.9), 2.0), cam,
                  detail=Settings.deep(4, sampler="pcg"), **kw)
    return stage.build()


def test_the_staged_scene_builds_three_bottoms_and_one_top():
    """Builds { bottom: 3, top: 1 } (instances.rs:263); a partial move lays one
    more top and no bottom (instances.rs:267-270)."""
    s = staged(synth.staged_poses(False))
    assert len(s.scene.triangles) == 0 and len(s.scene.meshes) == 4  # (ball, red) and (ball, grey) apart
    assert [int(m["material"][0]) for m in s.scene.meshes] == [0, 1, 0, 2]
    assert s.scene.world_triangle_count == 2 + 1024 + 1024 + 2
    assert s.scene.sky == pytest.approx((0.08, 0.09, 0.1))
    b = SceneBuffers(s.scene, s.settings)
    assert b.builds() == (3, 1)
    assert b.move_instances(synth.staged_poses(True)[:2])
    assert b.builds() == (3, 2)


def test_placements_share_their_dressed_triangles():
    s = staged(synth.staged_poses(False))
    inst = s.scene.instances
    assert list(inst["mesh"]) == [0, 1, 2, 3]
    again = Stage([quad(1.0)], [Placement(0, synth.IDENTITY, 0), Placement(0, synth.placed((1, 0, 0), 0.0, 1.0), 0)],
                  materials(), Sky(1, 1, np.ones((1, 4), np.float32)), Sun(), s.scene.camera).build()
    assert len(again.scene.meshes) == 1 and list(again.scene.instances["mesh"]) == [0, 0]


def test_reference_refusals():
    cam = synth.look_at((0, 2, 4), (0, 0, 0), 60, 1.0)
    sky = Sky(1, 1, np.ones((1, 4), np.float32))
    ok = quad(1.0)
    with pytest.raises(TraceError, match="at least one material"):
        Stage([ok], [], np.zeros(0, materials().dtype), sky, Sun(), cam).build()
    with pytest.raises(TraceError, match="missing mesh"):
        Stage([ok], [Placement(1, synth.IDENTITY, 0)], materials(), sky, Sun(), cam).build()
    with pytest.raises(TraceError, match="missing material"):
        Stage([ok], [Placement(0, synth.IDENTITY, 7)], materials(), sky, Sun(), cam).build()
    bad = quad(1.0)
    bad.indices = np.array([0, 1, 9], np.uint32)
    with pytest.raises(TraceError, match="outside the vertex buffer"):
        Stage([bad], [], materials(), sky, Sun(), cam).build()
    short = quad(1.0)
    short.normals = short.normals[:3]
    with pytest.raises(TraceError, match="different vertex counts"):
        Stage([short], [], materials(), sky, Sun(), cam).build()
    with pytest.raises(TraceError, match="fraction from 0 to 1"):
        Stage([ok], [Placement(0, synth.IDENTITY, 0, alpha_cutoff=1.5)], materials(), sky, Sun(), cam).build()
    with pytest.raises(TraceError, match="invalid projection or lens"):
        Stage([ok], [], materials(), sky, Sun(), cam, projection=("orthographic", 0.0, 1.0)).build()
    with pytest.raises(TraceError, match="image-based skies"):
        Stage([ok], [], materials(), Sky(2, 1, np.array([[1, 1, 1, 1], [0, 0, 0, 1]], np.float32)), Sun(),
              cam).build()


def unit_triangle(alpha):
    """The triangle of stage.rs's own tests (stage.rs:865-880)."""
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    return Mesh(p, np.tile([0, 0, 1], (3, 1)).astype(np.float32), np.tile([1, 0, 0, 1], (3, 1)).astype(np.float32),
                np.array([[0, 0], [1, 0], [0, 1]], np.float32), np.array([0, 1, 2], np.uint32),
                alpha=None if alpha is None else np.asarray(alpha, np.float32))


def area(tri):
    a, b, c = tri["v"].astype(np.float64)
    e1, e2 = b - a, c - a
    return 0.5 * abs(e1[0] * e2[1] - e1[1] * e2[0])


def unit_stage(alphas_and_cutoffs):
    cam = synth.look_at((0, 0, 4), (0, 0, 0), 60, 1.0)
    meshes = [unit_triangle(a) for a, _ in alphas_and_cutoffs]
    placements = [Placement(i, synth.IDENTITY, 0, alpha_cutoff=c) for i, (_, c) in enumerate(alphas_and_cutoffs)]
    return Stage(meshes, placements, materials(), Sky(1, 1, np.ones((1, 4), np.float32)), Sun(), cam).build()


def test_alpha_below_the_cutoff_is_cut_away():
    """alpha_below_the_cutoff_is_cut_where_the_live_renderer_discards
    (stage.rs:910-933): kept triangle counts and areas, and uv = (x, y) at every
    kept corner."""
    cases = [([1.0, 1.0, 1.0], 1, 0.5), ([0.0, 0.0, 0.0], 0, 0.0), ([1.0, 0.0, 0.0], 1, 0.125),
             ([1.0, 1.0, 0.0], 2, 0.375)]
    for alpha, count, expected in cases:
        s = unit_stage([(alpha, 0.5)])
        kept = s.scene.meshes[0]
        assert len(kept) == count, alpha
        assert abs(sum(area(t) for t in kept) - expected) < 1e-6, alpha
        for t in kept:
            assert np.array_equal(t["v"][:, :2], t["uv"])


def test_one_mesh_keeps_a_polygon_for_each_cutoff():
    """one_mesh_keeps_a_polygon_for_each_cutoff (stage.rs:1161-1193): cutoffs
    0.25, 0.9 and the default 0.5 of one mesh give areas 0.28125, 0.005, 0.125."""
    s = unit_stage([([1.0, 0.0, 0.0], 0.25), ([1.0, 0.0, 0.0], 0.9), ([1.0, 0.0, 0.0], 0.5)])
    areas = [sum(area(t) for t in m) for m in s.scene.meshes]
    assert abs(areas[0] - 0.28125) < 1e-6 and abs(areas[1] - 0.005) < 1e-6 and abs(areas[2] - 0.125) < 1e-6


def test_instances_share_a_mesh_with_their_own_material_and_transform():
    """instances_share_a_mesh_with_their_own_material_and_transform (stage.rs:889-908)."""
    moved = np.eye(4, dtype=np.float32)
    moved[3] = [2.0, 0.0, -1.0, 1.0]
    cam = synth.look_at((0, 0, 4), (0, 0, 0), 60, 1.0)
    s = Stage([unit_triangle(None)], [Placement(0, synth.IDENTITY, 1), Placement(0, moved, 0)], materials(),
              Sky(1, 1, np.ones((1, 4), np.float32)), Sun(), cam).build()
    assert len(s.scene.triangles) == 0 and len(s.scene.materials) == 3
    meshes, inst = s.scene.meshes, s.scene.instances
    assert meshes[inst[0]["mesh"]]["material"][0] == 1 and meshes[inst[1]["mesh"]]["material"][0] == 0
    assert np.array_equal(meshes[inst[0]["mesh"]]["uv"][0], [[0, 0], [1, 0], [0, 1]])
    m = inst[1]["transform"].reshape(4, 4)  # column-major: row k of this array is column k
    v1 = meshes[inst[1]["mesh"]]["v"][0][1]
    assert np.array_equal(m[:3, :3].T @ v1 + m[3, :3], [3.0, 0.0, -1.0])


def test_a_cutoff_outside_zero_to_one_or_a_non_finite_clip_is_refused():
    """a_cutoff_outside_zero_to_one_or_a_non_finite_clip_is_refused (stage.rs:1195-1244)."""
    cam = synth.look_at((0, 0, 4), (0, 0, 0), 60, 1.0)
    sky = Sky(1, 1, np.ones((1, 4), np.float32))
    nan_clip = np.zeros((2, 4), np.float32)
    nan_clip[0, 0] = np.nan
    bad = [Placement(0, synth.IDENTITY, 0, alpha_cutoff=1.1), Placement(0, synth.IDENTITY, 0, alpha_cutoff=-0.01),
           Placement(0, synth.IDENTITY, 0, alpha_cutoff=float("nan")),
           Placement(0, synth.IDENTITY, 0, alpha_cutoff=float("inf")), Placement(0, synth.IDENTITY, 0, clip=nan_clip)]
    for p in bad:
        with pytest.raises(TraceError):
            Stage([unit_triangle(None)], [p], materials(), sky, Sun(), cam).build()
    for cutoff in (0.0, 1.0):
        Stage([unit_triangle(None)], [Placement(0, synth.IDENTITY, 0, alpha_cutoff=cutoff)], materials(), sky, Sun(),
              cam).build()
    spare = unit_triangle(None)
    spare.indices = np.array([0, 1, 3], np.uint32)
    with pytest.raises(TraceError, match="outside the vertex buffer"):
        Stage([unit_triangle(None), spare], [Placement(0, synth.IDENTITY, 0)], materials(), sky, Sun(), cam).build()
