"""The product's host-side scene packing (SceneBuffers::build restated in
pfx_b200/csrc/build.cpp) against the oracle and the reference's own tests."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from pfx_b200 import abi, synth
from pfx_b200.trace import LIGHT, SceneBuffers, SceneDesc, Settings

KAT = json.loads((Path(__file__).parent / "golden" / "reference_kat.json").read_text())
NODE = np.dtype([("lo", "<f4", 4), ("hi", "<f4", 4), ("first", "<u4"), ("count", "<u4"), ("pad", "<u4", 2)])
LROW = np.dtype([("a", "<f4", 4), ("b", "<f4", 4), ("c", "<f4", 4), ("d", "<f4", 4)])


def scene_of(tris, lights=None, **kw):
    mats = np.concatenate([synth.material()] * (int(tris["material"].max()) + 1))
    return SceneDesc(tris, mats, synth.look_at((0, 0, 10), (0, 0, 0), 45, 1.0),
                     lights=lights if lights is not None else np.zeros(0, LIGHT), **kw)


def test_world_bvh_equals_the_oracle_build_on_the_lcg_fixture():
    verts, _ = synth.lcg_triangles()
    tris = synth.triangles(verts)
    sb = SceneBuffers(scene_of(tris), Settings())
    nodes, order = oracle.bvh_build(verts)
    assert np.array_equal(sb.array("nodes"), nodes)
    assert np.array_equal(sb.order(), order)
    # triangles are stored in slot (BVH) order, 96 bytes each (gpu.rs:765-780)
    packed = sb.array("triangles").view(np.float32).reshape(-1, 24)
    assert np.array_equal(packed[:, 0:3], verts[order][:, 0])
    assert np.array_equal(packed[:, 4:7], verts[order][:, 1])


def test_world_bvh_equals_the_oracle_build_on_the_sphere_scene():
    w = synth.plain_512()
    sb = SceneBuffers(w.scene, w.settings)
    nodes, order = oracle.bvh_build(w.scene.triangles["v"])
    assert np.array_equal(sb.array("nodes"), nodes)
    assert np.array_equal(sb.order(), order)


def test_world_bvh_equals_the_oracle_build_on_the_full_4k_room():
    # the bench's scene: 1.19 M world triangles, every node and slot
    w = synth.room_4k()
    assert len(w.scene.triangles) > 1_000_000
    sb = SceneBuffers(w.scene, w.settings)
    nodes, order = oracle.bvh_build(w.scene.triangles["v"])
    assert np.array_equal(sb.array("nodes"), nodes)
    assert np.array_equal(sb.order(), order)


def test_two_level_layout():
    # levels.rs:393-470: top tree of 2g-1 nodes, g inverse-row nodes, then the
    # world BVH and one BVH per distinct mesh; instance leaves carry the mesh
    # root, the slot base, the record and the inverse rows.
    w = synth.instanced_1080(target=20_000)
    sb = SceneBuffers(w.scene, w.settings)
    nodes = sb.array("nodes").view(NODE)
    inst = w.scene.instances
    g = 1 + len(inst)
    leaves = nodes[: 2 * g - 1][nodes[: 2 * g - 1]["pad"][:, 0] == 1]
    assert len(leaves) == g
    records = sorted(int(x) for x in leaves["lo"][:, 3].view(np.uint32))
    assert records == list(range(g))
    # two distinct meshes -> two bottom-level trees; slots = world + cube + icosphere
    assert sb.buffers.triangle_count == 2 + 12 + 1280
    # inverse rows of an instance invert its transform
    for leaf in leaves:
        rec = int(np.array(leaf["lo"][3], np.float32).view(np.uint32))
        if rec == 0:
            assert leaf["pad"][1] == 0
            continue
        rows = nodes[leaf["pad"][1]]
        inv = np.stack([rows["lo"], rows["hi"], np.array([rows["first"], rows["count"], *rows["pad"]],
                                                         np.uint32).view(np.float32)])
        m = inst[rec - 1]["transform"].reshape(4, 4).T.astype(np.float64)
        prod = inv.astype(np.float64) @ m
        assert np.allclose(prod[:, :3], np.eye(3), atol=1e-4)


def street(count):
    # tree.rs:401-417
    out = []
    for k in range(count):
        side = -6.0 if k % 2 == 0 else 6.0
        if k % 3 == 0:
            out.append(synth.spot_light((side, 5.0, k * 4.0), (0.0, -1.0, 0.0), 40.0, 50.0, 30.0,
                                        (1.0, 0.8, 0.6), rng_range=18.0))
        else:
            out.append(synth.point_light((side, 5.0, k * 4.0), 40.0, (1.0, 0.8, 0.6), rng_range=18.0))
    return np.concatenate(out)


def leaves_of(rows, base, count, at, seen):
    node = rows[at]
    n, link = int(node["d"][1]), int(node["d"][2])
    if n == 0:
        leaves_of(rows, base, count, at + 1, seen)
        leaves_of(rows, base, count, link, seen)
    else:
        assert n <= 8
        seen.extend(range(link, link + n))


@pytest.mark.parametrize("count", KAT["tree_counts"]["counts"])
def test_every_light_sits_in_exactly_one_leaf(count):
    base = KAT["tree_counts"]["base"]
    looped = np.concatenate([synth.rect_light((0, 9, k), (0.5, 0, 0), (0, 0, 0.5), 1.0) for k in range(base)])
    lights = np.concatenate([looped, street(count)])
    sb = SceneBuffers(scene_of(synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1)), lights), Settings())
    rows = sb.array("lights").view(LROW)
    head = sb.array("emitters").view(np.float32)[:4]
    assert head[1] == base and head[3] == count
    seen = []
    leaves_of(rows, base, count, base + count, seen)
    assert sorted(seen) == list(range(base, base + count))
    # each tree row is a packed copy of a distinct input light
    pos = {tuple(p) for p in rows[base:base + count]["a"][:, :3].tolist()}
    assert len(pos) == count
    assert len(rows) - base - count < 2 * count


def test_a_node_bounds_its_lights_energy_and_reach():
    lights = street(128)
    sb = SceneBuffers(scene_of(synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1)), lights), Settings())
    rows = sb.array("lights").view(LROW)
    root = rows[128]
    energy = float(sum(lights["colour"][i].sum() * lights["intensity"][i] / 3.0 for i in range(128)))
    assert abs(root["a"][3] - energy) <= energy * 1e-5
    assert root["b"][3] == 18.0
    pos = lights["position"]
    assert np.all(root["a"][:3] <= pos) and np.all(pos <= root["b"][:3])
    # merged cones hold every spot axis (tree.rs:475-492 as a property of the root)
    axis = root["c"][:3].astype(np.float64)
    for i in range(128):
        if lights["shape"][i] == abi.LIGHT_SPOT:
            d = lights["direction"][i] / np.linalg.norm(lights["direction"][i])
            ang = math.acos(max(-1.0, min(1.0, float(np.dot(axis, d)))))
            assert ang <= root["c"][3] + 1e-4


def test_few_lights_keep_their_order_and_their_own_slots():
    looped = KAT["tree_looped"]["looped"]
    sb = SceneBuffers(scene_of(synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1)), street(looped)), Settings())
    head = sb.array("emitters").view(np.float32)[:4]
    assert (head[1], head[3]) == (looped, 0)
    assert len(sb.array("lights")) // 64 == looped
    sb = SceneBuffers(scene_of(synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1)), street(looped + 1)), Settings())
    head = sb.array("emitters").view(np.float32)[:4]
    assert (head[1], head[3]) == (0, looped + 1)


def test_lights_pack():
    k = KAT["light_pack"]
    point = synth.point_light((0.0, 2.0, 0.0), 4.0, (1.0, 0.5, 0.25), rng_range=10.0)
    rect = synth.rect_light((0.0, 2.0, 0.0), (0.5, 0.0, 0.0), (0.0, 0.0, 0.25), 1.0)
    rect["intensity"] = 2.0
    sb = SceneBuffers(scene_of(synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1)), np.concatenate([point, rect])),
                      Settings())
    rows = sb.array("lights").view(LROW)
    assert list(rows[0]["b"]) == k["point_b"]
    assert rows[0]["d"][3] == 1.0
    assert list(rows[1]["b"][:3]) == k["rect_b"]


def test_emitters_are_weighted_by_power():
    # lights.rs:465-507 through the scene packing: two quads of emissive
    # triangles (unit quad, emission 1; 2x2 quad, emission 0.5)
    k = KAT["emitters"]
    q1 = synth.quad((0.5, 2.0, 0.5), (0.5, 0, 0), (0, 0, 0.5), material=1)
    q2 = synth.quad((1.0, 5.0, 1.0), (1.0, 0, 0), (0, 0, 1.0), material=2)
    tris = np.concatenate([synth.quad((0, 0, 0), (5, 0, 0), (0, 0, 5), 0), q1, q2])
    mats = np.concatenate([synth.material(), synth.material(emission=(1, 1, 1)), synth.material(emission=(.5, .5, .5))])
    scene = SceneDesc(tris, mats, synth.look_at((0, 0, 10), (0, 0, 0), 45, 1.0),
                      lights=synth.point_light((0, 9, 0), 1.0))
    sb = SceneBuffers(scene, Settings())
    e = sb.array("emitters").view(np.float32).reshape(-1, 16)
    assert e[0, 0] == 4.0 and e[0, 1] == 1.0
    assert abs(e[0, 2] - k["total"]) < 1e-5
    probs = sorted(e[1:, 15].tolist())
    assert np.allclose(probs, sorted(k["probabilities"]), atol=1e-6)
    cdf = sb.array("emitter_cdf").view(np.float32)
    assert len(cdf) == 4 and cdf[-1] == 1.0
    assert np.allclose(cdf, np.cumsum(e[1:, 15]), atol=1e-6)
    # each emissive slot carries its 1-based emitter index in c.w
    tri = sb.array("triangles").view(np.float32).reshape(-1, 24)
    assert sorted(tri[:, 11].tolist()) == [0.0, 0.0, 1.0, 2.0, 3.0, 4.0]


def test_sobol_table_equals_the_oracle_patterns():
    w = synth.plain_512()
    sb = SceneBuffers(w.scene, Settings(sampler="sobol", sobol_samples=16))
    table = sb.sobol()
    assert table.shape == (256 * 256, 4)
    for pattern in (0, 37, 255):
        assert np.array_equal(table[pattern * 256:(pattern + 1) * 256], oracle.generate_4d(256, pattern))
    assert SceneBuffers(w.scene, Settings(sampler="sobol", sobol_samples=300)).buffers.sobol_length == 512
    assert SceneBuffers(w.scene, Settings(sampler="pcg")).buffers.sobol == None  # noqa: E711


def test_black_sky_cdf_is_uniform():
    w = synth.plain_512()
    sb = SceneBuffers(w.scene, w.settings)
    rows, cols = sb.sky()
    assert len(rows) == 128 and len(cols) == 256 * 128
    assert np.array_equal(rows, (np.arange(128, dtype=np.float32) + 1) / np.float32(128))
    assert np.array_equal(cols[:256], (np.arange(256, dtype=np.float32) + 1) / np.float32(256))


def test_two_levels_find_the_hits_of_the_flattened_triangles():
    """two_levels_find_the_hits_of_the_flattened_triangles (levels.rs:591-680):
    a world blob, one mesh placed twice, a mesh of its own and a copy of the
    shared mesh's triangles: three bottom-level builds (the copy shares the
    shared mesh's by geometry), 130 slots, and the two-level walk (the oracle's
    restatement of scene()) finds the nearest hit that brute force over the
    flattened, transformed triangles finds."""
    from pfx_b200.trace import INSTANCE, TRIANGLE, Camera, make_rays

    state = [29]

    def random():
        state[0] = (state[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return np.float32(state[0] >> 8) / np.float32(1 << 24)

    def blob(count):
        v = np.zeros((count, 3, 3), np.float32)
        for i in range(count):
            x, y, z = (random() * np.float32(2) - np.float32(1) for _ in range(3))
            v[i, 0] = (x, y, z)
            v[i, 1] = (x + random() * np.float32(0.4) + np.float32(0.05), y, z)
            v[i, 2] = (x, y + random() * np.float32(0.4) + np.float32(0.05), z + np.float32(0.1))
        return synth.triangles(v, np.tile(np.array([0, 0, 1], np.float32), (count, 3, 1)))

    shared = blob(60)
    world = blob(30)
    poses = [synth.placed((2.0, 0.0, 0.0), 0.3, 1.0), synth.placed((-2.0, 0.5, 1.0), -1.2, 0.7),
             synth.placed((0.0, -2.0, -1.0), 2.0, 1.5), synth.placed((1.0, 1.5, -2.0), 2.5, 0.5)]
    own = blob(40)
    meshes = [shared, own, shared.copy()]
    inst = np.zeros(4, INSTANCE)
    inst["mesh"] = [0, 0, 1, 2]
    inst["two_sided"] = 1
    inst["casts_shadow"] = 1
    inst["transform"] = np.stack([p.reshape(16) for p in poses])
    cam = Camera((0.0, 0.0, 5.0), (0.0, 0.0, -1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    scene = SceneDesc(world, synth.material(), cam, meshes=meshes, instances=inst)
    sb = SceneBuffers(scene, Settings())
    assert sb.builds()[0] == 3
    assert sb.buffers.triangle_count == 30 + 60 + 40

    flat = [world["v"].astype(np.float64)]
    for k, mesh in enumerate([shared, shared, own, shared]):
        m = poses[k].astype(np.float64)  # column-major rows: point' = p @ M[:3,:3] + M[3,:3]
        flat.append(mesh["v"].astype(np.float64) @ m[:3, :3] + m[3, :3])
    tris = np.concatenate(flat)
    origins, dirs = [], []
    for _ in range(3000):
        origins.append([random() * np.float32(10) - np.float32(5) for _ in range(3)])
        d = np.array([random() * np.float32(2) - np.float32(1) for _ in range(3)], np.float32)
        dirs.append(d / np.float32(np.sqrt(np.float32((d * d).sum()))))
    o, d = np.array(origins, np.float32), np.array(dirs, np.float32)
    got = oracle.trace(sb, make_rays(o, d, 1e20))

    a, e1, e2 = tris[:, 0], tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0]
    for i in range(len(o)):
        pv = np.cross(d[i].astype(np.float64), e2)
        det = (e1 * pv).sum(1)
        ok = np.abs(det) > 1e-12
        inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        sv = o[i].astype(np.float64) - a
        u = (sv * pv).sum(1) * inv
        qv = np.cross(sv, e1)
        v = (d[i].astype(np.float64) * qv).sum(1) * inv
        t = (e2 * qv).sum(1) * inv
        hit = ok & (u >= 0) & (u <= 1) & (v >= 0) & (u + v <= 1) & (t > 1e-4)
        if not hit.any():
            assert got["hit"][i] == 0, i
            continue
        brute = t[hit].min()
        assert got["hit"][i] == 1, i
        assert abs(float(got["t"][i]) - brute) <= 1e-4 * max(brute, 1.0), (i, got["t"][i], brute)


def test_an_empty_emitter_list_keeps_its_header():
    """empty_list_keeps_its_header (lights.rs:510-516) through the scene packing:
    two looped lights and no emissive triangle leave one header entry
    (0 emitters, 2 looped lights) and no CDF."""
    lights = np.concatenate([synth.point_light((0, 2, 0), 1.0), synth.point_light((1, 2, 0), 1.0)])
    sb = SceneBuffers(scene_of(synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1)), lights), Settings())
    e = sb.array("emitters").view(np.float32).reshape(-1, 16)
    assert len(e) == 1 and list(e[0, :2]) == [0.0, 2.0]
    assert len(sb.array("emitter_cdf")) == 0


@pytest.mark.parametrize("emission, emits", [((0.0, 0.0, 1.0), True), ((0.0, 0.0, 0.0), False),
                                             ((1.0, -0.5, 1.0), False), ((float("nan"), 1.0, 1.0), False)])
def test_only_positive_emission_emits(emission, emits):
    """only_positive_emission_emits (lights.rs:518-524): a triangle becomes an
    emitter only when no channel of its emission is negative or NaN and some
    channel is positive."""
    tris = synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1), 0)
    scene = SceneDesc(tris, synth.material(emission=emission), synth.look_at((0, 0, 10), (0, 0, 0), 45, 1.0))
    sb = SceneBuffers(scene, Settings())
    assert (sb.buffers.emitter_count == 2) == emits


def test_a_uniform_sky_cdf_sums_to_one():
    """cdf_sums_to_one (sky.rs:505-529) for the uniform skies this tracer takes:
    every row and column mass is non-negative, the masses sum to one and the
    last row CDF value is one."""
    w = synth.staged(synth.staged_poses(False))  # sky (0.08, 0.09, 0.1)
    sb = SceneBuffers(w.scene, w.settings)
    rows, cols = sb.sky()
    h, wdt = len(rows), len(cols) // len(rows)
    row_mass = np.diff(np.concatenate([[0.0], rows.astype(np.float64)]))
    col = cols.astype(np.float64).reshape(h, wdt)
    col_mass = np.diff(np.concatenate([np.zeros((h, 1)), col], 1), axis=1)
    assert np.all(row_mass >= -1e-5) and np.all(col_mass >= -1e-5)
    assert abs((row_mass[:, None] * col_mass).sum() - 1.0) < 1e-4
    assert abs(rows[-1] - 1.0) < 1e-6
