"""The product's scene packing (pfxt_scene_build) against the oracle's own
restatement of SceneBuffers::build (oracle/pack.cpp): every blob byte for
byte.  The oracle restates gpu.rs:566-1061 with tree.rs:220-395 (light tree,
split with Rust's select_nth_unstable_by), levels.rs:225-470 (two levels),
lights.rs:182-243, 391-440 (light rows, emitter list), record.rs:57-180
(material records) and sky.rs:212-275 (sky CDF) without reading anything the
product built."""
import numpy as np
import pytest

import oracle
from pfx_b200 import abi, synth
from pfx_b200.trace import LIGHT, SceneBuffers, SceneDesc, Settings

BLOBS = ("nodes", "triangles", "uv", "surfaces", "materials", "emitters", "emitter_cdf", "lights")


def assert_same_buffers(scene, settings):
    mine = SceneBuffers(scene, settings)
    ref = oracle.scene_buffers(scene, settings)
    for name in BLOBS:
        a, b = mine.array(name), ref.array(name)
        assert len(a) == len(b), f"{name}: {len(a)} bytes against the oracle's {len(b)}"
        if not np.array_equal(a, b):
            words = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
            raise AssertionError(f"{name}: {len(words)} words differ, first at word {words[0]}")
    assert np.array_equal(mine.order(), ref.order())
    for x, y in zip(mine.sky(), ref.sky()):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert np.array_equal(mine.sobol().view(np.uint32), ref.sobol().view(np.uint32))
    for k in ("triangle_count", "emitter_count", "light_count", "sky_width", "sky_height", "sobol_length"):
        assert getattr(mine.buffers, k) == getattr(ref.buffers, k), k
    assert mine.builds()[0] == ref.buffers.bottom_builds
    return mine, ref


# ------------------------------------------------------------ selection
def product_select(keys, index, rounds=16):
    k = np.ascontiguousarray(keys, np.float32)
    out = np.zeros(len(k), np.uint32)
    abi.check(abi.load().pfxt_debug_select_nth(k.ctypes.data, len(k), index, rounds, out.ctypes.data))
    return out


def total_key(keys):
    i = np.ascontiguousarray(keys, np.float32).view(np.int32).astype(np.int64)
    return i ^ ((i >> 31) & 0x7fffffff)


@pytest.mark.parametrize("rounds", [16, 2, 0])
def test_the_selection_is_the_same_permutation_in_both_restatements(rounds):
    """slice::select_nth_unstable_by with f32::total_cmp, written twice (the
    tree builder's and the oracle's): the same permutation on random keys with
    many ties, signed zeros and every size class (insertion sort, median of 3,
    the recursive pseudo-median, the median-of-medians fallback), and the
    selection property: nothing before `index` is greater, nothing after is
    less."""
    rng = np.random.default_rng(7 + rounds)
    sizes = list(range(1, 40)) + [63, 64, 65, 127, 128, 200, 513, 1000, 1024, 1025, 4097]
    for n in sizes:
        for kind in range(4):
            if kind == 0:
                keys = rng.normal(size=n).astype(np.float32)
            elif kind == 1:  # few distinct values: the equal-to-ancestor branch
                keys = rng.integers(0, 4, n).astype(np.float32)
            elif kind == 2:  # signed zeros and repeats
                keys = rng.choice(np.array([-0.0, 0.0, 1.0, -1.0], np.float32), n)
            else:  # sorted and reversed runs
                keys = np.sort(rng.normal(size=n)).astype(np.float32)
                if n % 2:
                    keys = keys[::-1].copy()
            for index in {0, n - 1, n // 2, int(rng.integers(0, n))}:
                a = product_select(keys, index, rounds)
                b = oracle.select_nth(keys, index, rounds)
                assert np.array_equal(a, b), (n, kind, index)
                assert sorted(a.tolist()) == list(range(n))
                t = total_key(keys[a])
                assert (t[:index] <= t[index]).all() and (t[index + 1:] >= t[index]).all()


# ------------------------------------------------------------ scenes
def street(count):
    """tree.rs:401-416: points on both sides of a street, every third a spot."""
    out = []
    for k in range(count):
        side = -6.0 if k % 2 == 0 else 6.0
        if k % 3 == 0:
            out.append(synth.spot_light((side, 5.0, k * 4.0), (0.0, -1.0, 0.0), 40.0, 50.0, 30.0,
                                        (1.0, 0.8, 0.6), rng_range=18.0))
        else:
            out.append(synth.point_light((side, 5.0, k * 4.0), 40.0, (1.0, 0.8, 0.6), rng_range=18.0))
    return np.concatenate(out)


def test_street_lights_through_the_tree_equal_the_oracle():
    # every_light_sits_in_exactly_one_leaf's street scenes (tree.rs:433-444),
    # with three looped rect lights before the tree's
    ground = synth.quad((0, 0, 0), (50, 0, 0), (0, 0, 50))
    looped = np.concatenate([synth.rect_light((0, 8, z), (1, 0, 0), (0, 0, 1), 5.0) for z in (0, 40, 80)])
    for count in (5, 32, 128, 1024):
        scene = SceneDesc(ground, synth.material(), synth.look_at((0, 5, -10), (0, 5, 0), 45, 1.0),
                          lights=np.concatenate([looped, street(count)]))
        mine, _ = assert_same_buffers(scene, Settings(sampler="pcg"))
        rows = mine.array("lights").view(np.float32).reshape(-1, 16)
        assert len(rows) > 3 + count  # the tree's nodes follow its lights


def test_the_sphere_cloud_equals_the_oracle():
    w = synth.plain_512()
    assert_same_buffers(w.scene, w.settings)


def test_emissive_world_triangles_and_a_sky_equal_the_oracle():
    w = synth.plain_512(sampler="pcg")
    mats = w.scene.materials.copy()
    mats["emission"][5] = (4.0, 3.0, 2.0)
    mats["emission"][9] = (0.5, 2.0, 6.0)
    w.scene.materials = mats
    w.scene.sky = (0.3, 0.4, 0.5)
    mine, _ = assert_same_buffers(w.scene, w.settings)
    assert mine.buffers.emitter_count > 100


@pytest.mark.parametrize("world", [False, True])
@pytest.mark.parametrize("moved", [False, True])
def test_the_instanced_stage_equals_the_oracle(world, moved):
    # an emissive panel instance (its own emitters), shared ball meshes, a sun
    w = synth.staged(synth.staged_poses(moved), world=world, empty=True)
    mine, _ = assert_same_buffers(w.scene, w.settings)
    assert mine.buffers.emitter_count == 2


def test_the_full_instanced_scene_equals_the_oracle():
    w = synth.instanced_1080()
    assert w.scene.world_triangle_count > 200_000
    assert_same_buffers(w.scene, w.settings)


def test_the_full_4k_room_equals_the_oracle():
    w = synth.room_4k()
    mine, _ = assert_same_buffers(w.scene, w.settings)
    assert mine.buffers.light_count == 128


def test_no_lights_and_no_emitters_equal_the_oracle():
    # the empty emitter list's header (lights.rs:510-516): its total is the
    # empty f64 sum, -0.0
    tris = synth.quad((0, 0, 0), (1, 0, 0), (0, 0, 1))
    scene = SceneDesc(tris, synth.material(), synth.look_at((0, 1, 3), (0, 0, 0), 45, 1.0),
                      lights=np.zeros(0, LIGHT))
    mine, _ = assert_same_buffers(scene, Settings())
    head = mine.array("emitters").view(np.float32)[:4]
    assert head[0] == 0.0 and np.signbit(head[2])
