"""The CPU oracle against the reference's own known answers (tests/golden)."""
import json
from pathlib import Path

import numpy as np

import oracle
from pfx_b200 import synth

KAT = json.loads((Path(__file__).parent / "golden" / "reference_kat.json").read_text())


def test_bvh_matches_brute_force_on_the_lcg_fixture():
    # bvh.rs:330-381: build twice (same bytes), then 2000 rays agree with brute force
    verts, rays = synth.lcg_triangles()
    assert len(verts) == KAT["bvh_lcg"]["triangles"] and len(rays) == KAT["bvh_lcg"]["rays"]
    nodes, order = oracle.bvh_build(verts)
    nodes2, order2 = oracle.bvh_build(verts)
    assert np.array_equal(nodes, nodes2) and np.array_equal(order, order2)
    hits = 0
    for o, d in rays:
        fast = oracle.bvh_intersect(nodes, order, verts, o, d)
        brute = oracle.brute_intersect(verts, o, d)
        assert fast == brute
        hits += fast >= 0
    assert hits > 50  # the fixture does hit things


def test_hash_known_answers():
    for kx, ky, want in KAT["hash_uint2"]["cases"]:
        assert oracle.hash_uint2(kx, ky) == int(want, 16)
    for seed, frame, want in KAT["animated_seed"]["cases"]:
        assert oracle.animated_seed(seed, frame) == int(want, 16)
    assert len({oracle.animated_seed(7, f) for f in range(240)}) == KAT["animated_seed"]["distinct_frames"]


def test_sequence_size():
    for samples, want in KAT["sequence_size"]["cases"]:
        assert oracle.sequence_size(samples) == want


def test_sobol_patterns_are_deterministic_and_stratified():
    a = oracle.generate_4d(256, 37)
    b = oracle.generate_4d(256, 37)
    assert np.array_equal(a, b)
    assert np.all((a >= 0.0) & (a < 1.0))
    pts = oracle.generate_4d(1024, 5)
    for n in KAT["sobol_table"]["stratified_prefixes"]:
        for axis in range(4):
            cells = (pts[:n, axis] * np.float32(n)).astype(np.int64)
            assert len(set(cells.tolist())) == n, (n, axis)


def test_automatic_min_samples():
    for threshold, want in KAT["automatic_min_samples"]["cases"]:
        assert oracle.automatic_min_samples(threshold) == want


def test_half_buffer_error():
    k = KAT["adaptive_error"]
    even, odd = np.float32(k["even"]), np.float32(k["odd"])
    allv = (even + odd) * np.float32(0.5)
    got = oracle.adaptive_error(even, 64.0, allv, 128.0)
    diff = np.abs(even[:3] - odd[:3]).sum() * 0.5
    want = diff / (1e-4 + np.sqrt(allv[:3].sum()))
    assert abs(got - want) < 1e-6
    assert oracle.adaptive_error(even, 0.0, allv, 8.0) == k["zero_prior"]
    v, pc, c, want = k["flat"]
    assert oracle.adaptive_error([v] * 4, pc, [v] * 4, c) == want


def test_falloff_known_answer():
    # lights.rs:585-586
    got = oracle.falloff(4.0, 0.0, 10.0, 2.0)
    want = 4.0 * (1.0 - 0.2 ** 4) ** 2 / 4.0
    assert abs(got - want) < 1e-6
    assert oracle.falloff(4.0, 0.0, 10.0, 10.0) == 0.0


def test_kernel_division_is_ieee_division():
    # the slab quotients of the kernels use div_rn (Markstein's correction);
    # it must round exactly like the reference's division
    assert oracle.check_div(1_500_000, seed=7) == 0
