"""Accuracy of the transcendentals that the kernels and the oracle share
(pfx_b200/csrc/pfxt_math.h), measured on the oracle's CPU build against FP64
references: a few ulp of the float32 result, and absolute error where the
result passes through zero (sin, cos near their roots; log near 1)."""
import numpy as np
import pytest

import oracle


def ulp_error(got, want):
    got = got.astype(np.float64)
    want32 = want.astype(np.float32)
    ulp = np.spacing(np.abs(want32)).astype(np.float64)
    return np.abs(got - want) / ulp


RNG = np.random.default_rng(12)


@pytest.mark.parametrize("fn,ref,lo,hi", [
    ("sin", np.sin, -100.0, 100.0),
    ("cos", np.cos, -100.0, 100.0),
    ("asin", np.arcsin, -1.0, 1.0),
    ("acos", np.arccos, -1.0, 1.0),
    ("exp", np.exp, -80.0, 80.0),
    ("log", np.log, 1e-30, 1e30),
])
def test_unary_functions_within_a_few_ulp(fn, ref, lo, hi):
    if fn == "log":
        x = np.exp(RNG.uniform(np.log(lo), np.log(hi), 200_000)).astype(np.float32)
    else:
        x = RNG.uniform(lo, hi, 200_000).astype(np.float32)
    got = oracle.math(fn, x)
    want = ref(x.astype(np.float64))
    err = ulp_error(got, want)
    if fn in ("sin", "cos"):
        # near the roots the float32 argument's own rounding dominates: absolute bound
        ok = (err <= 4) | (np.abs(got - want) <= 2e-7 * np.maximum(1.0, np.abs(x)))
    elif fn == "log":
        ok = (err <= 4) | (np.abs(got - want) <= 1e-7)
    else:
        ok = err <= 4
    assert ok.mean() == 1.0, (fn, float(err.max()), x[~ok][:4])


def test_atan2_all_quadrants():
    y = RNG.uniform(-10, 10, 200_000).astype(np.float32)
    x = RNG.uniform(-10, 10, 200_000).astype(np.float32)
    got = oracle.math("atan2", y, x).astype(np.float64)
    want = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    assert np.max(np.abs(got - want)) < 4e-7
    assert oracle.math("atan2", np.float32([0.0]), np.float32([1.0]))[0] == 0.0


def test_pow_on_shading_ranges():
    x = RNG.uniform(0.0, 1.0, 100_000).astype(np.float32)
    y = RNG.uniform(0.5, 5.0, 100_000).astype(np.float32)  # Schlick powers and the like
    got = oracle.math("pow", x, y).astype(np.float64)
    want = np.power(x.astype(np.float64), y.astype(np.float64))
    assert np.max(np.abs(got - want) / np.maximum(want, 1e-30)) < 8 * 2.0 ** -23 or \
        np.max(np.abs(got - want)) < 1e-6


def test_special_values():
    assert oracle.math("exp", np.float32([0.0]))[0] == 1.0
    assert oracle.math("log", np.float32([1.0]))[0] == 0.0
    assert oracle.math("cos", np.float32([0.0]))[0] == 1.0
    assert oracle.math("sin", np.float32([0.0]))[0] == 0.0
    assert abs(oracle.math("acos", np.float32([-1.0]))[0] - np.pi) < 4e-7
