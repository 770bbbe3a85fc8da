"""The radiance cache's tensor-core kernels against the FP64 oracle
(oracle/cache.py): inference, the gradients of the relative L2 loss (MLP
weights and hash table), one Adam step, and that online training learns.

The CUDA path computes with BF16 operands and FP32 accumulation; the oracle
rounds at the same places and accumulates in FP64, so the two differ by FP32
summation order (and the rare BF16 rounding flip that causes).  Tolerances:
normwise relative error 5e-3 for outputs, 1e-2 for gradients and updates."""
import numpy as np
import pytest

import oracle.cache as oc
from pfx_b200.cache import CacheSettings, RadianceCache, RECORD, random_queries

pytestmark = pytest.mark.gpu

SMALL = CacheSettings(log2_entries=12, base_resolution=4, max_resolution=256, batch=1024, steps=1, seed=3,
                      lo=(-1.0, -2.0, -3.0), hi=(2.0, 1.0, 4.0))
# the bench's cache: 2^19 entries per level, resolutions 16..2048 (hashed fine
# levels), with a smaller batch so the FP64 oracle finishes in seconds
FULL = CacheSettings(log2_entries=19, base_resolution=16, max_resolution=2048, batch=2048, steps=1, seed=4,
                     lo=(-15.0, 0.0, -15.0), hi=(15.0, 10.0, 15.0))
CONFIGS = pytest.mark.parametrize("settings", [SMALL, FULL], ids=["reduced", "bench"])


def make(settings, table_scale=1.0, seed=5):
    c = RadianceCache(settings)
    scales, res, dense = c.encoding()
    enc = oc.Encoding(scales, res, dense, settings.entries, settings.lo, settings.hi)
    rng = np.random.default_rng(seed)
    mlp, table = c.params()
    table = rng.uniform(-table_scale, table_scale, table.shape).astype(np.float32)
    c.set_params(table=table)
    return c, enc, mlp, table, rng


def records(rng, n, settings):
    r = np.zeros(n, RECORD)
    r["query"] = random_queries(n, rng, settings.lo, settings.hi)
    r["target"] = rng.uniform(0.0, 2.0, (n, 3)).astype(np.float32)
    r["weight"] = 1.0
    return r


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_encoding_geometry(gpu):
    c = RadianceCache(SMALL)
    scales, res, dense = c.encoding()
    assert np.all(np.diff(scales) > 0)
    assert abs(scales[0] - (SMALL.base_resolution - 1)) < 1e-4
    assert abs(scales[-1] - (SMALL.max_resolution - 1)) < 1e-2
    for l in range(16):
        assert bool((dense >> l) & 1) == (int(res[l]) ** 3 <= SMALL.entries)
    assert dense & 1 and not (dense >> 15) & 1  # both kinds of level are exercised


@CONFIGS
def test_inference_matches_oracle(gpu, settings):
    c, enc, mlp, table, rng = make(settings)
    q = random_queries(3000, rng, settings.lo, settings.hi)  # a ragged last tile
    got = c.infer(q)
    want = oc.infer(mlp, table, enc, q)
    assert np.isfinite(got).all()
    assert rel(got, want) < 5e-3, rel(got, want)
    # a query outside the bounds is clamped onto the grid, not rejected
    q2 = q[:4].copy()
    q2["position"] = np.float32(1e6)
    assert np.isfinite(c.infer(q2)).all()


@CONFIGS
def test_gradients_match_oracle(gpu, settings):
    c, enc, mlp, table, rng = make(settings)
    r = records(rng, 2048, settings)
    g_mlp, g_tab, loss = c.gradients(r)
    w_mlp, w_tab, w_loss = oc.gradients(mlp, table, enc, r)
    assert abs(loss - w_loss) <= 1e-3 * w_loss
    for name, lo, hi in (("W1", oc.W1, oc.W2), ("W2", oc.W2, oc.W3), ("W3", oc.W3, oc.MLP_PARAMS)):
        e = rel(g_mlp[lo:hi], w_mlp[lo:hi])
        assert e < 1e-2, (name, e)
    assert np.all(g_mlp[oc.W3 + 3 * 64:] == 0.0)  # padded output rows get no gradient
    e = rel(g_tab, w_tab)
    assert e < 1e-2, e
    # entries no record touches stay exactly zero
    assert np.all(g_tab[w_tab == 0.0] == 0.0)


@CONFIGS
def test_adam_step_matches_oracle(gpu, settings):
    s = CacheSettings(**{**settings.__dict__, "epsilon": 1e-4, "learning_rate": 1e-3})
    c, enc, mlp, table, rng = make(s)
    r = records(rng, s.batch, s)
    c.train(r)
    mlp1, table1 = c.params()
    g_mlp, g_tab, _ = oc.gradients(mlp, table, enc, r)
    b = (s.beta1, s.beta2)
    p_mlp, _, _ = oc.adam(mlp, np.zeros_like(g_mlp), np.zeros_like(g_mlp), g_mlp, 1, b, s.learning_rate, s.beta1,
                          s.beta2, s.epsilon)
    p_tab, _, _ = oc.adam(table.reshape(-1), np.zeros(table.size), np.zeros(table.size), g_tab.reshape(-1), 1, b,
                          s.learning_rate, s.beta1, s.beta2, s.epsilon)
    e_mlp = rel(mlp1 - mlp, p_mlp - mlp)
    e_tab = rel(table1.reshape(-1) - table.reshape(-1), p_tab - table.reshape(-1))
    assert e_mlp < 1e-2 and e_tab < 1e-2, (e_mlp, e_tab)
    assert c.stats()["steps"] == 1


def test_training_learns_a_radiance_field(gpu):
    s = CacheSettings(log2_entries=16, base_resolution=8, max_resolution=512, batch=4096, steps=1, seed=9,
                      learning_rate=1e-2)
    c = RadianceCache(s)
    rng = np.random.default_rng(11)

    def field(q):
        p = q["position"].astype(np.float64)
        d = q["direction"].astype(np.float64)
        base = 0.6 + 0.4 * np.sin(6.0 * p[:, 0]) * np.cos(4.0 * p[:, 1]) + 0.3 * p[:, 2]
        lobe = 0.5 * np.maximum(d[:, 1], 0.0) ** 2
        return ((base + lobe)[:, None] * (0.3 + q["diffuse"])).astype(np.float32)

    q = random_queries(4096, rng)
    want = field(q)

    def held_out_error():
        got = c.infer(q)
        return float(np.mean((got - want) ** 2 / (want ** 2 + 0.01)))

    before = held_out_error()
    losses = []
    for step in range(120):
        r = np.zeros(s.batch, RECORD)
        r["query"] = random_queries(s.batch, rng)
        r["target"] = field(r["query"])
        r["weight"] = 1.0
        losses.append(c.train(r))
    after = held_out_error()
    assert losses[-1] < 0.2 * losses[0], (losses[0], losses[-1])
    assert after < 0.2 * before, (before, after)


def test_a_wait_that_runs_out_is_reported_and_the_cache_stays_usable(gpu):
    """A kernel's wait for its tensor-core work gives up after a bounded number
    of polls; with the limit at 0 every wait gives up at once.  The call then
    fails with the cache's error (after the kernel drained the MMAs it issued
    and freed its tensor memory), and with the limit restored the same cache
    gives the same answers as before."""
    from pfx_b200.abi import TraceError
    c, enc, mlp, table, rng = make(SMALL)
    q = random_queries(512, rng, SMALL.lo, SMALL.hi)
    r = records(rng, SMALL.batch, SMALL)
    before = c.infer(q)
    g_before = c.gradients(r[:512])[0]
    c.set_wait_limit(0)
    with pytest.raises(TraceError, match="ran out of its limit"):
        c.infer(q)
    with pytest.raises(TraceError, match="ran out of its limit"):
        c.gradients(r[:512])
    c.set_wait_limit(1 << 22)
    assert np.array_equal(c.infer(q), before)
    assert rel(c.gradients(r[:512])[0], g_before) < 1e-6
    assert c.stats()["steps"] == 0
