"""The radiance-cache oracle (oracle/cache.py) pinned on the CPU: its backward
pass against PyTorch autograd in FP64 (rounding off), its encoding against
the published hash-grid definition, and the C ABI's settings validation."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle.cache as oc
from pfx_b200 import abi
from pfx_b200.cache import QUERY, RECORD, CacheSettings, random_queries


def encoding(log2=10, base=4, maximum=64, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    T = 1 << log2
    growth = np.exp(np.log(maximum / base) / 15)
    scales = np.array([base * growth ** l - 1 for l in range(16)], np.float32)
    res = np.ceil(scales.astype(np.float64)).astype(np.uint32) + 2
    dense = sum(1 << l for l in range(16) if int(res[l]) ** 3 <= T)
    return oc.Encoding(scales, res, dense, T, lo, hi)


def test_backward_matches_autograd():
    rng = np.random.default_rng(1)
    enc = encoding()
    n = 96
    r = np.zeros(n, RECORD)
    r["query"] = random_queries(n, rng)
    r["target"] = rng.uniform(0, 2, (n, 3)).astype(np.float32)
    mlp = np.zeros(oc.MLP_PARAMS, np.float32)
    mlp[: oc.W3] = rng.uniform(-0.3, 0.3, oc.W3)
    mlp[oc.W3: oc.W3 + 192] = rng.uniform(-0.3, 0.3, 192)
    table = rng.uniform(-1, 1, (16, enc.entries, 2)).astype(np.float32)
    d_mlp, d_tab, loss = oc.gradients(mlp, table, enc, r, rounded=False)

    # the same function in torch: grid features by the oracle's corner table
    tm = torch.tensor(mlp, dtype=torch.float64, requires_grad=True)
    tt = torch.tensor(table, dtype=torch.float64, requires_grad=True)
    u = enc.unit(r["query"]["position"])
    feats = []
    for l in range(16):
        idx, wt = enc.corners(u, l)
        f = (torch.tensor(wt)[:, :, None] * tt[l][torch.tensor(idx)]).sum(1)
        feats.append(f)
    x_grid = torch.cat(feats, 1)
    x_rest = torch.tensor(oc.encode(enc, np.zeros_like(table, np.float64), r["query"])[:, 32:])
    x = torch.cat([x_grid, x_rest], 1)
    w1 = tm[oc.W1:oc.W2].view(64, 64)
    w2 = tm[oc.W2:oc.W3].view(64, 64)
    w3 = tm[oc.W3:].view(16, 64)
    h1 = torch.relu(x @ w1.T)
    h2 = torch.relu(h1 @ w2.T)
    y = (h2 @ w3.T)[:, :3]
    t = torch.tensor(r["target"], dtype=torch.float64)
    l_t = ((y - t) ** 2 / (y.detach() ** 2 + 0.01)).mean()
    l_t.backward()
    assert abs(l_t.item() - loss) < 1e-12
    assert np.allclose(d_mlp, tm.grad.numpy(), rtol=1e-9, atol=1e-14)
    assert np.allclose(d_tab, tt.grad.numpy(), rtol=1e-9, atol=1e-14)


def test_hash_and_dense_indices():
    enc = encoding(log2=10, base=4, maximum=64)
    u = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.37, 0.51, 0.93]], np.float32)
    for l in range(16):
        idx, wt = enc.corners(u, l)
        assert np.allclose(wt.sum(1), 1.0)
        assert idx.min() >= 0 and idx.max() < enc.entries
        s, res = enc.scales[l], int(enc.resolutions[l])
        p = u.astype(np.float32) * s + np.float32(0.5)
        c0 = np.floor(p).astype(np.int64)
        assert (c0 + 1).max() < res  # every corner lies inside the level's grid
        if (enc.dense >> l) & 1:
            assert np.array_equal(idx[:, 0], c0[:, 0] + c0[:, 1] * res + c0[:, 2] * res * res)
        else:
            h = (c0[:, 0] * 1) ^ (c0[:, 1] * 2654435761) ^ (c0[:, 2] * 805459861)
            assert np.array_equal(idx[:, 0], h % enc.entries)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], np.float64)
    assert np.array_equal(oc.bf16(x), np.array([1.0, 1.0, 1.0 + 2 ** -6, -2.5, oc.bf16(3.0e-3)[()]]))
    assert oc.bf16(1.0 + 2 ** -8 + 2 ** -12) == 1.0 + 2 ** -7


def test_records_are_the_abi_layout():
    assert QUERY.itemsize == 80 and RECORD.itemsize == 96
    assert C.sizeof(abi.CacheSettings) == 4 * 22
    assert C.sizeof(abi.CacheStats) == 32


@pytest.mark.parametrize("bad", [{"log2_entries": 9}, {"batch": 100}, {"base_resolution": 1},
                                 {"learning_rate": 0.0}, {"train_fraction": 1.5}, {"lo": (0, 0, 1), "hi": (1, 1, 1)}])
def test_settings_are_validated_before_the_device(bad):
    lib = abi.load()
    s = CacheSettings(**{**CacheSettings().__dict__, **bad})
    h = C.c_void_p()
    assert lib.pfxt_cache_create(C.byref(s.c()), C.byref(h)) == abi.ERR_INVALID
    assert not h.value
