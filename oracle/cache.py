"""CPU oracle of the radiance cache's network, in FP64 (test infrastructure).

Only tests, smoke() and bench.py's CPU baseline may import this module; the
product is libpfxtrace.so.  The reference tracer (pfx crates/trace) has no
radiance cache, so there is no reference code to follow: this restates the
published methods the CUDA kernels implement -

  * multiresolution hash encoding (Mueller, Evans, Schied, Keller 2022,
    "Instant neural graphics primitives"): per level l a grid of scale s_l,
    position u in [0,1]^3 mapped to u*s_l + 0.5, trilinear interpolation of
    the 8 corners' features; levels whose (resolution)^3 fits the table are
    indexed densely, the others by the spatial hash
    x*1 ^ y*2654435761 ^ z*805459861 modulo the table size;
  * neural radiance caching (Mueller, Rousselle, Novak, Keller 2021): one-blob
    encoded direction and normal, roughness and albedos as further inputs,
    ReLU MLP, relative L2 loss (y - t)^2 / (sg(y)^2 + 0.01);
  * Adam (Kingma & Ba 2015), here lazy: a parameter whose gradient is exactly
    zero keeps its value and moments.

Rounding is mirrored where the CUDA path rounds - FP16 table features, BF16
weights, inputs, activations and output gradients - and everything else is
FP64, so the CUDA results differ from these only by FP32 accumulation order.
The position-to-cell arithmetic is done in FP32 exactly as on the device, so
grid indices agree bit for bit.  Parity of the backward pass is pinned by
PyTorch autograd in FP64 (tests/test_cache_oracle.py) with the rounding off.
"""
from __future__ import annotations

import numpy as np

LEVELS, HIDDEN, INPUTS, OUT_ROWS = 16, 64, 64, 16
W1, W2, W3 = 0, HIDDEN * INPUTS, 2 * HIDDEN * INPUTS
MLP_PARAMS = W3 + OUT_ROWS * HIDDEN
PRIMES = (np.uint32(1), np.uint32(2654435761), np.uint32(805459861))


def bf16(x) -> np.ndarray:
    """Round to BF16 (nearest even) through FP32, as __float2bfloat16_rn of an FP32 value."""
    x32 = np.asarray(x, np.float64).astype(np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f16(x) -> np.ndarray:
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float64)


class Encoding:
    """Grid geometry as the library reports it (pfxt_cache_encoding) plus the bounds."""

    def __init__(self, scales, resolutions, dense, entries, lo, hi):
        self.scales = np.asarray(scales, np.float32)
        self.resolutions = np.asarray(resolutions, np.uint32)
        self.dense = int(dense)
        self.entries = int(entries)
        self.lo = np.asarray(lo, np.float32)
        self.inv = (np.float32(1.0) / (np.asarray(hi, np.float32) - self.lo)).astype(np.float32)

    def unit(self, pos) -> np.ndarray:
        u = ((np.asarray(pos, np.float32) - self.lo) * self.inv).astype(np.float32)
        u = np.where(u > 0, np.where(u < 1, u, np.float32(1)), np.float32(0))  # NaN -> 0
        return u.astype(np.float32)

    def corners(self, u, l):
        """(indices (n, 8), weights (n, 8)) of level l."""
        s = self.scales[l]
        p = (u * s + np.float32(0.5)).astype(np.float32)
        f = np.floor(p)
        w = (p - f).astype(np.float32)
        base = f.astype(np.uint32)
        res = np.uint32(self.resolutions[l])
        idx = np.zeros((len(u), 8), np.int64)
        wt = np.zeros((len(u), 8), np.float64)
        for k in range(8):
            o = np.array([k & 1, (k >> 1) & 1, k >> 2], np.uint32)
            c = base + o
            if (self.dense >> l) & 1:
                i = c[:, 0] + c[:, 1] * res + c[:, 2] * res * res
            else:
                i = (c[:, 0] * PRIMES[0]) ^ (c[:, 1] * PRIMES[1]) ^ (c[:, 2] * PRIMES[2])
            idx[:, k] = (i & np.uint32(self.entries - 1)).astype(np.int64)
            a = np.where(o[0], w[:, 0], np.float32(1) - w[:, 0]).astype(np.float64)
            b = np.where(o[1], w[:, 1], np.float32(1) - w[:, 1]).astype(np.float64)
            d = np.where(o[2], w[:, 2], np.float32(1) - w[:, 2]).astype(np.float64)
            wt[:, k] = a * b * d
        return idx, wt


def one_blob(v) -> np.ndarray:
    """Hat-function one-blob of values in [-1, 1], 4 bins (FP32 as on the device)."""
    t = ((np.asarray(v, np.float32) + np.float32(1)) * np.float32(0.5) * np.float32(4)).astype(np.float32)
    out = np.zeros(t.shape + (4,), np.float32)
    for i in range(4):
        h = np.float32(1) - np.abs(t - np.float32(i + 0.5))
        out[..., i] = np.maximum(h, np.float32(0))
    return out.astype(np.float64)


def encode(enc: Encoding, table16: np.ndarray, queries) -> np.ndarray:
    """Network inputs (n, 64), FP64 before the BF16 rounding; table16 (16, T, 2) FP16 values."""
    n = len(queries)
    x = np.zeros((n, INPUTS))
    u = enc.unit(queries["position"])
    for l in range(LEVELS):
        idx, wt = enc.corners(u, l)
        feats = table16[l][idx]  # (n, 8, 2)
        x[:, 2 * l] = (wt * feats[..., 0]).sum(1)
        x[:, 2 * l + 1] = (wt * feats[..., 1]).sum(1)
    x[:, 32:44] = one_blob(queries["direction"]).reshape(n, 12)
    x[:, 44:56] = one_blob(queries["normal"]).reshape(n, 12)
    r = queries["roughness"].astype(np.float32)
    x[:, 56] = np.where(r > 0, np.where(r < 1, r, 1), 0)
    x[:, 57:60] = queries["diffuse"]
    x[:, 60:63] = queries["specular"]
    x[:, 63] = queries["transmission"]
    return x


def weights(mlp: np.ndarray, rounded: bool = True):
    w1 = mlp[W1:W2].reshape(HIDDEN, INPUTS).astype(np.float64)
    w2 = mlp[W2:W3].reshape(HIDDEN, HIDDEN).astype(np.float64)
    w3 = mlp[W3:].reshape(OUT_ROWS, HIDDEN).astype(np.float64)
    if rounded:
        return bf16(w1), bf16(w2), bf16(w3)
    return w1, w2, w3


def forward(mlp, x, rounded: bool = True):
    """(y (n, 3), activations) of the MLP on inputs x."""
    r = bf16 if rounded else (lambda a: np.asarray(a, np.float64))
    w1, w2, w3 = weights(mlp, rounded)
    xb = r(x)
    h1 = r(np.maximum(xb @ w1.T, 0))
    h2 = r(np.maximum(h1 @ w2.T, 0))
    y = h2 @ w3.T
    return y[:, :3], (xb, h1, h2)


def infer(mlp, table, enc: Encoding, queries) -> np.ndarray:
    x = encode(enc, f16(table), queries)
    return forward(mlp, x)[0]


def gradients(mlp, table, enc: Encoding, records, rounded: bool = True):
    """(dmlp (9216,), dtable (16, T, 2), mean loss) of the relative L2 loss."""
    r = bf16 if rounded else (lambda a: np.asarray(a, np.float64))
    tab = f16(table) if rounded else np.asarray(table, np.float64)
    q = records["query"]
    x = encode(enc, tab, q)
    y, (xb, h1, h2) = forward(mlp, x, rounded)
    w1, w2, w3 = weights(mlp, rounded)
    t = records["target"].astype(np.float64)
    n = len(records)
    d = y - t
    den = y * y + 0.01
    loss = float((d * d / den).sum() / (3 * n))
    dy = np.zeros((n, OUT_ROWS))
    dy[:, :3] = r(2 * d / den / (3 * n))
    dh2 = r((dy @ w3) * (h2 > 0))
    dh1 = r((dh2 @ w2) * (h1 > 0))
    dx = dh1 @ w1[:, :32]
    dmlp = np.zeros(MLP_PARAMS)
    dmlp[W1:W2] = (dh1.T @ xb).reshape(-1)
    dmlp[W2:W3] = (dh2.T @ h1).reshape(-1)
    dmlp[W3:] = (dy.T @ h2).reshape(-1)
    dtab = np.zeros((LEVELS, enc.entries, 2))
    u = enc.unit(q["position"])
    for l in range(LEVELS):
        idx, wt = enc.corners(u, l)
        for f in range(2):
            np.add.at(dtab[l, :, f], idx.reshape(-1), (wt * dx[:, 2 * l + f][:, None]).reshape(-1))
    return dmlp, dtab, loss


def adam(p, m, v, g, step, beta_pow, lr, b1, b2, eps):
    """One lazy Adam step in FP64; beta_pow = (b1^t, b2^t) after this step's update."""
    p, m, v = p.astype(np.float64).copy(), m.astype(np.float64).copy(), v.astype(np.float64).copy()
    live = g != 0
    m[live] = b1 * m[live] + (1 - b1) * g[live]
    v[live] = b2 * v[live] + (1 - b2) * g[live] ** 2
    c1, c2 = 1 - beta_pow[0], 1 - beta_pow[1]
    p[live] = p[live] - lr * (m[live] / c1) / (np.sqrt(v[live] / c2) + eps)
    return p, m, v
