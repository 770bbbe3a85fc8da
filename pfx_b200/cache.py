"""The neural radiance cache through the C ABI (pfxt_cache_* in include/pfxt.h).

A 16-level hash grid (2 FP16 features per level) plus one-blob direction and
normal, roughness, diffuse and specular albedo and transmission feed a
64-64-3 ReLU MLP evaluated and trained on the tensor cores (BF16 operands,
FP32 accumulation, FP32 master weights, Adam).  Attach it to a tracer with
`Trace.set_cache`; paths then end into the cache at `query_bounce`.  The
reference tracer has no cache; nothing here has a counterpart in pfx.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import check

QUERY = np.dtype([("position", "<f4", 3), ("roughness", "<f4"), ("direction", "<f4", 3), ("transmission", "<f4"),
                  ("normal", "<f4", 3), ("pad0", "<f4"), ("diffuse", "<f4", 3), ("pad1", "<f4"),
                  ("specular", "<f4", 3), ("pad2", "<f4")])
RECORD = np.dtype([("query", QUERY), ("target", "<f4", 3), ("weight", "<f4")])
assert QUERY.itemsize == 80 and RECORD.itemsize == 96

LEVELS, HIDDEN, INPUTS, OUT_ROWS = 16, 64, 64, 16
W1, W2, W3 = 0, HIDDEN * INPUTS, 2 * HIDDEN * INPUTS
MLP_PARAMS = W3 + OUT_ROWS * HIDDEN


@dataclass
class CacheSettings:
    log2_entries: int = 19
    base_resolution: int = 16
    max_resolution: int = 2048
    batch: int = 65536
    steps: int = 4
    seed: int = 1
    query_bounce: int = 1
    record_bounces: int = 4
    learning_rate: float = 1e-2
    beta1: float = 0.9
    beta2: float = 0.99
    epsilon: float = 1e-15
    train_fraction: float = 0.01
    error_bound: float = 1.0
    min_roughness: float = 0.25
    delay_bounces: int = 2
    lo: tuple = (0.0, 0.0, 0.0)
    hi: tuple = (1.0, 1.0, 1.0)

    def c(self) -> abi.CacheSettings:
        s = abi.CacheSettings()
        for name, _ in abi.CacheSettings._fields_:
            v = getattr(self, name)
            if name in ("lo", "hi"):
                setattr(s, name, abi.f3(*v))
            else:
                setattr(s, name, v)
        return s

    @property
    def entries(self) -> int:
        return 1 << self.log2_entries


class RadianceCache:
    """A cache on the current CUDA device (the product path; raises without the library)."""

    def __init__(self, settings: CacheSettings | None = None):
        self.settings = settings or CacheSettings()
        self._lib = abi.load()
        h = C.c_void_p()
        check(self._lib.pfxt_cache_create(C.byref(self.settings.c()), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            self._lib.pfxt_cache_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def infer(self, queries: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(queries, QUERY)
        out = np.zeros((len(q), 3), np.float32)
        check(self._lib.pfxt_cache_infer(self._h, q.ctypes.data, len(q), out.ctypes.data))
        return out

    def gradients(self, records: np.ndarray, table: bool = True):
        r = np.ascontiguousarray(records, RECORD)
        mlp = np.zeros(MLP_PARAMS, np.float32)
        tab = np.zeros((LEVELS, self.settings.entries, 2), np.float32) if table else None
        loss = C.c_float()
        check(self._lib.pfxt_cache_gradients(self._h, r.ctypes.data, len(r), mlp.ctypes.data,
                                             tab.ctypes.data if table else None, C.byref(loss)))
        return mlp, tab, float(loss.value)

    def train(self, records: np.ndarray) -> float:
        r = np.ascontiguousarray(records, RECORD)
        loss = C.c_float()
        check(self._lib.pfxt_cache_train(self._h, r.ctypes.data, len(r), C.byref(loss)))
        return float(loss.value)

    def params(self):
        mlp = np.zeros(MLP_PARAMS, np.float32)
        tab = np.zeros((LEVELS, self.settings.entries, 2), np.float32)
        check(self._lib.pfxt_cache_params(self._h, mlp.ctypes.data, tab.ctypes.data))
        return mlp, tab

    def set_params(self, mlp: np.ndarray | None = None, table: np.ndarray | None = None) -> None:
        m = None if mlp is None else np.ascontiguousarray(mlp, np.float32)
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        if m is not None:
            assert m.size == MLP_PARAMS
        if t is not None:
            assert t.size == LEVELS * self.settings.entries * 2
        check(self._lib.pfxt_cache_set_params(self._h, None if m is None else m.ctypes.data,
                                              None if t is None else t.ctypes.data))

    def encoding(self):
        scales = np.zeros(LEVELS, np.float32)
        res = np.zeros(LEVELS, np.uint32)
        dense = C.c_uint32()
        check(self._lib.pfxt_cache_encoding(self._h, scales.ctypes.data, res.ctypes.data, C.byref(dense)))
        return scales, res, int(dense.value)

    def set_wait_limit(self, polls: int) -> None:
        """Polls before a kernel's wait for its tensor-core work gives up (the
        call then fails and the cache stays usable); 0 makes every wait give up."""
        check(self._lib.pfxt_cache_set_wait_limit(self._h, int(polls)))

    def stats(self) -> dict:
        s = abi.CacheStats()
        check(self._lib.pfxt_cache_get_stats(self._h, C.byref(s)))
        return {"steps": int(s.steps), "loss": float(s.loss), "records": int(s.records), "queries": int(s.queries),
                "training_paths": int(s.training_paths), "cells_ok": int(s.cells_ok)}


def random_queries(n: int, rng: np.random.Generator, lo=(0, 0, 0), hi=(1, 1, 1)) -> np.ndarray:
    """Seeded queries spread over the box: unit directions and normals, albedos in [0, 1]."""
    q = np.zeros(n, QUERY)
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    q["position"] = (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)
    for key in ("direction", "normal"):
        v = rng.normal(size=(n, 3))
        q[key] = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    q["roughness"] = rng.random(n).astype(np.float32)
    q["transmission"] = (rng.random(n) < 0.1).astype(np.float32)
    q["diffuse"] = rng.random((n, 3)).astype(np.float32)
    q["specular"] = rng.random((n, 3)).astype(np.float32)
    return q
