"""The C ABI library loads and exports every entry point of include/pfxt.h."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from pfx_b200 import abi, synth
from pfx_b200.trace import SceneBuffers, Settings, Trace, TraceError

HEADER = Path(__file__).resolve().parent.parent / "include" / "pfxt.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(pfxt_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = abi.load()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes prototypes cover the header exactly
    assert sorted(n for n, _, _ in abi.PROTOTYPES) == names


def test_abi_version_and_error_string():
    lib = abi.load()
    assert lib.pfxt_abi_version() == 1
    assert isinstance(lib.pfxt_last_error(), bytes)


def test_invalid_light_is_refused_with_a_message():
    w = synth.plain_512()
    bad = w.scene.lights.copy()
    bad["intensity"][0] = -1.0
    w.scene.lights = bad
    with pytest.raises(TraceError) as e:
        SceneBuffers(w.scene, w.settings)
    assert e.value.code == abi.ERR_INVALID
    assert "invalid trace light" in e.value.message


def test_out_of_range_material_is_invalid_geometry():
    w = synth.plain_512()
    t = w.scene.triangles.copy()
    t["material"][5] = 10_000
    w.scene.triangles = t
    with pytest.raises(TraceError) as e:
        SceneBuffers(w.scene, w.settings)
    assert "invalid trace geometry" in e.value.message


def test_non_finite_vertex_is_invalid_geometry():
    w = synth.plain_512()
    t = w.scene.triangles.copy()
    t["v"][3, 1, 2] = np.nan
    w.scene.triangles = t
    with pytest.raises(TraceError):
        SceneBuffers(w.scene, w.settings)


def test_create_without_a_device_is_a_refusal():
    lib = abi.load()
    if lib.pfxt_device_count() > 0:
        pytest.skip("a CUDA device is present")
    w = synth.plain_512()
    with pytest.raises(TraceError) as e:
        Trace(w.scene, w.settings, 8, 8)
    assert e.value.code == abi.ERR_REFUSED


def test_adaptive_rounds_through_the_abi():
    from pfx_b200.trace import Adaptive
    assert Adaptive(0.01, 16, 100, 1.5).rounds() == [8, 16, 24, 36, 54, 81, 100]
    assert Adaptive(0.01, 16, 64, 1.5).rounds() == [8, 16, 24, 36, 54, 64]


def test_the_rust_crate_declares_every_entry_point():
    """pfx-trace-cuda/src/ffi.rs (the binding a pfx maintainer links; no Rust
    toolchain here to compile it) declares exactly the header's functions."""
    ffi = (HEADER.parent.parent / "pfx-trace-cuda" / "src" / "ffi.rs").read_text()
    declared = sorted(set(re.findall(r"pub fn (pfxt_[a-z_0-9]+)\(", ffi)))
    assert declared == declared_symbols()
