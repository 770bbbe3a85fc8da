"""The denoiser: OIDN's RT filter on the GPU, the reference's
`pfx_denoise::Denoiser` (crates/denoise/src/lib.rs:58-361) over the C ABI.

    d = Denoiser()                         # OIDN's rt_hdr_alb_nrm.tza weights
    clean = d.denoise(color, albedo, normal)          # (H, W, 4) float32 host arrays
    d.denoise_device(w, h, color_ptr, albedo_ptr, normal_ptr, out_ptr, stream)
    d.denoise_trace(trace, out_ptr)        # a tracer's films (Trace::color/albedo/normal)

The product path is the CUDA library; nothing here computes pixels.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import abi
from .abi import check

OIDN_VERSION = "2.5.1"
# Where pfx_b200/weights/fetch_oidn_weights.py puts OIDN's weights.
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "weights" / "rt_hdr_alb_nrm.tza"


def default_weights() -> bytes:
    if not DEFAULT_WEIGHTS.exists():
        raise FileNotFoundError(f"{DEFAULT_WEIGHTS} is missing: run pfx_b200/weights/fetch_oidn_weights.py "
                                "with a pfx checkout, or pass the .tza blob")
    return DEFAULT_WEIGHTS.read_bytes()


class Denoiser:
    """Denoiser::new (lib.rs:81-110) on the current CUDA device."""

    def __init__(self, weights: bytes | str | Path | None = None):
        if weights is None:
            weights = default_weights()
        elif isinstance(weights, (str, Path)):
            weights = Path(weights).read_bytes()
        self._lib = abi.load()
        self._blob = C.create_string_buffer(bytes(weights), len(weights))
        h = C.c_void_p()
        check(self._lib.pfxt_denoiser_create(self._blob, len(weights), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            self._lib.pfxt_denoiser_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def denoise(self, color: np.ndarray, albedo: np.ndarray, normal: np.ndarray) -> np.ndarray:
        """Denoiser::denoise (lib.rs:112-140): (H, W, 4) float32 host images."""
        h, w = color.shape[:2]
        if albedo.shape[:2] != (h, w) or normal.shape[:2] != (h, w):
            raise ValueError("image size mismatch")
        ins = [np.ascontiguousarray(x, np.float32).reshape(h, w, 4) for x in (color, albedo, normal)]
        out = np.empty((h, w, 4), np.float32)
        check(self._lib.pfxt_denoise(self._h, w, h, *(x.ctypes.data for x in ins), out.ctypes.data))
        return out

    def denoise_device(self, width: int, height: int, color: int, albedo: int, normal: int, out: int,
                       stream: int = 0) -> None:
        """Denoiser::denoise_textures_into (lib.rs:157-183): device pointers, no wait."""
        check(self._lib.pfxt_denoise_device(self._h, width, height, color, albedo, normal, out, stream))

    def denoise_trace(self, trace, out: int) -> None:
        """The tracer's films in, `out` (device, width x height RGBA32F) written on its stream."""
        check(self._lib.pfxt_denoise_trace(self._h, trace.handle, out))

    def tiles(self):
        """Denoiser::tiles (lib.rs:112-116): (tile width, tile height, count) of the last size, or None."""
        w, h, n = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(self._lib.pfxt_denoiser_tiles(self._h, C.byref(w), C.byref(h), C.byref(n)))
        return None if n.value == 0 else (w.value, h.value, n.value)

    def last(self) -> tuple[float, int]:
        """Waits for the last denoise: (device ms, multiply-adds)."""
        ms, macs = C.c_float(), C.c_uint64()
        check(self._lib.pfxt_denoiser_last(self._h, C.byref(ms), C.byref(macs)))
        return ms.value, macs.value

    def set_max_tile_pixels(self, pixels: int) -> None:
        check(self._lib.pfxt_denoiser_set_max_tile_pixels(self._h, pixels))

    def set_wait_limit(self, polls: int) -> None:
        check(self._lib.pfxt_denoiser_set_wait_limit(self._h, polls))


def write_tza(tensors: dict) -> bytes:
    """An OIDN tensor archive (version 2) of FP16 tensors: name -> array
    (OIHW for weights, x for biases).  Used to hand the denoiser weights of
    one's own, e.g. seeded random ones in tests."""
    import struct

    data, table = bytearray(), []
    header = 12
    for name, arr in tensors.items():
        a = np.ascontiguousarray(arr, np.float16)
        offset = header + len(data)
        data += a.tobytes()
        data += bytes((-len(data)) % 16)
        table.append((name, a.shape, offset))
    out = bytearray(struct.pack("<HBBQ", 0x41D7, 2, 0, header + len(data)))
    out += data
    out += struct.pack("<I", len(table))
    for name, shape, offset in table:
        nb = name.encode()
        out += struct.pack("<H", len(nb)) + nb + struct.pack("<B", len(shape))
        out += struct.pack(f"<{len(shape)}I", *shape)
        out += b"x" if len(shape) == 1 else b"oihw"
        out += b"h" + struct.pack("<Q", offset)
    return bytes(out)
