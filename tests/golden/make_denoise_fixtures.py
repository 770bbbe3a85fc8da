"""Writes tests/golden/denoise_desk.npz from the reference's own denoiser
fixtures (crates/denoise/tests/fixtures/desk.{color,albedo,normal,oidn}.pfm):
a 32x24 crop of the desk traced at 16 spp, and OIDN 2.5.1's CPU output for it,
the vectors crates/denoise/tests/oidn.rs checks the reference's denoiser
against (tolerance 1e-3 x (1 + |OIDN's value|) per channel).

The PFMs are read as crates/denoise/src/pfm.rs reads them: little-endian
floats scaled by |scale|, rows stored bottom to top, three channels put in
RGBA with alpha 1.

    python tests/golden/make_denoise_fixtures.py [path to the reference checkout]
"""
import sys
from pathlib import Path

import numpy as np


def read_pfm(path: Path) -> np.ndarray:
    data = path.read_bytes()
    fields, at = [], 0
    while len(fields) < 4:
        while data[at:at + 1].isspace():
            at += 1
        start = at
        while at < len(data) and not data[at:at + 1].isspace():
            at += 1
        fields.append(data[start:at].decode())
    at += 1
    channels = {"PF": 3, "Pf": 1}[fields[0]]
    width, height, scale = int(fields[1]), int(fields[2]), float(fields[3])
    assert scale < 0.0, "little-endian PFM only"
    values = np.frombuffer(data, "<f4", width * height * channels, at).reshape(height, width, channels)
    values = values[::-1] * np.float32(abs(scale))
    out = np.ones((height, width, 4), np.float32)
    for c in range(3):
        out[..., c] = values[..., min(c, channels - 1)]
    return out


def main() -> None:
    root = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    fixtures = root / "crates" / "denoise" / "tests" / "fixtures"
    arrays = {part: read_pfm(fixtures / f"desk.{part}.pfm") for part in ("color", "albedo", "normal", "oidn")}
    out = Path(__file__).parent / "denoise_desk.npz"
    np.savez_compressed(out, **arrays)
    print(out, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
