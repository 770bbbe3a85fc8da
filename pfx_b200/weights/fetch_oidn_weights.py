"""Copies OIDN's RT filter weights (rt_hdr_alb_nrm.tza, OIDN 2.5.1, Apache
License 2.0) from a pfx checkout, where crates/denoise/weights ships them,
next to this script.  The copy is a build artefact (git-ignored); the
denoiser reads whatever .tza blob its caller hands it.

    python pfx_b200/weights/fetch_oidn_weights.py [pfx checkout, default /root/reference]
"""
import shutil
import sys
from pathlib import Path

NAME = "rt_hdr_alb_nrm.tza"
HERE = Path(__file__).resolve().parent


def fetch(checkout: str = "/root/reference") -> Path | None:
    src = Path(checkout) / "crates" / "denoise" / "weights" / NAME
    dst = HERE / NAME
    if dst.exists() and (not src.exists() or dst.stat().st_size == src.stat().st_size):
        return dst
    if not src.exists():
        return None
    shutil.copyfile(src, dst)
    return dst


if __name__ == "__main__":
    print(fetch(*sys.argv[1:2]))
