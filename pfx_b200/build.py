"""Build libpfxtrace.so in-tree for sm_100a.

The library is plain C ABI (include/pfxt.h) over hand-written CUDA kernels; it
does not link against torch.  Objects go to pfx_b200/_build/, the shared
library to pfx_b200/lib/libpfxtrace.so.  Recompiles only what changed.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
REPO = ROOT.parent
CSRC = ROOT / "csrc"
BUILD = ROOT / "_build"
LIB = ROOT / "lib" / "libpfxtrace.so"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA / "bin" / "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Exact fp32: no FMA contraction, IEEE division and square root, so the device
# arithmetic matches the host restatement bit for bit.
EXACT = ["-fmad=false", "--prec-div=true", "--prec-sqrt=true", "--ftz=false"]
HOST = ["-fPIC", "-ffp-contract=off", "-fno-fast-math", "-O2"]
INCLUDES = [f"-I{REPO / 'include'}", f"-I{CSRC}"]

# (source, extra nvcc flags).  Kernels whose results are compared with a
# tolerance rather than bit for bit may opt out of EXACT.
SOURCES = [
    ("build.cpp", []),
    ("layout.cpp", []),
    ("capi.cu", EXACT),
    ("tracer_host.cu", EXACT),
    ("traverse.cu", EXACT),
    ("tracer.cu", EXACT),
    ("noalloc.cu", EXACT),
    ("bvh_gpu.cu", EXACT),
    ("cache.cu", EXACT),
    ("denoise.cu", EXACT),
]

HEADERS = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [REPO / "include" / "pfxt.h"]


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[-1]}")


def compile_one(src: str, extra: list[str], verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    path = CSRC / src
    obj = BUILD / (src + ".o")
    if not _newer(obj, [path, *HEADERS, Path(__file__)]):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, *extra, *INCLUDES,
               "-Xcompiler", ",".join(HOST), "-c", str(path), "-o", str(obj)]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", "-std=c++17", *HOST, *INCLUDES, f"-I{CUDA / 'include'}", "-c", str(path), "-o", str(obj)]
    _run(cmd)
    return obj


def build(force: bool = False) -> Path:
    if force and BUILD.exists():
        for f in BUILD.glob("*.o"):
            f.unlink()
    objs = [compile_one(src, extra) for src, extra in SOURCES]
    LIB.parent.mkdir(parents=True, exist_ok=True)
    if _newer(LIB, objs):
        _run([NVCC, "-shared", *ARCH, *[str(o) for o in objs], "-o", str(LIB),
              "-Xcompiler", "-fPIC", "-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
