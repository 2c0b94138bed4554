"""Build libwadi_b200.so in-tree with nvcc for sm_100a (``python -m wadi2d_b200.build``).

The library is compiled without FMA contraction and with IEEE division and square root, so that its float32
arithmetic is the reference CPU twin's statement for statement (wadi2d/solver/cpu/kernels.py, Numba without fast math).
The step's face and update passes are compiled a second time with W2B_FAST and FMA contraction into namespace
``w2b::fast`` (the approximate division, square root and cube root of ``w2b_common.cuh``); ``W2BParams.arith`` picks
one build per handle. Each unit is compiled to an object in ``_build/`` (in parallel), then linked.
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = ["w2b_step.cu", "w2b_tables.cu", "w2b_source.cu", "w2b_mlp.cu", "w2b_api.cu"]
OUT = PKG / "libwadi_b200.so"
OBJ = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    *ARCH, "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC",
]  # fmt: skip
FAST_FLAGS = ["-DW2B_FAST", "-fmad=true"]  # in place of -fmad=false: contraction on in the fast unit


def units() -> list[tuple[Path, Path, list[str]]]:
    """(source, object, extra flags) of every compilation unit."""
    out = []
    for s in SOURCES:
        src = PKG / "csrc" / s
        if src.exists():
            out.append((src, OBJ / (src.stem + ".o"), []))
    step = PKG / "csrc" / "w2b_step.cu"
    out.append((step, OBJ / "w2b_step_fast.o", FAST_FLAGS))
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    us = units()
    deps = [u[0] for u in us] + list((PKG / "csrc").glob("*.cuh")) + [ROOT / "include" / "wadi_b200.h", Path(__file__)]
    if OUT.exists() and not force and OUT.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return OUT
    OBJ.mkdir(exist_ok=True)
    procs = []
    for src, obj, extra in us:
        flags = [f for f in NVCC_FLAGS if not (extra and f == "-fmad=false")]
        cmd = ["nvcc", *flags, *extra, f"-I{ROOT / 'include'}", "-c", "-o", str(obj), str(src)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    subprocess.run(["nvcc", *ARCH, "-shared", "-o", str(OUT), *(str(u[1]) for u in us)], check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
