"""Build libwadi_b200.so in-tree with nvcc for sm_100a (``python -m wadi2d_b200.build``).

The step is compiled without FMA contraction and with IEEE division and square root, so that its float32 arithmetic
is the reference CPU twin's statement for statement (wadi2d/solver/cpu/kernels.py, Numba without fast math).
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = ["w2b_step.cu", "w2b_tables.cu", "w2b_source.cu", "w2b_mlp.cu", "w2b_api.cu"]
OUT = PKG / "libwadi_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-shared",
]  # fmt: skip


def sources() -> list[Path]:
    return [PKG / "csrc" / s for s in SOURCES if (PKG / "csrc" / s).exists()]


def build(force: bool = False, verbose: bool = False) -> Path:
    srcs = sources()
    deps = srcs + list((PKG / "csrc").glob("*.cuh")) + [ROOT / "include" / "wadi_b200.h"]
    if OUT.exists() and not force and OUT.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return OUT
    cmd = ["nvcc", *NVCC_FLAGS, f"-I{ROOT / 'include'}", "-o", str(OUT), *map(str, srcs)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
