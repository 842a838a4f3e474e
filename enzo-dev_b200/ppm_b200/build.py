"""Builds libppm_b200.so (sm_100a) in-tree with nvcc.

    python -m ppm_b200.build        (from enzo-dev_b200/)

FP64 parity with the reference's arithmetic needs every multiply and add rounded
separately: -fmad=false for device code and -ffp-contract=off for host code
(the host builds the inteuler coefficient tables).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent                      # enzo-dev_b200/
REPO = ROOT.parent
CSRC = ROOT / "csrc"
OUT_DIR = ROOT / "_build"
LIB = OUT_DIR / "libppm_b200.so"
INCLUDE = REPO / "include"

SOURCES = ["ppm_kernels.cu", "ppm_split.cu", "ppm_capi.cu", "ppm_noalloc.cu", "ppm_mlp.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    newest_header = max(p.stat().st_mtime for p in headers)
    objs = []
    for src in SOURCES:
        obj = OUT_DIR / (Path(src).stem + ".o")
        stale = (force or not obj.exists() or obj.stat().st_mtime < newest_header
                 or obj.stat().st_mtime < (CSRC / src).stat().st_mtime)
        if stale:
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC),
                   "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
