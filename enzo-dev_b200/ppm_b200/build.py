"""Builds the library (sm_100a) in-tree with nvcc, in two variants of the same sources.

    python -m ppm_b200.build [--force] [-v]        (from enzo-dev_b200/)

- "exact": _build/libppm_b200.so.  Bit-identical to the FP64 oracle: every multiply
  and add rounded separately (-fmad=false for device code, -ffp-contract=off for host
  code, which builds the inteuler coefficient tables) and the reference's divisions
  as written.
- "fast": _build/libppm_b200_fast.so.  Fused multiply-adds (-fmad=true) and, where one
  divisor serves several quotients, one reciprocal and multiplications
  (PPM_FAST_ALGEBRA): the same algorithm, not the same bits, held to the tolerance
  bar of 1e-12 relative after one step and 1e-10 after 100 steps against the oracle.
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

SOURCES = ["ppm_kernels.cu", "ppm_split.cu", "ppm_capi.cu", "ppm_noalloc.cu", "ppm_mlp.cu",
           "ppm_guess_tc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fno-gnu-unique and the version script keep every symbol but the C ABI local to its
# library: both variants can be loaded in one process without one's template statics
# (gnu_unique objects, which the dynamic linker otherwise unifies process-wide) or
# functions standing in for the other's.
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-gnu-unique",
              "--expt-relaxed-constexpr"]
EXPORTS_MAP = CSRC / "exports.map"
VARIANTS = {
    "exact": {"lib": LIB, "obj": OUT_DIR, "flags": ["-fmad=false"]},
    "fast": {"lib": OUT_DIR / "libppm_b200_fast.so", "obj": OUT_DIR / "fast",
             "flags": ["-fmad=true", "-DPPM_FAST_ALGEBRA=1"]},
}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def needs_build(variant: str = "exact") -> bool:
    lib = VARIANTS[variant]["lib"]
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = (list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
            + [Path(__file__)])
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, variant: str = "exact") -> Path:
    v = VARIANTS[variant]
    lib, obj_dir = v["lib"], v["obj"]
    if not force and not needs_build(variant):
        return lib
    obj_dir.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    newest_header = max(p.stat().st_mtime for p in headers)
    objs = []
    for src in SOURCES:
        obj = obj_dir / (Path(src).stem + ".o")
        stale = (force or not obj.exists() or obj.stat().st_mtime < newest_header
                 or obj.stat().st_mtime < (CSRC / src).stat().st_mtime)
        if stale:
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *v["flags"], "-I", str(INCLUDE), "-I", str(CSRC),
                   "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = lib.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart",
                    "-Xlinker", f"--version-script={EXPORTS_MAP}"], check=True)
    os.replace(tmp, lib)
    return lib


def build_all(force: bool = False, verbose: bool = False) -> list:
    return [build(force, verbose, name) for name in VARIANTS]


if __name__ == "__main__":
    for path in build_all(force="--force" in sys.argv, verbose="-v" in sys.argv):
        print(path)
