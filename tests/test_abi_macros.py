"""The C ABI under Enzo's default build macros (CPU only).

Enzo compiles with CONFIG_INTEGERS = 64 and CONFIG_PRECISION = 64 by default
(Make.config.settings:61, :79), which put `#define int long_int` and
`#define float double` in force before any other header is included
(macros_and_parameters.h:217, :257).  A translation unit that includes ppm_b200.h
under those macros must still see the library's struct layouts and prototypes:
tests/abi_enzo_macros.cpp does exactly that, links against the library and calls
ppm_b200_abi_check, ppm_b200_version and ppm_b200_error_string through it.  The same
program built against a copy of the header without the macro guard reports a
mismatch, which shows that the check can fail.
"""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

from ppm_b200 import capi

REPO = Path(__file__).resolve().parents[1]
SRC = REPO / "tests" / "abi_enzo_macros.cpp"
CUDA_LIB = Path("/usr/local/cuda/lib64")


def _compile_and_run(include_dir: Path, exe: Path):
    lib = capi.library_path()
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    cmd = [cxx, "-std=c++17", "-O1", "-w", "-I", str(include_dir), str(SRC), "-o", str(exe),
           "-L", str(lib.parent), "-lppm_b200", f"-Wl,-rpath,{lib.parent}",
           "-Wl,--allow-shlib-undefined"]
    if CUDA_LIB.exists():
        cmd += [f"-Wl,-rpath-link,{CUDA_LIB}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.pathsep.join(
        [str(lib.parent)] + [p for p in env.get("LD_LIBRARY_PATH", "").split(os.pathsep) if p])
    return subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=60)


def test_header_keeps_its_layout_under_enzo_macros(tmp_path):
    capi.lib()  # the library is built
    r = _compile_and_run(REPO / "include", tmp_path / "abi_ok")
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "abi_check=0 " in r.stdout


def test_unguarded_header_is_caught_by_the_layout_check(tmp_path):
    capi.lib()
    txt = (REPO / "include" / "ppm_b200.h").read_text()
    for line in ('#pragma push_macro("int")', '#pragma push_macro("float")', "#undef int",
                 "#undef float", '#pragma pop_macro("float")', '#pragma pop_macro("int")'):
        assert line in txt, line
        txt = txt.replace(line, "")
    inc = tmp_path / "include"
    inc.mkdir()
    (inc / "ppm_b200.h").write_text(txt)
    r = _compile_and_run(inc, tmp_path / "abi_bad")
    assert r.returncode != 0, r.stdout


def test_abi_check_rejects_a_wrong_list():
    import ctypes as C
    L = capi.lib()
    L.ppm_b200_abi_check.restype = C.c_int
    L.ppm_b200_abi_check.argtypes = [C.POINTER(C.c_longlong), C.c_int]
    assert L.ppm_b200_abi_check(None, 0) == capi.ERR_INVALID
    arr = (C.c_longlong * 3)(1, 2, 3)
    assert L.ppm_b200_abi_check(arr, 3) == capi.ERR_INVALID
