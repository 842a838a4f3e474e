"""CPU-side checks of the C ABI: the library builds, loads, and exports every
entry point that include/ppm_b200.h declares (no compute calls without a GPU)."""
import ctypes as C
import re
from pathlib import Path

from ppm_b200 import capi

REPO = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (REPO / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(ppm_b200_\w+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_header_declares_the_api():
    names = declared_symbols()
    assert set(capi.EXPORTS) <= names, set(capi.EXPORTS) - names


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
        assert C.cast(getattr(L, name), C.c_void_p).value


def test_version_and_error_strings():
    L = capi.lib()
    assert L.ppm_b200_version() == 100
    assert capi.error_string(capi.ERR_NEGATIVE).startswith("negative")
    assert capi.error_string(capi.ERR_UNSUPPORTED).startswith("configuration")


def test_unsupported_configuration_is_rejected_before_any_device_work():
    # Options outside this library (flattening types above 3, diffusion, steepening other than
    # 0/1, more colours than MAX_COLOR, Riemann solvers other than two-shock, HLL and
    # HLLC): the caller keeps the Fortran path.  The context pointer is never touched.
    L = capi.lib()
    from ppm_b200 import harness as H
    g = H.Grid.uniform((8, 8, 8))
    hp = H.HydroParams()
    f = H.new_fields(g, False)
    for field, value in (("flattening", 4), ("diffusion", 1), ("steepening", 2),
                         ("number_of_colours", 46), ("number_of_colours", -1),
                         ("riemann_solver", 2), ("riemann_solver", 6),
                         ("pressure_free", 2), ("eos_type", 1), ("eos_type", 2)):
        P = capi.make_params(hp, 0.1)
        setattr(P, field, value)
        G, keep = capi.make_grid(g, f)
        rc = L.ppm_b200_solve_ppm_de(C.c_void_p(1), C.byref(P), 0, C.byref(G), 0, 0, None, None,
                                     None)
        assert rc == capi.ERR_UNSUPPORTED, field


def test_colours_without_field_pointers_are_invalid():
    # number_of_colours > 0 needs grid.colours with that many non-NULL fields; the check
    # precedes any use of the context
    L = capi.lib()
    from ppm_b200 import harness as H
    g = H.Grid.uniform((8, 8, 8))
    f = H.new_fields(g, False)
    P = capi.make_params(H.HydroParams(), 0.1)
    P.number_of_colours = 2
    G, keep = capi.make_grid(g, f)
    rc = L.ppm_b200_solve_ppm_de(C.c_void_p(1), C.byref(P), 0, C.byref(G), 0, 0, None, None,
                                 None)
    assert rc == capi.ERR_INVALID
    arr = (C.c_void_p * 2)(f["d"].ctypes.data, None)
    G.colours = C.cast(arr, C.c_void_p)
    rc = L.ppm_b200_solve_ppm_de(C.c_void_p(1), C.byref(P), 0, C.byref(G), 0, 0, None, None,
                                 None)
    assert rc == capi.ERR_INVALID
