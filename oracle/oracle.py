"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C FP64 restatement of Enzo's PPM-DE hot path
(``ppm_oracle.c``; see its header for the reference file:line map).  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
load it -- always as the checker or the timed CPU reference, never as part of
the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libppm_oracle.so"

FIELD_NAMES = ("d", "te", "v1", "v2", "v3", "ge")
MAX_COLOUR = 45  # MAX_COLOR, fortran.def:2


def colour_names(fields):
    """Colour fields of a field dict: keys col0, col1, ... (the colnum[] order)."""
    n = 0
    while f"col{n}" in fields:
        n += 1
    return [f"col{k}" for k in range(n)]


class OraParams(C.Structure):
    _fields_ = [
        ("rank", C.c_int),
        ("dims", C.c_int * 3),
        ("start", C.c_int * 3),
        ("end", C.c_int * 3),
        ("gamma", C.c_double),
        ("dt", C.c_double),
        ("eta1", C.c_double),
        ("eta2", C.c_double),
        ("small_rho", C.c_double),
        ("tiny_number", C.c_double),
        ("min_support", C.c_double),
        ("dual", C.c_int),
        ("gravity", C.c_int),
        ("pressure_free", C.c_int),
        ("fallback", C.c_int),
        ("max_velocity_index", C.c_int),
        ("steepen", C.c_int),
        ("flatten", C.c_int),
        ("ncolour", C.c_int),
        ("riemann", C.c_int),
        ("colour_species", C.c_void_p),
        ("eos_type", C.c_int),
        ("eos_sound_speed", C.c_double),
    ]


class OraFluxes(C.Structure):
    _fields_ = [
        ("left_start", (C.c_longlong * 3) * 3),
        ("left_end", (C.c_longlong * 3) * 3),
        ("right_start", (C.c_longlong * 3) * 3),
        ("right_end", (C.c_longlong * 3) * 3),
        ("left", (C.POINTER(C.c_double) * 3) * 6),
        ("right", (C.POINTER(C.c_double) * 3) * 6),
        ("colour_left", (C.POINTER(C.c_double) * 3) * MAX_COLOUR),
        ("colour_right", (C.POINTER(C.c_double) * 3) * MAX_COLOUR),
    ]


class OraStats(C.Structure):
    _fields_ = [
        ("interfaces", C.c_longlong),
        ("newton_iters", C.c_longlong),
        ("newton_hist", C.c_longlong * 8),
        ("fallbacks", C.c_longlong),
        ("fatal", C.c_int),
    ]

    def as_dict(self):
        return {
            "interfaces": int(self.interfaces),
            "newton_iters": int(self.newton_iters),
            "newton_hist": [int(x) for x in self.newton_hist],
            "fallbacks": int(self.fallbacks),
            "fatal": int(self.fatal),
        }


_lib = None
_kind = "parity"
_loaded = {}
# builds of the same source: "parity" is the checker (-O2, no contraction); "native"
# (-O3 -march=native, no contraction: the same bits) and "native_fma" (-O3
# -march=native, contraction allowed) are the timed CPU baselines, built by `make
# native` on the machine that runs them
BUILDS = {"parity": LIB_PATH, "native": HERE / "_build" / "libppm_oracle_native.so",
          "native_fma": HERE / "_build" / "libppm_oracle_native_fma.so"}


def build(kind: str = "parity") -> Path:
    """Compile the oracle (make in oracle/)."""
    target = [] if kind == "parity" else ["native"]
    subprocess.run(["make", "-s", "-C", str(HERE), *target], check=True)
    return BUILDS[kind]


def select(kind: str) -> None:
    """Make later calls use the given build ("parity", "native" or "native_fma")."""
    global _lib, _kind
    if kind not in BUILDS:
        raise ValueError(kind)
    if kind != _kind:
        _kind = kind
        _lib = _loaded.get(kind)


def lib():
    global _lib
    if _lib is None:
        path = BUILDS[_kind]
        if not path.exists():
            build(_kind)
        L = C.CDLL(str(path))
        dp = C.POINTER(C.c_double)
        L.ora_solve_ppm_de.argtypes = [C.POINTER(OraParams), C.c_int, C.c_void_p, dp * 3, dp * 3,
                                       C.c_int, C.POINTER(OraFluxes), C.c_longlong * 3,
                                       C.POINTER(OraStats), C.c_int]
        L.ora_solve_ppm_de.restype = C.c_int
        L.ora_sweep.argtypes = [C.c_int, C.POINTER(OraParams), C.c_void_p, dp, dp * 3, dp * 3,
                                C.c_int, C.POINTER(OraFluxes), C.c_longlong * 3,
                                C.POINTER(OraStats), C.c_int]
        L.ora_sweep.restype = C.c_int
        L.ora_compute_pressure.argtypes = [C.POINTER(OraParams), dp * 6, dp]
        L.ora_compute_pressure.restype = None
        L.ora_calc_dt.argtypes = [C.POINTER(OraParams), dp * 6, dp, dp * 3, C.c_double,
                                  C.c_double * 3]
        L.ora_calc_dt.restype = C.c_double
        L.ora_twoshock_point.argtypes = [C.c_double * 6, C.c_double, C.c_double, C.c_double,
                                         dp, dp, C.POINTER(C.c_int)]
        L.ora_twoshock_point.restype = None
        L.ora_expansion_terms.argtypes = [C.POINTER(OraParams), dp * 6, C.c_void_p, C.c_double,
                                          C.c_double, C.c_double]
        L.ora_expansion_terms.restype = None
        L.ora_correct_fluxes.argtypes = [C.POINTER(OraParams), C.c_void_p, C.c_int,
                                         C.POINTER(OraFluxes), C.POINTER(OraFluxes),
                                         C.c_longlong * 3]
        L.ora_correct_fluxes.restype = C.c_int
        L.ora_correct_fluxes_sublings.argtypes = [C.POINTER(OraParams), C.c_void_p, C.c_int,
                                                  C.POINTER(OraFluxes), C.POINTER(OraFluxes),
                                                  C.c_longlong * 3, C.c_longlong * 3,
                                                  C.c_int * 3]
        L.ora_correct_fluxes_sublings.restype = C.c_int
        _lib = L
        _loaded[_kind] = L
    return _lib


def _ptr(a):
    if a is None:
        return C.POINTER(C.c_double)()
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_params(grid, hp, dt, ncolour=0) -> OraParams:
    """grid: object with rank, dims(3), start(3), end(3); hp: HydroParams-like."""
    P = OraParams()
    P.rank = grid.rank
    for d in range(3):
        P.dims[d] = grid.dims[d]
        P.start[d] = grid.start[d]
        P.end[d] = grid.end[d]
    P.gamma = hp.gamma
    P.dt = dt
    P.eta1 = hp.eta1
    P.eta2 = hp.eta2
    P.small_rho = hp.small_rho
    P.tiny_number = hp.tiny_number
    P.min_support = hp.min_support
    P.dual = int(hp.dual)
    P.gravity = int(hp.gravity)
    P.pressure_free = int(hp.pressure_free)
    P.fallback = int(hp.fallback)
    P.max_velocity_index = grid.rank
    P.steepen = int(getattr(hp, "steepen", 0))
    P.flatten = int(getattr(hp, "flatten", 0))
    P.ncolour = int(ncolour)
    P.riemann = int(getattr(hp, "riemann", 5))
    P.eos_type = int(getattr(hp, "eos_type", 0))
    P.eos_sound_speed = float(getattr(hp, "eos_sound_speed", 2.65e4))
    return P


def _fields6(fields):
    arr = (C.POINTER(C.c_double) * 6)()
    for i, n in enumerate(FIELD_NAMES):
        arr[i] = _ptr(fields.get(n))
    return arr


def _fields_all(fields):
    """The six hydro fields, then the colour fields (kept alive by the returned array)."""
    cols = colour_names(fields)
    arr = (C.POINTER(C.c_double) * (6 + len(cols)))()
    for i, n in enumerate(FIELD_NAMES + tuple(cols)):
        arr[i] = _ptr(fields.get(n))
    return arr, len(cols)


def _cw3(cellwidth):
    arr = (C.POINTER(C.c_double) * 3)()
    for d in range(3):
        arr[d] = _ptr(cellwidth[d] if d < len(cellwidth) else None)
    return arr


def solve_ppm_de(grid, hp, dt, cycle, fields, cellwidth, accel=None, subgrids=None,
                 ggs=(0, 0, 0), nthreads=1):
    """Advance `fields` (dict of float64 arrays, x fastest) by one split step in place.

    Returns (rc, stats dict).  subgrids: list of OraFluxes (filled in place)."""
    L = lib()
    F, ncol = _fields_all(fields)
    P = make_params(grid, hp, dt, ncol)
    acc = (C.POINTER(C.c_double) * 3)()
    if accel is not None:
        for d in range(3):
            acc[d] = _ptr(accel[d] if d < len(accel) else None)
    st = OraStats()
    nsub = 0 if not subgrids else len(subgrids)
    subarr = None
    if nsub:
        subarr = (OraFluxes * nsub)(*subgrids)
    g = (C.c_longlong * 3)(*ggs)
    rc = L.ora_solve_ppm_de(C.byref(P), int(cycle), F, acc, _cw3(cellwidth), nsub,
                            subarr, g, C.byref(st), int(nthreads))
    if nsub:
        for i in range(nsub):
            subgrids[i] = subarr[i]
    return rc, st.as_dict()


def sweep(dim, grid, hp, dt, fields, pressure, cellwidth, accel=None, nthreads=1):
    L = lib()
    F, ncol = _fields_all(fields)
    P = make_params(grid, hp, dt, ncol)
    acc = (C.POINTER(C.c_double) * 3)()
    if accel is not None:
        for d in range(3):
            acc[d] = _ptr(accel[d] if d < len(accel) else None)
    st = OraStats()
    g = (C.c_longlong * 3)(0, 0, 0)
    rc = L.ora_sweep(int(dim), C.byref(P), F, _ptr(pressure), acc,
                     _cw3(cellwidth), 0, None, g, C.byref(st), int(nthreads))
    return rc, st.as_dict()


def compute_pressure(grid, hp, fields):
    L = lib()
    P = make_params(grid, hp, 0.0)
    p = np.zeros_like(fields["d"])
    L.ora_compute_pressure(C.byref(P), _fields6(fields), _ptr(p))
    return p


def calc_dt(grid, hp, fields, pressure, cellwidth, aye=1.0, vgrid=(0.0, 0.0, 0.0)):
    """calc_dt (without the Courant factor)."""
    L = lib()
    P = make_params(grid, hp, 0.0)
    return L.ora_calc_dt(C.byref(P), _fields6(fields), _ptr(pressure), _cw3(cellwidth),
                         float(aye), (C.c_double * 3)(*vgrid))


def twoshock_point(states6, gamma, pmin, guess=0.0):
    L = lib()
    pb = C.c_double()
    ub = C.c_double()
    it = C.c_int()
    L.ora_twoshock_point((C.c_double * 6)(*states6), gamma, pmin, guess, C.byref(pb),
                         C.byref(ub), C.byref(it))
    return pb.value, ub.value, it.value

def expansion_terms(grid, hp, fields, old, time, old_time, coefficient):
    """grid::ComovingExpansionTerms on host fields (in place); old: fields at OldTime
    or None."""
    L = lib()
    P = make_params(grid, hp, 0.0)
    F = _fields6(fields)
    O = C.cast(_fields6(old), C.c_void_p) if old is not None else None
    L.ora_expansion_terms(C.byref(P), F, O, float(time), float(old_time), float(coefficient))


def _species(P, ncol, species):
    """Species flags (one per colour) into P; returns the array to keep alive."""
    if not species:
        return None
    arr = (C.c_int * max(ncol, 1))(*[int(bool(x)) for x in species])
    P.colour_species = C.cast(arr, C.c_void_p)
    return arr


def correct_fluxes(grid, hp, fields, initial, refined, ggs, species=None):
    """grid::CorrectForRefinedFluxes (proper subgrids) on host fields, in place.  initial /
    refined: lists of OraFluxes (the refined ones are updated where a correction is
    undone).  ggs: global index of the grid's first zone.  Returns the C status."""
    L = lib()
    F, ncol = _fields_all(fields)
    P = make_params(grid, hp, 0.0, ncol)
    keep = _species(P, ncol, species)
    n = len(initial)
    ini = (OraFluxes * n)(*initial)
    ref = (OraFluxes * n)(*refined)
    rc = L.ora_correct_fluxes(C.byref(P), F, n, ini, ref,
                              (C.c_longlong * 3)(*[int(x) for x in ggs]))
    for k in range(n):
        refined[k] = ref[k]
    return rc


def correct_fluxes_sublings(grid, hp, fields, own, refined, ggs, level_dims, periodic,
                            species=None):
    """The SUBling calls of grid::CorrectForRefinedFluxes on host fields, in place.  own:
    OraFluxes of the grid's own boundary; refined: list of OraFluxes (updated where a
    correction is undone).  Returns the C status."""
    L = lib()
    F, ncol = _fields_all(fields)
    P = make_params(grid, hp, 0.0, ncol)
    keep = _species(P, ncol, species)
    n = len(refined)
    ref = (OraFluxes * n)(*refined)
    rc = L.ora_correct_fluxes_sublings(C.byref(P), F, n, C.byref(own), ref,
                                       (C.c_longlong * 3)(*[int(x) for x in ggs]),
                                       (C.c_longlong * 3)(*[int(x) for x in level_dims]),
                                       (C.c_int * 3)(*[int(bool(x)) for x in periodic]))
    for k in range(n):
        refined[k] = ref[k]
    return rc
