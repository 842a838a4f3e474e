"""ctypes binding of the C ABI in include/ppm_b200.h (libppm_b200.so).

This is the Python mirror of the reference's call site: ``Context.solve_ppm_de``
takes what ``grid::SolvePPM_DE`` takes (cycle number, subgrid flux boxes, the
grid's global start) and fields in Enzo's BaryonField layout, either as host
numpy arrays (copied in and out inside the call) or as device tensors.
The library is required: there is no CPU fallback on this path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import build as _build

OK = 0
ERR_UNSUPPORTED = -1
ERR_INVALID = -2
ERR_CUDA = -3
ERR_NEGATIVE = -4
ERR_NONFINITE = -5
ERR_TOO_LARGE = -6
ERR_TIMEOUT = -7
MEM_HOST = 0
MEM_DEVICE = 1
RIEMANN_TWOSHOCK = 5
RIEMANN_HLL = 1
RIEMANN_HLLC = 4
RECONSTRUCTION_PPM = 1

EXPORTS = (
    "ppm_b200_create", "ppm_b200_destroy", "ppm_b200_solve_ppm_de", "ppm_b200_euler_sweep",
    "ppm_b200_compute_pressure", "ppm_b200_compute_timestep", "ppm_b200_set_boundary",
    "ppm_b200_synchronize", "ppm_b200_launch_count", "ppm_b200_error_string",
    "ppm_b200_version", "ppm_b200_profile", "ppm_b200_profile_read",
    "ppm_b200_euler_sweep_static", "ppm_b200_solve_level", "ppm_b200_set_graphs",
    "ppm_b200_compute_timestep_level", "ppm_b200_set_boundary_level",
    "ppm_b200_copy_zones_level", "ppm_b200_correct_fluxes", "ppm_b200_debug_tma_stall",
    "ppm_b200_correct_fluxes_sublings",
    "ppm_b200_profile_stages", "ppm_b200_set_guess", "ppm_b200_riemann_log",
    "ppm_b200_riemann_log_count", "ppm_b200_guess_features", "ppm_b200_guess_grad",
    "ppm_b200_guess_adam", "ppm_b200_guess_eval", "ppm_b200_expansion_terms",
    "ppm_b200_expansion_terms_level", "ppm_b200_set_cfl", "ppm_b200_abi_check",
    "ppm_b200_set_level_config", "ppm_b200_get_level_config", "ppm_b200_autotune_level",
    "ppm_b200_device_bytes", "ppm_b200_set_sweep_mode",
)

GUESS_WEIGHTS = 4673  # W1[6][64] b1[64] W2[64][64] b2[64] w3[64] b3
BC_CODES = {"periodic": 0, "outflow": 1, "none": 2}  # ppm_b200_set_boundary bc_type

# the five kernels of one sweep, in launch order (ppm_b200_profile_stages)
SWEEP_STAGES = ("reconstruct_dpu", "reconstruct_vwge", "riemann", "update", "fallback")

_dp = C.POINTER(C.c_double)


class Params(C.Structure):
    _fields_ = [
        ("gamma", C.c_double), ("dt", C.c_double), ("eta1", C.c_double), ("eta2", C.c_double),
        ("small_rho", C.c_double), ("tiny_number", C.c_double), ("min_support", C.c_double),
        ("dual_energy", C.c_int), ("gravity", C.c_int), ("pressure_free", C.c_int),
        ("riemann_solver", C.c_int), ("riemann_fallback", C.c_int), ("reconstruction", C.c_int),
        ("steepening", C.c_int), ("flattening", C.c_int), ("diffusion", C.c_int),
        ("conservative_rec", C.c_int), ("positive_rec", C.c_int), ("eos_type", C.c_int),
        ("number_of_colours", C.c_int), ("learned_guess", C.c_int),
        ("dt_device", C.c_void_p), ("colour_species", C.c_void_p),
        ("eos_sound_speed", C.c_double), ("reserved", C.c_int * 2),
    ]


class GridDesc(C.Structure):
    _fields_ = [
        ("rank", C.c_int), ("dims", C.c_int * 3), ("start", C.c_int * 3), ("end", C.c_int * 3),
        ("density", C.c_void_p), ("total_energy", C.c_void_p), ("velocity", C.c_void_p * 3),
        ("gas_energy", C.c_void_p), ("acceleration", C.c_void_p * 3),
        ("cell_width", C.c_void_p * 3), ("colours", C.c_void_p),
    ]


class Fluxes(C.Structure):
    _fields_ = [
        ("left_start", (C.c_longlong * 3) * 3), ("left_end", (C.c_longlong * 3) * 3),
        ("right_start", (C.c_longlong * 3) * 3), ("right_end", (C.c_longlong * 3) * 3),
        ("left", (C.c_void_p * 3) * 6), ("right", (C.c_void_p * 3) * 6),
        ("colour_left", C.c_void_p), ("colour_right", C.c_void_p),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("interfaces", C.c_longlong), ("newton_iters", C.c_longlong),
        ("newton_hist", C.c_longlong * 8), ("fallbacks", C.c_longlong),
        ("fatal_cells", C.c_longlong), ("guess_rejected", C.c_longlong),
        ("warp_newton_iters", C.c_longlong), ("warps", C.c_longlong),
    ]

    def as_dict(self):
        return {
            "interfaces": int(self.interfaces), "newton_iters": int(self.newton_iters),
            "newton_hist": [int(x) for x in self.newton_hist], "fallbacks": int(self.fallbacks),
            "fatal_cells": int(self.fatal_cells), "guess_rejected": int(self.guess_rejected),
            "warp_newton_iters": int(self.warp_newton_iters), "warps": int(self.warps),
        }


class LevelConfig(C.Structure):
    _fields_ = [("schedule", C.c_int), ("riemann_threads", C.c_int * 4),
                ("persistent", C.c_int * 4), ("class_cells", C.c_longlong * 2),
                ("max_scratch_bytes", C.c_longlong)]

    def as_dict(self):
        return {"schedule": LEVEL_SCHEDULES[self.schedule],
                "riemann_threads": list(self.riemann_threads),
                "persistent": list(self.persistent),
                "class_cells": list(self.class_cells),
                "max_scratch_bytes": int(self.max_scratch_bytes)}


class LevelTuning(C.Structure):
    _fields_ = [("class_grids", C.c_int * 3), ("class_active", C.c_longlong * 3),
                ("class_ms", (C.c_double * 6) * 3), ("batched_ms", C.c_double * 6),
                ("classes_ms", C.c_double), ("chosen", LevelConfig)]

    def as_dict(self):
        cand = [f"{t} faces/block{' persistent' if pers else ''}" for t in (64, 128, 256)
                for pers in (0, 1)]
        return {"candidates": cand,
                "class_grids": list(self.class_grids),
                "class_active_cells": list(self.class_active),
                "class_ms": [list(r) for r in self.class_ms],
                "batched_ms": list(self.batched_ms), "classes_ms": self.classes_ms,
                "chosen": self.chosen.as_dict()}


# ppm_b200_level_config.schedule
LEVEL_SCHEDULES = {0: "batched", 1: "classes", 2: "per_grid"}


class PPMError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__(f"{what}: ppm_b200 error {code} ({error_string(code)})")


_libs = {}


def default_variant() -> str:
    """The build variant loaded when none is named: $PPM_B200_VARIANT, else "exact"
    (bit-identical to the oracle); "fast" is the tolerance-mode build."""
    v = os.environ.get("PPM_B200_VARIANT", "exact")
    if v not in _build.VARIANTS:
        raise ValueError(f"PPM_B200_VARIANT={v!r}: expected one of {sorted(_build.VARIANTS)}")
    return v


def library_path(variant: str | None = None) -> Path:
    """The shared library of a build variant: $PPM_B200_LIB overrides the exact build's
    path, otherwise the in-tree build."""
    variant = variant or default_variant()
    env = os.environ.get("PPM_B200_LIB")
    if env and variant == "exact":
        return Path(env)
    return _build.VARIANTS[variant]["lib"]


def lib(build_if_missing: bool = True, variant: str | None = None):
    """Load the library of a build variant (building it when missing and nvcc is
    available).  Each variant is its own handle; both can be loaded at once."""
    variant = variant or default_variant()
    if variant in _libs:
        return _libs[variant]
    path = library_path(variant)
    if not path.exists():
        if not build_if_missing or path != _build.VARIANTS[variant]["lib"]:
            raise RuntimeError(f"{path} is missing; run python -m ppm_b200.build")
        _build.build(variant=variant)
    L = C.CDLL(str(path))
    vp = C.c_void_p
    L.ppm_b200_create.argtypes = [C.c_int, vp, C.POINTER(vp)]
    L.ppm_b200_destroy.argtypes = [vp]
    L.ppm_b200_solve_ppm_de.argtypes = [vp, C.POINTER(Params), C.c_int, C.POINTER(GridDesc),
                                        C.c_int, C.c_int, C.POINTER(Fluxes),
                                        C.POINTER(C.c_longlong), C.POINTER(Stats)]
    L.ppm_b200_euler_sweep.argtypes = [vp, C.c_int, C.POINTER(Params), C.POINTER(GridDesc),
                                       vp, C.c_int, C.c_int, C.POINTER(Fluxes),
                                       C.POINTER(C.c_longlong), C.POINTER(Stats)]
    L.ppm_b200_compute_pressure.argtypes = [vp, C.POINTER(Params), C.POINTER(GridDesc), vp,
                                            C.c_int]
    L.ppm_b200_compute_timestep.argtypes = [vp, C.POINTER(Params), C.POINTER(GridDesc), C.c_int,
                                            C.c_double, C.c_double, C.POINTER(C.c_double),
                                            vp, C.POINTER(C.c_double)]
    L.ppm_b200_set_boundary.argtypes = [vp, C.POINTER(GridDesc), C.c_int, C.c_int,
                                        C.POINTER(C.c_int)]
    L.ppm_b200_synchronize.argtypes = [vp, C.POINTER(Stats)]
    L.ppm_b200_launch_count.argtypes = [vp]
    L.ppm_b200_launch_count.restype = C.c_longlong
    L.ppm_b200_error_string.argtypes = [C.c_int]
    L.ppm_b200_error_string.restype = C.c_char_p
    L.ppm_b200_version.argtypes = []
    L.ppm_b200_euler_sweep_static.argtypes = [C.c_int, C.POINTER(Params), C.POINTER(GridDesc),
                                              vp, C.POINTER(GridDesc), vp, C.POINTER(Stats)]
    L.ppm_b200_profile.argtypes = [vp, C.c_int]
    L.ppm_b200_profile_stages.argtypes = [vp, C.POINTER(C.c_double)]
    L.ppm_b200_solve_level.argtypes = [vp, C.POINTER(Params), C.c_int, C.POINTER(GridDesc),
                                       C.c_int, C.POINTER(Stats)]
    L.ppm_b200_set_graphs.argtypes = [vp, C.c_int]
    L.ppm_b200_set_level_config.argtypes = [vp, C.POINTER(LevelConfig)]
    L.ppm_b200_device_bytes.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.ppm_b200_set_sweep_mode.argtypes = [vp, C.c_int]
    L.ppm_b200_get_level_config.argtypes = [vp, C.POINTER(LevelConfig)]
    L.ppm_b200_autotune_level.argtypes = [vp, C.POINTER(Params), C.c_int, C.POINTER(GridDesc),
                                          C.c_int, C.POINTER(LevelTuning)]
    fp = C.POINTER(C.c_float)
    L.ppm_b200_set_guess.argtypes = [vp, vp]
    L.ppm_b200_set_cfl.argtypes = [vp, vp, C.c_double, C.c_double, C.POINTER(C.c_double)]
    L.ppm_b200_expansion_terms.argtypes = [vp, C.POINTER(Params), C.POINTER(GridDesc),
                                           C.POINTER(GridDesc), C.c_double, C.c_double,
                                           C.c_double, C.c_int]
    L.ppm_b200_expansion_terms_level.argtypes = [vp, C.POINTER(Params), C.POINTER(GridDesc),
                                                 C.POINTER(GridDesc), C.c_int, C.c_double,
                                                 C.c_double, C.c_double]
    L.ppm_b200_riemann_log.argtypes = [vp, vp, C.c_longlong, C.c_int]
    L.ppm_b200_riemann_log_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.ppm_b200_guess_features.argtypes = [vp, vp, C.c_longlong, C.c_double, C.c_double, vp]
    L.ppm_b200_guess_grad.argtypes = [vp, vp, vp, vp, C.c_longlong, vp, vp]
    L.ppm_b200_guess_adam.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_float, C.c_float,
                                      C.c_float, C.c_float]
    L.ppm_b200_guess_eval.argtypes = [vp, vp, C.c_longlong, vp]
    L.ppm_b200_compute_timestep_level.argtypes = [vp, C.POINTER(Params), C.POINTER(GridDesc),
                                                  C.c_int, C.c_double, C.c_double,
                                                  C.POINTER(C.c_double), vp,
                                                  C.POINTER(C.c_double)]
    L.ppm_b200_copy_zones_level.argtypes = [vp, C.POINTER(GridDesc), C.c_int,
                                            C.POINTER(C.c_longlong), C.c_longlong * 3,
                                            C.c_int * 3, C.c_int, C.c_int]
    L.ppm_b200_copy_zones_level.restype = C.c_int
    L.ppm_b200_correct_fluxes.argtypes = [vp, C.POINTER(Params), C.POINTER(GridDesc), C.c_int,
                                          C.c_int, C.POINTER(Fluxes), C.POINTER(Fluxes),
                                          C.c_longlong * 3]
    L.ppm_b200_correct_fluxes.restype = C.c_int
    L.ppm_b200_correct_fluxes_sublings.argtypes = [vp, C.POINTER(Params), C.POINTER(GridDesc),
                                                   C.c_int, C.c_int, C.POINTER(Fluxes),
                                                   C.POINTER(Fluxes), C.c_longlong * 3,
                                                   C.c_longlong * 3, C.c_int * 3]
    L.ppm_b200_correct_fluxes_sublings.restype = C.c_int
    L.ppm_b200_debug_tma_stall.argtypes = [vp, C.c_int]
    L.ppm_b200_debug_tma_stall.restype = C.c_int
    L.ppm_b200_set_boundary_level.argtypes = [vp, C.POINTER(GridDesc), C.c_int, C.c_int,
                                              C.c_int, C.POINTER(C.c_int)]
    L.ppm_b200_profile_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
    for name in EXPORTS:
        fn = getattr(L, name)
        if name not in ("ppm_b200_launch_count", "ppm_b200_error_string"):
            fn.restype = C.c_int
    _libs[variant] = L
    return L


def error_string(code: int) -> str:
    return lib().ppm_b200_error_string(int(code)).decode()


def _addr(x):
    """Address of a host numpy array or a device tensor (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        assert x.dtype == np.float64 and x.flags["C_CONTIGUOUS"], "float64 C-contiguous required"
        return x.ctypes.data
    # torch tensor
    assert x.dtype.__str__() == "torch.float64" and x.is_contiguous()
    return x.data_ptr()


def make_params(hp, dt, learned_guess=False, dt_device=None) -> Params:
    P = Params()
    P.gamma = hp.gamma
    P.dt = float(dt)
    P.eta1 = hp.eta1
    P.eta2 = hp.eta2
    P.small_rho = hp.small_rho
    P.tiny_number = hp.tiny_number
    P.min_support = hp.min_support
    P.dual_energy = int(hp.dual)
    P.gravity = int(hp.gravity)
    P.pressure_free = int(hp.pressure_free)
    P.riemann_solver = int(getattr(hp, "riemann", RIEMANN_TWOSHOCK))
    P.riemann_fallback = int(hp.fallback)
    P.reconstruction = RECONSTRUCTION_PPM
    P.steepening = int(getattr(hp, "steepen", 0))
    P.flattening = int(getattr(hp, "flatten", 0))
    P.learned_guess = int(learned_guess)
    P.eos_type = int(getattr(hp, "eos_type", 0))
    P.eos_sound_speed = float(getattr(hp, "eos_sound_speed", 2.65e4))
    P.dt_device = _addr(dt_device) if dt_device is not None else None
    return P


def colour_names(fields):
    """Colour fields of a field dict: keys col0, col1, ... in colnum[] order."""
    n = 0
    while f"col{n}" in fields:
        n += 1
    return [f"col{k}" for k in range(n)]


def make_grid(grid, fields, accel=None):
    """Returns (GridDesc, keepalive list).  Colour fields: keys col0, col1, ..."""
    G = GridDesc()
    G.rank = grid.rank
    for d in range(3):
        G.dims[d] = grid.dims[d]
        G.start[d] = grid.start[d]
        G.end[d] = grid.end[d]
    G.density = _addr(fields["d"])
    G.total_energy = _addr(fields["te"])
    for d, n in enumerate(("v1", "v2", "v3")):
        G.velocity[d] = _addr(fields.get(n)) if d < grid.rank else None
    G.gas_energy = _addr(fields.get("ge"))
    keep = []
    for d in range(3):
        if accel is not None and d < len(accel) and accel[d] is not None:
            G.acceleration[d] = _addr(accel[d])
        cw = np.ascontiguousarray(grid.cellwidth[d], dtype=np.float64)
        keep.append(cw)
        G.cell_width[d] = cw.ctypes.data
    cols = colour_names(fields)
    if cols:
        arr = (C.c_void_p * len(cols))(*[_addr(fields[n]) for n in cols])
        keep.append(arr)
        G.colours = C.cast(arr, C.c_void_p)
    return G, keep


def make_fluxes(box, keep=None):
    """box: dict with left_start/left_end/right_start/right_end (3x3) and arrays
    left[slot][dim], right[slot][dim] (numpy, may be None), and optionally
    colour_left[n][dim] / colour_right[n][dim].  Returns Fluxes; keep (a list) holds the
    colour pointer arrays alive."""
    F = Fluxes()
    for key in ("left_start", "left_end", "right_start", "right_end"):
        arr = getattr(F, key)
        for i in range(3):
            for j in range(3):
                arr[i][j] = int(box[key][i][j])
    for side in ("left", "right"):
        arr = getattr(F, side)
        for s in range(6):
            for d in range(3):
                a = box[side][s][d]
                arr[s][d] = _addr(a) if a is not None else None
    for side in ("colour_left", "colour_right"):
        rows = box.get(side)
        if not rows:
            continue
        ptrs = (C.c_void_p * (3 * len(rows)))()
        for n, row in enumerate(rows):
            for d in range(3):
                a = row[d]
                ptrs[3 * n + d] = _addr(a) if a is not None else None
        if keep is not None:
            keep.append(ptrs)
        setattr(F, side, C.cast(ptrs, C.c_void_p))
    return F


def euler_sweep_static(dim, grid, hp, dt, fields_in, pressure, fields_out, stream=None,
                       accel=None):
    """ppm_b200_euler_sweep_static: one sweep with no device allocation.

    For callers that cannot allocate device memory when they advance a grid (a
    memory arena owns the device, or the call happens where an allocation could
    synchronise).  fields_in / fields_out / pressure are device tensors owned by the
    caller; the sweep's scratch is a fixed array inside the library (grids up to
    64^3 active cells).  Returns (rc, stats dict); no exception on a nonzero rc."""
    L = lib()
    P = make_params(hp, dt)
    Gi, keep_i = make_grid(grid, fields_in, accel)
    Go, keep_o = make_grid(grid, fields_out)
    st = Stats()
    rc = L.ppm_b200_euler_sweep_static(int(dim), C.byref(P), C.byref(Gi), _addr(pressure),
                                       C.byref(Go), stream, C.byref(st))
    return rc, st.as_dict()


class Context:
    """One ppm_b200_context (one per rank / device)."""

    def __init__(self, device: int = 0, stream=None, variant: str | None = None):
        self.variant = variant or default_variant()
        self.L = lib(variant=self.variant)
        h = C.c_void_p()
        rc = self.L.ppm_b200_create(int(device), stream, C.byref(h))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ppm_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launches(self) -> int:
        return int(self.L.ppm_b200_launch_count(self.h))

    def solve_ppm_de(self, grid, hp, dt, cycle, fields, memory=MEM_HOST, accel=None,
                     subgrids=None, ggs=(0, 0, 0), want_stats=True, learned_guess=False,
                     dt_device=None, check=True):
        P = make_params(hp, dt, learned_guess, dt_device)
        P.number_of_colours = len(colour_names(fields))
        G, keep = make_grid(grid, fields, accel)
        st = Stats()
        nsub = 0 if not subgrids else len(subgrids)
        sub = None
        if nsub:
            sub = (Fluxes * nsub)(*[make_fluxes(b, keep) for b in subgrids])
        g = (C.c_longlong * 3)(*[int(x) for x in ggs])
        rc = self.L.ppm_b200_solve_ppm_de(self.h, C.byref(P), int(cycle), C.byref(G), int(memory),
                                          nsub, sub, g, C.byref(st) if want_stats else None)
        if check and rc != OK:
            raise PPMError(rc, "ppm_b200_solve_ppm_de")
        return rc, st.as_dict()

    def euler_sweep(self, dim, grid, hp, dt, fields, pressure, memory=MEM_HOST, accel=None,
                    check=True, learned_guess=False):
        P = make_params(hp, dt, learned_guess)
        P.number_of_colours = len(colour_names(fields))
        G, keep = make_grid(grid, fields, accel)
        st = Stats()
        g = (C.c_longlong * 3)(0, 0, 0)
        rc = self.L.ppm_b200_euler_sweep(self.h, int(dim), C.byref(P), C.byref(G),
                                         _addr(pressure), int(memory), 0, None, g, C.byref(st))
        if check and rc != OK:
            raise PPMError(rc, "ppm_b200_euler_sweep")
        return rc, st.as_dict()

    def compute_pressure(self, grid, hp, fields, out, memory=MEM_HOST):
        P = make_params(hp, 0.0)
        G, keep = make_grid(grid, fields)
        rc = self.L.ppm_b200_compute_pressure(self.h, C.byref(P), C.byref(G), _addr(out),
                                              int(memory))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_compute_pressure")

    def compute_timestep(self, grid, hp, fields, memory=MEM_HOST, courant=None, aye=1.0,
                         vgrid=(0.0, 0.0, 0.0), dt_device=None, want_host=True):
        P = make_params(hp, 0.0)
        G, keep = make_grid(grid, fields)
        vg = (C.c_double * 3)(*vgrid)
        out = C.c_double(0.0)
        cf = hp.cfl if courant is None else courant
        rc = self.L.ppm_b200_compute_timestep(self.h, C.byref(P), C.byref(G), int(memory),
                                              float(cf), float(aye), vg,
                                              _addr(dt_device) if dt_device is not None else None,
                                              C.byref(out) if want_host else None)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_compute_timestep")
        return out.value

    def set_boundary(self, grid, fields, dual, bc=("periodic",) * 3):
        """Ghost fill of the hydro fields and of the colours (keys col0, col1, ...)."""
        G, keep = make_grid(grid, fields)
        codes = (C.c_int * 3)(*[BC_CODES[b] for b in bc])
        rc = self.L.ppm_b200_set_boundary(self.h, C.byref(G), int(bool(dual)),
                                          len(colour_names(fields)), codes)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_set_boundary")

    def _level(self, grids, fields_list, accels=None):
        """GridDesc array for a level: grids[k] with device fields fields_list[k]."""
        n = len(grids)
        arr = (GridDesc * n)()
        keep = []
        for k in range(n):
            acc = accels[k] if accels is not None else None
            G, kp = make_grid(grids[k], fields_list[k], acc)
            arr[k] = G
            keep.append(kp)
        return arr, keep

    def solve_level(self, grids, hp, dt, cycle, fields_list, accels=None, want_stats=False,
                    dt_device=None, check=True, learned_guess=False):
        """SolvePPM_DE of every grid of a level in one batch (device tensors)."""
        P = make_params(hp, dt, learned_guess, dt_device)
        P.number_of_colours = len(colour_names(fields_list[0])) if fields_list else 0
        arr, keep = self._level(grids, fields_list, accels)
        st = Stats()
        rc = self.L.ppm_b200_solve_level(self.h, C.byref(P), int(cycle), arr, len(grids),
                                         C.byref(st) if want_stats else None)
        if check and rc != OK:
            raise PPMError(rc, "ppm_b200_solve_level")
        return rc, st.as_dict()

    def set_sweep_mode(self, mode):
        """"split" (reconstruction and Riemann kernels over an interface-state scratch) or
        "fused" (one face kernel); the same results."""
        rc = self.L.ppm_b200_set_sweep_mode(self.h, {"split": 0, "fused": 1}[mode])
        if rc != OK:
            raise PPMError(rc, "ppm_b200_set_sweep_mode")

    def device_bytes(self):
        n = C.c_longlong(0)
        rc = self.L.ppm_b200_device_bytes(self.h, C.byref(n))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_device_bytes")
        return int(n.value)

    def level_config(self):
        c = LevelConfig()
        rc = self.L.ppm_b200_get_level_config(self.h, C.byref(c))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_get_level_config")
        return c

    def set_level_config(self, schedule=None, riemann_threads=None, persistent=None,
                         class_cells=None, max_scratch_bytes=None):
        """Change the level schedule; arguments left at None keep their current value.
        schedule: "batched", "classes" or "per_grid"; riemann_threads / persistent: four
        entries (size classes 0-2, then the batched schedule) or one for all."""
        c = self.level_config()
        if schedule is not None:
            c.schedule = {v: k for k, v in LEVEL_SCHEDULES.items()}[schedule]
        for name, val in (("riemann_threads", riemann_threads), ("persistent", persistent)):
            if val is not None:
                vals = [val] * 4 if isinstance(val, int) else list(val)
                arr = getattr(c, name)
                for k in range(4):
                    arr[k] = int(vals[k])
        if class_cells is not None:
            c.class_cells[0], c.class_cells[1] = (int(x) for x in class_cells)
        if max_scratch_bytes is not None:
            c.max_scratch_bytes = int(max_scratch_bytes)
        rc = self.L.ppm_b200_set_level_config(self.h, C.byref(c))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_set_level_config")
        return c.as_dict()

    def autotune_level(self, grids, hp, fields_list, dt, cycle=0, accels=None,
                       dt_device=None):
        """Runs the per-size-class autotuner on copies of the level's fields (time step dt,
        or *dt_device) and keeps its choice; returns its report."""
        P = make_params(hp, dt, False, dt_device)
        arr, keep = self._level(grids, fields_list, accels)
        t = LevelTuning()
        rc = self.L.ppm_b200_autotune_level(self.h, C.byref(P), int(cycle), arr, len(grids),
                                            C.byref(t))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_autotune_level")
        return t.as_dict()

    def set_graphs(self, enable=True):
        rc = self.L.ppm_b200_set_graphs(self.h, int(bool(enable)))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_set_graphs")

    def compute_timestep_level(self, grids, hp, fields_list, courant=None, aye=1.0,
                               vgrid=(0.0, 0.0, 0.0), dt_device=None, want_host=True):
        P = make_params(hp, 0.0)
        arr, keep = self._level(grids, fields_list)
        vg = (C.c_double * 3)(*vgrid)
        out = C.c_double(0.0)
        cf = hp.cfl if courant is None else courant
        rc = self.L.ppm_b200_compute_timestep_level(
            self.h, C.byref(P), arr, len(grids), float(cf), float(aye), vg,
            _addr(dt_device) if dt_device is not None else None,
            C.byref(out) if want_host else None)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_compute_timestep_level")
        return out.value

    def set_boundary_level(self, grids, fields_list, dual, bc=("periodic",) * 3):
        arr, keep = self._level(grids, fields_list)
        codes = (C.c_int * 3)(*[BC_CODES[b] for b in bc])
        nc = len(colour_names(fields_list[0])) if fields_list else 0
        rc = self.L.ppm_b200_set_boundary_level(self.h, arr, len(grids), int(bool(dual)), nc,
                                                codes)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_set_boundary_level")

    def debug_tma_stall(self, extra_bytes):
        """Test hook: make the x sweep's TMA chunk waits run out (0 restores)."""
        rc = self.L.ppm_b200_debug_tma_stall(self.h, int(extra_bytes))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_debug_tma_stall")

    @staticmethod
    def _species(P, fields, species, keep):
        """Colours (keys col0, ...) and the flags of those that keep their density
        fraction under flux correction (params.colour_species)."""
        P.number_of_colours = len(colour_names(fields)) if species else 0
        if species:
            arr = (C.c_int * len(species))(*[int(bool(x)) for x in species])
            keep.append(arr)
            P.colour_species = C.cast(arr, C.c_void_p)

    def correct_fluxes(self, grid, hp, fields, initial, refined, ggs, memory=MEM_HOST,
                       species=None):
        """grid::CorrectForRefinedFluxes for the proper subgrids of one grid.  initial /
        refined: lists of flux boxes (dicts as for make_fluxes, host numpy arrays); the
        refined arrays are updated in place where a correction is undone.  species: one
        flag per colour field (keys col0, ...): nonzero keeps its density fraction."""
        P = make_params(hp, 0.0)
        G, keep = make_grid(grid, fields)
        self._species(P, fields, species, keep)
        n = len(initial)
        ini = (Fluxes * n)(*[make_fluxes(b) for b in initial])
        ref = (Fluxes * n)(*[make_fluxes(b) for b in refined])
        g = (C.c_longlong * 3)(*[int(x) for x in ggs])
        rc = self.L.ppm_b200_correct_fluxes(self.h, C.byref(P), C.byref(G), int(memory), n, ini,
                                            ref, g)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_correct_fluxes")

    def correct_fluxes_sublings(self, grid, hp, fields, own, refined, ggs, level_dims, periodic,
                                memory=MEM_HOST, species=None):
        """The SUBling calls of grid::CorrectForRefinedFluxes for one grid: own = its own
        boundary flux box, refined = the sibling subgrids' projected flux boxes (dicts as
        for make_fluxes; refined arrays updated where a correction is undone)."""
        P = make_params(hp, 0.0)
        G, keep = make_grid(grid, fields)
        self._species(P, fields, species, keep)
        n = len(refined)
        ow = make_fluxes(own)
        ref = (Fluxes * n)(*[make_fluxes(b) for b in refined])
        g = (C.c_longlong * 3)(*[int(x) for x in ggs])
        ld = (C.c_longlong * 3)(*[int(x) for x in level_dims])
        per = (C.c_int * 3)(*[int(bool(x)) for x in periodic])
        rc = self.L.ppm_b200_correct_fluxes_sublings(self.h, C.byref(P), C.byref(G), int(memory),
                                                     n, C.byref(ow), ref, g, ld, per)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_correct_fluxes_sublings")

    def copy_zones_level(self, grids, fields_list, left, domain, periodic, dual):
        """grid::CopyZonesFromGrid over a level (siblings and periodic images) on device
        fields.  left[k]: level index of grid k's first zone (ghosts included) per axis;
        domain: the level's extent in zones; periodic: per-axis flags."""
        arr, keep = self._level(grids, fields_list)
        lf = (C.c_longlong * (3 * len(grids)))(*[int(v) for l in left for v in list(l) + [0] * (3 - len(l))])
        dom = (C.c_longlong * 3)(*[int(v) for v in list(domain) + [1] * (3 - len(domain))])
        per = (C.c_int * 3)(*[int(bool(v)) for v in list(periodic) + [0] * (3 - len(periodic))])
        nc = len(colour_names(fields_list[0])) if fields_list else 0
        rc = self.L.ppm_b200_copy_zones_level(self.h, arr, len(grids), lf, dom, per,
                                              int(bool(dual)), nc)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_copy_zones_level")

    def profile(self, enable=True):
        self.L.ppm_b200_profile(self.h, int(bool(enable)))

    def profile_read(self):
        ms = C.c_double(0.0)
        n = C.c_longlong(0)
        rc = self.L.ppm_b200_profile_read(self.h, C.byref(ms), C.byref(n))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_profile_read")
        return ms.value, n.value

    def set_cfl(self, dt_device, courant=1.0, aye=1.0, vgrid=(0.0, 0.0, 0.0)):
        """Fold the next cycle's time step into later solves (dt_device: float64 device
        tensor of one element, or None to stop)."""
        vg = (C.c_double * 3)(*vgrid)
        rc = self.L.ppm_b200_set_cfl(self.h, dt_device.data_ptr() if dt_device is not None
                                     else None, float(courant), float(aye), vg)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_set_cfl")

    # ---- comoving expansion terms
    def expansion_terms(self, grid, hp, fields, old, time, old_time, coefficient,
                        memory=MEM_HOST):
        """grid::ComovingExpansionTerms (in place); old: fields at OldTime or None."""
        P = make_params(hp, 0.0)
        G, keep = make_grid(grid, fields)
        Og, keep2 = make_grid(grid, old) if old is not None else (None, None)
        rc = self.L.ppm_b200_expansion_terms(self.h, C.byref(P), C.byref(G),
                                             C.byref(Og) if Og is not None else None,
                                             float(time), float(old_time), float(coefficient),
                                             int(memory))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_expansion_terms")

    def expansion_terms_level(self, grids, hp, fields_list, olds, time, old_time,
                              coefficient):
        P = make_params(hp, 0.0)
        arr, keep = self._level(grids, fields_list)
        oarr, keep2 = self._level(grids, olds) if olds is not None else (None, None)
        rc = self.L.ppm_b200_expansion_terms_level(self.h, C.byref(P), arr, oarr, len(grids),
                                                   float(time), float(old_time),
                                                   float(coefficient))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_expansion_terms_level")

    # ---- learned Newton start
    def set_guess(self, weights):
        """weights: host float32 array of GUESS_WEIGHTS values (None clears)."""
        if weights is None:
            rc = self.L.ppm_b200_set_guess(self.h, None)
        else:
            w = np.ascontiguousarray(weights, dtype=np.float32)
            assert w.size == GUESS_WEIGHTS
            rc = self.L.ppm_b200_set_guess(self.h, w.ctypes.data)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_set_guess")

    def riemann_log(self, records, stride):
        """records: device float64 tensor (capacity, 8) or None to stop."""
        if records is None:
            rc = self.L.ppm_b200_riemann_log(self.h, None, 0, 0)
        else:
            rc = self.L.ppm_b200_riemann_log(self.h, records.data_ptr(), records.shape[0],
                                             int(stride))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_riemann_log")

    def riemann_log_count(self):
        n = C.c_longlong(0)
        rc = self.L.ppm_b200_riemann_log_count(self.h, C.byref(n))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_riemann_log_count")
        return n.value

    def guess_features(self, records, n, gamma, pmin, samples):
        rc = self.L.ppm_b200_guess_features(self.h, records.data_ptr(), int(n), float(gamma),
                                            float(pmin), samples.data_ptr())
        if rc != OK:
            raise PPMError(rc, "ppm_b200_guess_features")

    def guess_grad(self, weights, samples, index, n, grad, loss):
        rc = self.L.ppm_b200_guess_grad(self.h, weights.data_ptr(), samples.data_ptr(),
                                        index.data_ptr() if index is not None else None,
                                        int(n), grad.data_ptr(), loss.data_ptr())
        if rc != OK:
            raise PPMError(rc, "ppm_b200_guess_grad")

    def guess_adam(self, weights, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        rc = self.L.ppm_b200_guess_adam(self.h, weights.data_ptr(), grad.data_ptr(),
                                        m.data_ptr(), v.data_ptr(), int(step), float(lr),
                                        float(beta1), float(beta2), float(eps))
        if rc != OK:
            raise PPMError(rc, "ppm_b200_guess_adam")

    def guess_eval(self, features, n, y):
        rc = self.L.ppm_b200_guess_eval(self.h, features.data_ptr(), int(n), y.data_ptr())
        if rc != OK:
            raise PPMError(rc, "ppm_b200_guess_eval")

    def profile_stages(self):
        """{stage: ms} of the five sweep kernels, summed over the last profile_read."""
        arr = (C.c_double * 5)()
        rc = self.L.ppm_b200_profile_stages(self.h, arr)
        if rc != OK:
            raise PPMError(rc, "ppm_b200_profile_stages")
        return dict(zip(SWEEP_STAGES, list(arr)))

    def synchronize(self):
        st = Stats()
        rc = self.L.ppm_b200_synchronize(self.h, C.byref(st))
        return rc, st.as_dict()
