"""Subgrid flux boxes for the flux-correction tests (struct fluxes, Fluxes.h:29-37): a
subgrid covering zones lo..hi (this grid's zone indices) of a coarse grid whose first
zone has global index ggs.  Flux values are seeded; the refined ones are the initial
ones plus a perturbation, some of them large enough to drive a density or an energy
non-positive (the reference's undo path)."""
import ctypes as C

import numpy as np

import oracle as O


def flux_box(lo, hi, ggs, rng, dual, rank=3, refined_of=None, kick=0.0):
    b = {"left_start": [[0] * 3 for _ in range(3)], "left_end": [[0] * 3 for _ in range(3)],
         "right_start": [[0] * 3 for _ in range(3)], "right_end": [[0] * 3 for _ in range(3)],
         "left": [[None] * 3 for _ in range(6)], "right": [[None] * 3 for _ in range(6)]}
    for dim in range(rank):
        for j in range(rank):
            s, e = lo[j] + ggs[j], hi[j] + ggs[j]
            b["left_start"][dim][j] = s if j != dim else lo[j] + ggs[j]
            b["left_end"][dim][j] = e if j != dim else lo[j] + ggs[j]
            b["right_start"][dim][j] = s if j != dim else hi[j] + ggs[j]
            b["right_end"][dim][j] = e if j != dim else hi[j] + ggs[j]
        size = 1
        for j in range(rank):
            if j != dim:
                size *= hi[j] - lo[j] + 1
        slots = [0, 1] + [2 + v for v in range(rank)] + ([5] if dual else [])
        for s_ in slots:
            for side in ("left", "right"):
                if refined_of is None:
                    # initial: flux-sized values (fluxes are dt/dx-scaled, a fraction of a cell)
                    b[side][s_][dim] = 0.05 * rng.standard_normal(size)
                else:
                    base = refined_of[side][s_][dim]
                    v = base + 0.01 * rng.standard_normal(size)
                    if kick:  # a few large refined fluxes: negative corrected states
                        m = rng.random(size) < 0.15
                        v[m] += kick * np.sign(rng.standard_normal(m.sum()))
                    b[side][s_][dim] = v
    return b


def copy_box(b):
    out = {k: [list(r) for r in b[k]] for k in ("left_start", "left_end", "right_start",
                                                "right_end")}
    for side in ("left", "right"):
        out[side] = [[(a.copy() if a is not None else None) for a in row] for row in b[side]]
    return out


def ora_fluxes(b):
    of = O.OraFluxes()
    for key in ("left_start", "left_end", "right_start", "right_end"):
        arr = getattr(of, key)
        for i in range(3):
            for j in range(3):
                arr[i][j] = int(b[key][i][j])
    for side in ("left", "right"):
        arr = getattr(of, side)
        for s_ in range(6):
            for d in range(3):
                a = b[side][s_][d]
                arr[s_][d] = (a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None
                              else C.POINTER(C.c_double)())
    return of
