"""Colour fields for the colour tests: keys col0, col1, ... of a field dict (the colnum[]
order of Grid_SolveHydroEquations.C:90-285).  Colours in Enzo are densities (species,
metal density, SN colour) advected with the flow."""
import numpy as np


def add_colours(g, f, seed=0, fractions=(0.25, 0.3), extra=1, marker=True):
    """Colours that are fixed mass fractions of the density (one per entry of fractions),
    `extra` smooth positive random fields, and (marker) a density-weighted step along x
    that is zero on one side.  The fractions inherit the density's ghost zones; the other
    colours' ghost zones are whatever the generator gives (both solvers see the same)."""
    rng = np.random.default_rng(seed)
    n = 0
    for frac in fractions:
        f[f"col{n}"] = frac * f["d"]
        n += 1
    shp = g.shape
    for _ in range(extra):
        a = rng.standard_normal(shp)
        for ax in range(3):
            if shp[ax] > 1:
                a = 0.5 * a + 0.25 * (np.roll(a, 1, ax) + np.roll(a, -1, ax))
        f[f"col{n}"] = np.exp(0.5 * a) * 1e-3
        n += 1
    if marker:
        x = np.arange(shp[2])[None, None, :]
        f[f"col{n}"] = np.where(x < shp[2] // 2, 1.0, 0.0) * f["d"]
        n += 1
    for k in range(n):
        f[f"col{k}"] = np.ascontiguousarray(f[f"col{k}"], dtype=np.float64)
    return n


def colour_keys(f):
    n = 0
    while f"col{n}" in f:
        n += 1
    return [f"col{k}" for k in range(n)]


def hydro_only(f):
    return {k: v for k, v in f.items() if not k.startswith("col")}


def active(g, a):
    return a[g.active_slices()]

