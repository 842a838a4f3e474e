"""The oracle's colour fields (NumberOfColours > 0: inteuler.F:276-282, :436-450,
:500-515, :546-551; flux_twoshock.F:251-259, :375-380; flux_hll.F:236-262, :328-332;
euler.F:171-186; Grid_xEulerSweep.C:124-132, :361-371, :409-416).  No bit-level output
of the reference's colour path exists in its tree, so these pin the restatement by what
the reference's colour arithmetic implies:
  - colours never change the hydro fields (bit for bit);
  - a colour that is a fixed mass fraction of the density stays that fraction (the
    colour states are the density states scaled by the fraction, and the colour flux
    dt*ub*colb/dx is the mass flux scaled by it), also through the HLL fallback and
    the dual-energy override, with the mass flux's subgrid capture scaled likewise;
  - one sweep of a periodic grid conserves each colour;
  - a zero colour becomes euler.F's floor min_color = 1e-5 * tiny;
  - a density-weighted marker on the Sod tube is carried by the contact
    discontinuity of the exact solution (the reference's SodShockTube answer test)."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from colour_util import add_colours, colour_keys
from parity_util import copy_fields, random_state
from ppm_b200 import harness as H
from shocktube_driver import GOLDEN

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import exact_riemann  # noqa: E402

MIN_COLOR = 1.0e-5 * 1.0e-20  # euler.F:104-105


def _dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)


def _step(g, hp, dt, cyc, f, **kw):
    rc, st = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth, **kw)
    assert rc == 0, st
    return st


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("flatten,steepen", [(0, 0), (3, 1)])
def test_colours_leave_hydro_unchanged(dual, flatten, steepen):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=dual, flatten=flatten, steepen=steepen)
    g = H.Grid.uniform((16, 12, 10))
    f = random_state(g, hp, seed=3, mach=2.0)
    plain = copy_fields(f)
    add_colours(g, f, seed=4)
    for cyc in range(3):
        dt = _dt(g, hp, plain)
        _step(g, hp, dt, cyc, plain)
        _step(g, hp, dt, cyc, f)
        for k, v in plain.items():
            assert np.array_equal(v, f[k]), (cyc, k)
        H.fill_ghosts(g, plain, "periodic")
        H.fill_ghosts(g, f, "periodic")


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("flatten", [0, 3])
def test_mass_fraction_colour_tracks_density(dual, flatten):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=dual, flatten=flatten)
    g = H.Grid.uniform((16, 14, 12))
    f = random_state(g, hp, seed=8, mach=2.5, contrast=1.0)
    add_colours(g, f, fractions=(0.25, 0.3), extra=0, marker=False)
    for cyc in range(4):
        _step(g, hp, _dt(g, hp, f), cyc, f)
        H.fill_ghosts(g, f, "periodic")
    for k, frac in (("col0", 0.25), ("col1", 0.3)):
        rel = np.abs(f[k] / (frac * f["d"]) - 1.0)
        assert rel.max() < 1e-12, (k, rel.max())


def test_mass_fraction_colour_through_hll_fallback():
    # negative total energy in a few cells forces flux_hll on them (flux_twoshock.F:401-456)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, fallback=1)
    g = H.Grid.uniform((20, 12, 10))
    f = random_state(g, hp, seed=7)
    for (k, j, i) in [(5, 6, 8), (5, 6, 9), (8, 4, 14), (4, 10, 5)]:
        f["te"][k, j, i] = -1e-3
    add_colours(g, f, fractions=(0.5,), extra=0, marker=False)
    st = _step(g, hp, _dt(g, hp, f), 0, f)
    assert st["fallbacks"] == 4
    rel = np.abs(f["col0"] / (0.5 * f["d"]) - 1.0)
    assert rel.max() < 1e-12


def test_colours_conserved_by_a_periodic_sweep():
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=True)
    g = H.Grid.uniform((14, 12, 10))
    f = random_state(g, hp, seed=21, mach=1.5)
    add_colours(g, f, seed=22, fractions=(0.3,), extra=2, marker=True)
    act = g.active_slices()
    for dim in range(3):
        H.fill_ghosts(g, f, "periodic")
        before = {k: f[k][act].sum() for k in colour_keys(f)}
        p = O.compute_pressure(g, hp, f)
        dt = _dt(g, hp, f)
        rc, _ = O.sweep(dim, g, hp, dt, f, p, g.cellwidth)
        assert rc == 0
        for k, s0 in before.items():
            assert abs(f[k][act].sum() - s0) <= 1e-13 * abs(s0), (dim, k)


def test_zero_colour_takes_the_euler_floor():
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=False)
    g = H.Grid.uniform((12, 10, 8))
    f = random_state(g, hp, seed=5)
    f["col0"] = np.zeros_like(f["d"])
    p = O.compute_pressure(g, hp, f)
    rc, _ = O.sweep(0, g, hp, _dt(g, hp, f), f, p, g.cellwidth)
    assert rc == 0
    # the first sweep floors every active cell: its fluxes are of order color_floor
    s, e = g.start[0], g.end[0] + 1
    assert np.all(f["col0"][:, :, s:e] == MIN_COLOR)
    assert np.all(f["col0"][:, :, :s] == 0.0) and np.all(f["col0"][:, :, e:] == 0.0)
    # later sweeps keep every cell at or above it
    g2 = copy_fields(f)
    _step(g, hp, _dt(g, hp, g2), 1, g2)
    assert np.all(g2["col0"][g.active_slices()] >= MIN_COLOR)


def _flux_box(g, lo, hi, ncol):
    """A subgrid over zones lo..hi (inclusive, this grid's indices) with capture arrays
    for the six hydro slots and every colour (left/right faces of each dim)."""
    F = O.OraFluxes()
    keep = []
    for dim in range(3):
        for j in range(3):
            s, e = lo[j], hi[j]
            F.left_start[dim][j] = s if j != dim else lo[j]
            F.left_end[dim][j] = e if j != dim else lo[j]
            F.right_start[dim][j] = s if j != dim else hi[j]
            F.right_end[dim][j] = e if j != dim else hi[j]
        size = 1
        for j in range(3):
            if j != dim:
                size *= hi[j] - lo[j] + 1
        for side in ("left", "right"):
            for slot in range(6):  # the oracle fills every hydro slot
                a = np.zeros(size)
                keep.append(a)
                getattr(F, side)[slot][dim] = a.ctypes.data_as(C.POINTER(C.c_double))
            for n in range(ncol):
                c = np.zeros(size)
                keep.append(c)
                getattr(F, "colour_" + side)[n][dim] = c.ctypes.data_as(C.POINTER(C.c_double))
    return F, keep


def test_colour_subgrid_fluxes_are_mass_fluxes_scaled():
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((14, 12, 10))
    f = random_state(g, hp, seed=12, mach=2.0)
    add_colours(g, f, fractions=(0.25, 0.75), extra=0, marker=False)
    box, keep = _flux_box(g, (6, 5, 5), (10, 9, 8), 2)
    subs = [box]
    _step(g, hp, _dt(g, hp, f), 0, f, subgrids=subs, ggs=(0, 0, 0))
    got = subs[0]
    for dim in range(3):
        size = 1
        for j in range(3):
            if j != dim:
                size *= got.right_end[dim][j] - got.right_start[dim][j] + 1
        for side in ("left", "right"):
            d = np.ctypeslib.as_array(getattr(got, side)[0][dim], shape=(size,))
            assert np.any(d != 0.0)
            for n, frac in enumerate((0.25, 0.75)):
                c = np.ctypeslib.as_array(getattr(got, "colour_" + side)[n][dim], shape=(size,))
                assert np.allclose(c, frac * d, rtol=1e-12, atol=1e-300), (dim, side, n)


def test_sod_marker_follows_the_contact():
    pr = GOLDEN["problems"]["SodShockTube"]
    hp = H.HydroParams(gamma=GOLDEN["gamma"], cfl=GOLDEN["cfl"], dual=True)
    g = H.Grid.uniform((GOLDEN["nzones"],))
    f = H.shock_tube(g, hp, pr["x0"], pr["left"], pr["right"])
    x = g.centers(0)
    f["col0"] = np.where(x < pr["x0"], 1.0, 0.0)[None, None, :] * f["d"]
    H.fill_ghosts(g, f, "outflow")
    t, cyc = 0.0, 0
    while t < pr["t"] - 1e-14:
        dt = min(_dt(g, hp, f), pr["t"] - t)
        _step(g, hp, dt, cyc, f)
        H.fill_ghosts(g, f, "outflow")
        t += dt
        cyc += 1
    (dl, ul, pl), (dr, ur, prr) = pr["left"], pr["right"]
    _, us = exact_riemann.star_state(dl, ul, pl, dr, ur, prr, hp.gamma)
    xc = pr["x0"] + us * pr["t"]  # the contact of the exact solution
    frac = (f["col0"] / f["d"])[0, 0, :]
    s, e = g.start[0], g.end[0] + 1
    xa, fa = x[s:e], frac[s:e]
    assert np.all(fa[xa < xc - 0.06] > 0.99)
    assert np.all(fa[xa > xc + 0.06] < 0.01)
    # positive everywhere; PPM's small overshoots at the contact stay below 1 %
    assert np.all(fa > 0.0) and np.all(fa < 1.01)
