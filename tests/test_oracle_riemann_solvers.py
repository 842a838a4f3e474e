"""The oracle's HLL and HLLC solvers (RiemannSolver = 1 / 4: flux_hll.F:6-415,
flux_hllc.F:6-421, the switch of Grid_xEulerSweep.C:223-283), pinned by the reference's
shock-tube answer tests and by what the two solvers do to a contact:
  - HLLC passes every shock tube of the reference (Sod, Toro 1-7) at the reference's
    tolerances, with and without dual energy;
  - HLL, which has no contact wave, passes the problems whose solution has no contact
    that must stay sharp inside the tested windows (Toro 1-4);
  - a stationary contact (uniform pressure, no flow): HLLC and the two-shock solver keep
    its density exactly, HLL diffuses it;
  - a negative density stops HLL (flux_hll.F:336-380) and sends HLLC cells to the
    per-cell HLL fallback (flux_hllc.F:331-389)."""
import dataclasses

import numpy as np
import pytest

import oracle as O
import shocktube_driver as SD
from parity_util import copy_fields, random_state
from ppm_b200 import harness as H

HLL, HLLC, TWOSHOCK = 1, 4, 5


def _step(g, hp, dt, cyc, f):
    rc, st = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
    assert rc == 0, st


def _dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return O.calc_dt(g, hp, f, p, g.cellwidth)


def _run(name, dual, riemann, monkeypatch):
    base = H.HydroParams

    def params(**kw):
        return dataclasses.replace(base(**kw), riemann=riemann)

    monkeypatch.setattr(SD.H, "HydroParams", params)
    return SD.run_problem(name, _step, _dt, dual=dual)


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("name", sorted(SD.GOLDEN["problems"]))
def test_hllc_passes_the_shock_tubes(name, dual, monkeypatch):
    g, hp, f, cycles = _run(name, dual, HLLC, monkeypatch)
    assert cycles > 10
    assert SD.check_against_exact(name, g, hp, f) == []


@pytest.mark.parametrize("name", ["Toro-1-ShockTube", "Toro-2-ShockTube", "Toro-3-ShockTube",
                                  "Toro-4-ShockTube"])
def test_hll_passes_the_shock_tubes_without_sharp_contacts(name, monkeypatch):
    g, hp, f, cycles = _run(name, True, HLL, monkeypatch)
    assert SD.check_against_exact(name, g, hp, f) == []


@pytest.mark.parametrize("riemann,exact", [(HLL, False), (HLLC, True), (TWOSHOCK, True)])
def test_stationary_contact(riemann, exact):
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=True, riemann=riemann)
    g = H.Grid.uniform((32,))
    f = H.new_fields(g, True)
    x = g.centers(0)
    f["d"][...] = np.where(x < 0.5, 1.0, 0.125)[None, None, :]
    f["ge"][...] = 1.0 / ((hp.gamma - 1.0) * f["d"])
    f["te"][...] = f["ge"]
    H.fill_ghosts(g, f, "outflow")
    d0 = f["d"].copy()
    _step(g, hp, hp.cfl * _dt(g, hp, f), 0, f)
    assert np.array_equal(f["d"], d0) == exact
    assert np.all(f["v1"] == 0.0)


@pytest.mark.parametrize("riemann", [HLL, HLLC])
def test_solvers_differ_from_two_shock_on_shocks(riemann):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((14, 12, 10))
    f = random_state(g, hp, seed=3, mach=2.0)
    a, b = copy_fields(f), copy_fields(f)
    dt = hp.cfl * _dt(g, hp, f)
    _step(g, hp, dt, 0, a)
    _step(g, dataclasses.replace(hp, riemann=riemann), dt, 0, b)
    assert not np.array_equal(a["d"], b["d"])
    rel = np.abs(a["d"] - b["d"]).max() / np.abs(a["d"]).max()
    assert rel < 0.2  # the same flow, a different approximate solver


def test_negative_density_stops_hll_and_falls_back_in_hllc():
    # an oversized step (5 x the Courant limit) drains cells below zero density
    for riemann, fallback in ((HLL, True), (HLLC, False)):
        hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, fallback=fallback,
                           riemann=riemann)
        g = H.Grid.uniform((20, 12, 10))
        f = random_state(g, hp, seed=7, mach=3.0, contrast=1.5)
        rc, st = O.solve_ppm_de(g, hp, 5.0 * _dt(g, hp, f), 0, f, g.cellwidth)
        assert rc != 0 and st["fatal"] == 1 and st["fallbacks"] == 0
    # a milder one that HLLC's fallback cells survive
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, fallback=True, riemann=HLLC)
    f = random_state(g, hp, seed=10, mach=3.0, contrast=1.5)
    rc, st = O.solve_ppm_de(g, hp, 3.9 * _dt(g, hp, f), 0, f, g.cellwidth)
    assert rc == 0 and st["fallbacks"] == 2
