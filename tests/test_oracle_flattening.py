"""The oracle's slope flattening (calcdiss.F types 1, 2 and 3) and density steepening
(inteuler.F:166-193, intvar.F:106-113), against the reference's own answer tests: every
shock tube (Sod, Toro 1-7) still passes at the reference's tolerances with the
corrections on, the corrections change the shocked solutions, and on smooth data
(no pressure jump above calcdiss's 33 % threshold) flattening leaves every bit unchanged."""
import dataclasses

import numpy as np
import pytest

import oracle as O
import shocktube_driver as SD
from ppm_b200 import harness as H
from parity_util import random_state


def _step(g, hp, dt, cyc, f):
    rc, st = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
    assert rc == 0, st


def _dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return O.calc_dt(g, hp, f, p, g.cellwidth)


def _run(name, dual, flatten, steepen, monkeypatch):
    base = H.HydroParams

    def params(**kw):
        return dataclasses.replace(base(**kw), flatten=flatten, steepen=steepen)

    monkeypatch.setattr(SD.H, "HydroParams", params)
    return SD.run_problem(name, _step, _dt, dual=dual)


@pytest.mark.parametrize("flatten,steepen", [(1, 0), (2, 0), (3, 0), (0, 1), (3, 1), (2, 1)])
@pytest.mark.parametrize("name", sorted(SD.GOLDEN["problems"]))
def test_shock_tubes_pass_with_corrections(name, flatten, steepen, monkeypatch):
    g, hp, f, cycles = _run(name, True, flatten, steepen, monkeypatch)
    assert cycles > 10
    assert SD.check_against_exact(name, g, hp, f) == []


@pytest.mark.parametrize("flatten,steepen", [(1, 0), (2, 0), (3, 0), (0, 1)])
def test_corrections_act_on_sod(flatten, steepen, monkeypatch):
    _, _, plain, _ = _run("SodShockTube", True, 0, 0, monkeypatch)
    _, _, corr, _ = _run("SodShockTube", True, flatten, steepen, monkeypatch)
    assert not np.array_equal(plain["d"], corr["d"])


@pytest.mark.parametrize("flatten", [1, 2, 3])
def test_flattening_leaves_smooth_flow_unchanged(flatten):
    g = H.Grid.uniform((24, 6, 5))
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=True)
    rng = np.random.default_rng(5)
    f0 = random_state(g, hp, seed=9)
    # a smooth, weak perturbation: pressure ratios between cells two apart stay < 1.33
    x = g.centers(0)
    for k in f0:
        f0[k][...] = f0[k].mean()
    f0["d"][...] = 1.0 + 0.05 * np.sin(2 * np.pi * x)[None, None, :]
    f0["v1"][...] = 0.1 * np.cos(2 * np.pi * x)[None, None, :] + 0.01 * rng.standard_normal(1)
    p = 1.0 / hp.gamma
    f0["ge"][...] = p / ((hp.gamma - 1.0) * f0["d"])
    f0["te"][...] = f0["ge"] + 0.5 * (f0["v1"] ** 2 + f0["v2"] ** 2 + f0["v3"] ** 2)
    H.fill_ghosts(g, f0, "periodic")
    a = {k: v.copy() for k, v in f0.items()}
    b = {k: v.copy() for k, v in f0.items()}
    hq = dataclasses.replace(hp, flatten=flatten)
    for cyc in range(3):
        dt = hp.cfl * _dt(g, hp, a)
        _step(g, hp, dt, cyc, a)
        _step(g, hq, dt, cyc, b)
        H.fill_ghosts(g, a, "periodic")
        H.fill_ghosts(g, b, "periodic")
    for k in a:
        assert np.array_equal(a[k], b[k]), k
