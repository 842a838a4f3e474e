"""Slope flattening (PPMFlatteningParameter 1, 2 and 3, calcdiss.F) and density steepening
(PPMSteepeningParameter 1, inteuler.F:166-193) on the GPU against the CPU oracle:
bit-identical fields after every step on shock-dominated problems (a Sedov blast, a
random supersonic state, the Sod tube), for single grids and a batched level."""
import dataclasses

import numpy as np
import pytest

import oracle as O
from ppm_b200 import capi
from ppm_b200 import harness as H
from parity_util import compare, copy_fields, random_state
from shocktube_driver import GOLDEN, check_against_exact

pytestmark = pytest.mark.gpu

CORRECTIONS = [(1, 0), (2, 0), (3, 0), (0, 1), (3, 1), (1, 1), (2, 1)]


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _oracle_dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)


def _steps(ctx, g, hp, f_gpu, f_ora, n, bc):
    for cyc in range(n):
        dt = _oracle_dt(g, hp, f_ora)
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        rc, _ = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu)
        assert rc == capi.OK
        for k, r in compare(f_gpu, f_ora, g).items():
            assert r["bitexact"], (cyc, k, r)
        H.fill_ghosts(g, f_ora, bc)
        H.fill_ghosts(g, f_gpu, bc)


@pytest.mark.parametrize("flatten,steepen", CORRECTIONS)
@pytest.mark.parametrize("dual", [False, True])
def test_sedov_blast_matches_oracle(ctx, flatten, steepen, dual):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=dual, flatten=flatten, steepen=steepen)
    g = H.Grid.uniform((20, 18, 16))
    f = H.sedov(g, hp)
    H.fill_ghosts(g, f, "outflow")
    _steps(ctx, g, hp, f, copy_fields(f), 6, "outflow")


@pytest.mark.parametrize("flatten,steepen", CORRECTIONS)
def test_supersonic_random_state_matches_oracle(ctx, flatten, steepen):
    hp = H.HydroParams(gamma=1.4, cfl=0.3, dual=True, flatten=flatten, steepen=steepen)
    g = H.Grid.uniform((17, 12, 10))
    f = random_state(g, hp, seed=31, mach=3.0, contrast=1.5)
    H.fill_ghosts(g, f, "periodic")
    _steps(ctx, g, hp, f, copy_fields(f), 5, "periodic")


def test_sod_with_corrections_matches_oracle_and_exact(ctx):
    name = "SodShockTube"
    pr = GOLDEN["problems"][name]
    hp = H.HydroParams(gamma=GOLDEN["gamma"], cfl=GOLDEN["cfl"], dual=True, flatten=3,
                       steepen=1)
    g = H.Grid.uniform((GOLDEN["nzones"],))
    f_gpu = H.shock_tube(g, hp, pr["x0"], pr["left"], pr["right"])
    H.fill_ghosts(g, f_gpu, "outflow")
    f_ora = copy_fields(f_gpu)
    t, cyc = 0.0, 0
    while t < pr["t"] - 1e-14:
        dt = min(_oracle_dt(g, hp, f_ora), pr["t"] - t)
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu)
        for k, r in compare(f_gpu, f_ora, g).items():
            assert r["bitexact"], (cyc, k, r)
        H.fill_ghosts(g, f_ora, "outflow")
        H.fill_ghosts(g, f_gpu, "outflow")
        t += dt
        cyc += 1
    assert check_against_exact(name, g, hp, f_gpu) == []


def test_level_with_corrections_matches_per_grid_and_oracle(ctx):
    import torch
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True, flatten=3, steepen=1)
    rng = np.random.default_rng(4)
    grids = [H.Grid.uniform(tuple(int(x) for x in rng.integers(8, 22, size=3))) for _ in range(7)]
    host = []
    for k, g in enumerate(grids):
        f = H.sedov(g, hp) if k % 2 == 0 else random_state(g, hp, seed=k, mach=2.0)
        H.fill_ghosts(g, f, "periodic")
        host.append(f)
    dt = min(_oracle_dt(g, hp, f) for g, f in zip(grids, host))
    dev = [{n: torch.from_numpy(v.copy()).cuda() for n, v in f.items()} for f in host]
    rc, _ = ctx.solve_level(grids, hp, dt, 1, dev)
    assert rc == capi.OK
    for k, g in enumerate(grids):
        ora = copy_fields(host[k])
        rc, _ = O.solve_ppm_de(g, hp, dt, 1, ora, g.cellwidth)
        assert rc == 0
        got = {n: v.cpu().numpy() for n, v in dev[k].items()}
        for n, r in compare(got, ora, g).items():
            assert r["bitexact"], (k, n, r)


def test_unsupported_flattening_types_are_rejected(ctx):
    g = H.Grid.uniform((8, 8, 8))
    for flatten in (4, 5):
        hp = H.HydroParams(dual=True, flatten=flatten)
        f = random_state(g, hp, seed=1)
        with pytest.raises(capi.PPMError) as e:
            ctx.solve_ppm_de(g, hp, 1e-3, 0, f)
        assert e.value.code == capi.ERR_UNSUPPORTED
