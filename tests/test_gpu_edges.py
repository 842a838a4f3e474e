"""Edge cases of the sweep on the GPU against the oracle: the longest pencil the
reference allows (fortran.def: 1031 cells with ghosts), one longer (rejected), a 3-D
grid with a one-cell active extent (that sweep is skipped, Grid_SolvePPM_DE.C:89-136),
an empty level, and a non-finite input (reported, no fault)."""
import numpy as np
import pytest

import oracle as O
from ppm_b200 import capi
from ppm_b200 import harness as H
from parity_util import compare, copy_fields, random_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _steps(ctx, g, hp, f_gpu, f_ora, n, bc="periodic"):
    for cyc in range(n):
        p = O.compute_pressure(g, hp, f_ora)
        dt = hp.cfl * O.calc_dt(g, hp, f_ora, p, g.cellwidth)
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        rc, _ = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu)
        assert rc == capi.OK
        for k, r in compare(f_gpu, f_ora, g).items():
            assert r["bitexact"], (cyc, k, r)
        H.fill_ghosts(g, f_ora, bc)
        H.fill_ghosts(g, f_gpu, bc)


@pytest.mark.parametrize("shape", [(1025,), (1025, 3, 2)])
def test_longest_allowed_pencil(ctx, shape):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    g = H.Grid.uniform(shape)
    assert g.dims[0] == 1031
    f = random_state(g, hp, seed=3)
    _steps(ctx, g, hp, f, copy_fields(f), 3)


def test_pencil_longer_than_the_reference_limit_is_rejected(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((1026,))
    f = random_state(g, hp, seed=3)
    rc, _ = ctx.solve_ppm_de(g, hp, 1e-4, 0, f, check=False)
    assert rc == capi.ERR_TOO_LARGE


def test_one_cell_active_extent_skips_that_sweep(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    g = H.Grid.uniform((12, 1, 10))
    f = random_state(g, hp, seed=4)
    for cyc in range(3):  # every rotation of the sweep order
        f_ora = copy_fields(f)
        p = O.compute_pressure(g, hp, f_ora)
        dt = hp.cfl * O.calc_dt(g, hp, f_ora, p, g.cellwidth)
        rc, st_o = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        rc, st_g = ctx.solve_ppm_de(g, hp, dt, cyc, f)
        assert rc == capi.OK
        assert st_g["interfaces"] == st_o["interfaces"]
        for k, r in compare(f, f_ora, g).items():
            assert r["bitexact"], (cyc, k, r)


def test_empty_level_is_invalid(ctx):
    hp = H.HydroParams(dual=True)
    rc, _ = ctx.solve_level([], hp, 1e-3, 0, [], check=False)
    assert rc == capi.ERR_INVALID


def test_non_finite_input_is_reported(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((10, 8, 6))
    f = random_state(g, hp, seed=5)
    f["d"][5, 6, 7] = np.nan
    rc, _ = ctx.solve_ppm_de(g, hp, 1e-4, 0, f, check=False)
    assert rc == capi.ERR_NONFINITE
    # the context stays usable
    f = random_state(g, hp, seed=5)
    rc, _ = ctx.solve_ppm_de(g, hp, 1e-4, 0, f, check=False)
    assert rc == capi.OK
