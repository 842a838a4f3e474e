"""PressureFree on the GPU against the oracle: bit-identical fields after every step
(two-shock with the pressureless face solve, HLLC, colours, the level batch) and the
time step with a tiny sound speed (calc_dt.F:78-137)."""
import numpy as np
import pytest

import oracle as O
from colour_util import add_colours
from parity_util import compare, copy_fields, random_state
from ppm_b200 import capi
from ppm_b200 import harness as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)


def _steps(ctx, g, hp, f, n):
    f_gpu, f_ora = copy_fields(f), copy_fields(f)
    for cyc in range(n):
        dt = _dt(g, hp, f_ora)
        assert ctx.compute_timestep(g, hp, f_gpu) == dt
        rc, st_o = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        rc, st_g = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu)
        assert rc == capi.OK
        assert st_g["interfaces"] == st_o["interfaces"] == 0 or hp.riemann != 5
        for k, r in compare(f_gpu, f_ora, g).items():
            assert r["bitexact"], (cyc, k, r)
        H.fill_ghosts(g, f_ora, "periodic")
        H.fill_ghosts(g, f_gpu, "periodic")


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("riemann", [5, 4])
def test_pressure_free_matches_oracle(ctx, dual, riemann):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.3, dual=dual, pressure_free=True,
                       riemann=riemann)
    g = H.Grid.uniform((16, 12, 10))
    f = random_state(g, hp, seed=71, mach=1.0, contrast=0.5)
    _steps(ctx, g, hp, f, 3)


def test_pressure_free_with_colours_and_corrections(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.3, dual=True, pressure_free=True, flatten=3,
                       steepen=1)
    g = H.Grid.uniform((14, 12, 10))
    f = random_state(g, hp, seed=72, mach=1.0)
    add_colours(g, f, seed=73)
    _steps(ctx, g, hp, f, 3)


def test_pressure_free_level_matches_oracle(ctx):
    torch = pytest.importorskip("torch")
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.3, dual=True, pressure_free=True)
    rng = np.random.default_rng(74)
    grids, host = [], []
    for k in range(5):
        g = H.Grid.uniform(tuple(int(x) for x in rng.integers(8, 18, size=3)))
        f = random_state(g, hp, seed=80 + k, mach=1.0)
        grids.append(g)
        host.append(f)
    dt = min(_dt(g, hp, f) for g, f in zip(grids, host))
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    rc, _ = ctx.solve_level(grids, hp, dt, 1, dev)
    assert rc == capi.OK
    torch.cuda.synchronize()
    for k, g in enumerate(grids):
        ora = copy_fields(host[k])
        assert O.solve_ppm_de(g, hp, dt, 1, ora, g.cellwidth)[0] == 0
        got = {n: v.cpu().numpy() for n, v in dev[k].items()}
        for n, r in compare(got, ora, g).items():
            assert r["bitexact"], (k, n, r)
