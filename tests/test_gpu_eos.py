"""The isothermal equation of state (EOSType 3) on the GPU against the oracle: the
pressure kernel's rho*cs^2 with the total-energy reset, the reset at the end of every
solve, and the time step with the isothermal pressure (explicit and folded into the last
sweep), bit for bit, single grids and a level."""
import numpy as np
import pytest

import oracle as O
from parity_util import compare, copy_fields, random_state
from ppm_b200 import capi
from ppm_b200 import harness as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _hp(dual, **kw):
    return H.HydroParams(gamma=5.0 / 3.0, cfl=0.3, dual=dual, eos_type=3, eos_sound_speed=0.7,
                         **kw)


def _dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)


@pytest.mark.parametrize("dual", [False, True])
def test_isothermal_steps_match_oracle(ctx, dual):
    hp = _hp(dual)
    g = H.Grid.uniform((16, 12, 10))
    f = random_state(g, hp, seed=5, mach=1.0)
    f_gpu, f_ora = copy_fields(f), copy_fields(f)
    for cyc in range(3):
        dt = _dt(g, hp, f_ora)  # resets the oracle's energies, as ComputeTimeStep would
        assert ctx.compute_timestep(g, hp, f_gpu) == dt
        ctx.compute_pressure(g, hp, f_gpu, np.zeros_like(f_gpu["d"]))  # its reset too
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        assert ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu)[0] == capi.OK
        for k, r in compare(f_gpu, f_ora, g).items():
            assert r["bitexact"], (cyc, k, r)
        H.fill_ghosts(g, f_ora, "periodic")
        H.fill_ghosts(g, f_gpu, "periodic")


def test_isothermal_level_with_folded_time_step(ctx):
    torch = pytest.importorskip("torch")
    hp = _hp(True)
    rng = np.random.default_rng(6)
    grids, host = [], []
    for k in range(4):
        g = H.Grid.uniform(tuple(int(x) for x in rng.integers(8, 16, size=3)))
        grids.append(g)
        host.append(random_state(g, hp, seed=20 + k, mach=1.0))
    ora = [copy_fields(f) for f in host]
    dt = min(_dt(g, hp, f) for g, f in zip(grids, ora))
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in ora]
    dt_next = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.set_cfl(dt_next, courant=hp.cfl)
    try:
        rc, _ = ctx.solve_level(grids, hp, dt, 0, dev)
        assert rc == capi.OK
        torch.cuda.synchronize()
    finally:
        ctx.set_cfl(None)
    for k, g in enumerate(grids):
        assert O.solve_ppm_de(g, hp, dt, 0, ora[k], g.cellwidth)[0] == 0
        got = {n: v.cpu().numpy() for n, v in dev[k].items()}
        for n, r in compare(got, ora[k], g).items():
            assert r["bitexact"], (k, n, r)
    assert float(dt_next.item()) == min(_dt(g, hp, f) for g, f in zip(grids, ora))


def test_other_eos_types_are_unsupported(ctx):
    g = H.Grid.uniform((8, 8, 8))
    for eos in (1, 2, 4):
        hp = H.HydroParams(dual=True, eos_type=eos)
        rc, _ = ctx.solve_ppm_de(g, hp, 1e-3, 0, random_state(g, hp, seed=1), check=False)
        assert rc == capi.ERR_UNSUPPORTED
