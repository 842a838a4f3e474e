"""A Zel'dovich pancake (the cold cosmological flow of the fifth benchmark configuration,
one level of it) advanced through comoving cycles on the GPU and by the oracle: the
expansion terms (grid::ComovingExpansionTerms) then SolvePPM_DE with gravity and dual
energy, bit-identical after every cycle, for a single grid and for the same pancake split
into a level of patches."""
import numpy as np
import pytest

import oracle as O
from parity_util import compare, copy_fields
from ppm_b200 import capi
from ppm_b200 import harness as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _accel(g, scale=1e-3):
    """The linear-theory gravity of the pancake: along x, towards the caustic."""
    n = g.end[0] - g.start[0] + 1
    x = (np.arange(g.dims[0]) - g.start[0] + 0.5 - 0.5 * n) * 2.0 * np.pi / n
    ax = np.broadcast_to(-scale * np.sin(x)[None, None, :], g.shape).copy()
    return [ax] + [np.zeros(g.shape) for _ in range(g.rank - 1)]


@pytest.mark.parametrize("shape", [(48,), (32, 8, 8)])
def test_comoving_pancake_cycles_match_oracle(ctx, shape):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True, gravity=True, eta1=0.001,
                       eta2=0.1)
    g = H.Grid.uniform(shape)
    f = H.zeldovich_pancake(g, hp)
    acc = _accel(g)
    f_ora, f_gpu = copy_fields(f), copy_fields(f)
    t = 1.0
    for cyc in range(4):
        p = O.compute_pressure(g, hp, f_ora)
        dt = hp.cfl * O.calc_dt(g, hp, f_ora, p, g.cellwidth)
        coef = 0.004  # dt * adot / a: the expansion limits a cosmological step to a few 1e-3
        O.expansion_terms(g, hp, f_ora, None, t + dt, t, coef)
        ctx.expansion_terms(g, hp, f_gpu, None, t + dt, t, coef)
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth, accel=acc)
        assert rc == 0
        rc, _ = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu, accel=acc)
        assert rc == capi.OK
        for k, r in compare(f_gpu, f_ora, g).items():
            assert r["bitexact"], (cyc, k, r)
        H.fill_ghosts(g, f_ora, "periodic")
        H.fill_ghosts(g, f_gpu, "periodic")
        t += dt
    # the flow converges on the caustic: the central density has grown
    act = g.active_slices()
    assert f_gpu["d"][act].max() > f["d"][act].max()
