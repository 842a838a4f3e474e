"""The next cycle's time step folded into the last sweep (ppm_b200_set_cfl): the value
written by a solve equals the separate calc_dt pass (ppm_b200_compute_timestep) on the
updated fields bit for bit -- single grids of every rank, with and without dual energy
and gravity, with HLL-fallback pencils, levels, and CUDA-graph replays."""
import numpy as np
import pytest

from ppm_b200 import capi
from ppm_b200 import harness as H
from parity_util import random_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    t.cuda.set_device(0)
    return t


def _dev(f, torch):
    return {k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()}


@pytest.mark.parametrize("shape,dual,grav,fallback_cells", [
    ((16, 12, 10), True, False, False),
    ((16, 12, 10), False, False, False),
    ((14, 11, 9), True, True, False),
    ((20, 12, 10), True, False, True),
    ((24, 18), True, False, False),
    ((40,), False, False, False),
])
def test_folded_time_step_equals_calc_dt(torch, shape, dual, grav, fallback_cells):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.45, dual=dual, gravity=grav)
    g = H.Grid.uniform(shape, width=tuple(0.5 + 0.1 * d for d in range(len(shape))))
    f = random_state(g, hp, seed=55)
    if fallback_cells:
        for (k, j, i) in [(5, 6, 8), (5, 6, 9), (8, 4, 14)]:
            f["te"][k, j, i] = -1e-3
    accel = None
    if grav:
        rng = np.random.default_rng(5)
        accel = [torch.from_numpy(0.1 * rng.standard_normal(g.shape)).cuda()
                 for _ in range(g.rank)]
    fd = _dev(f, torch)
    ctx = capi.Context(0)
    nxt = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.set_cfl(nxt, courant=hp.cfl, aye=0.9, vgrid=(0.01, -0.02, 0.03))
    for cyc in range(3):
        dt = ctx.compute_timestep(g, hp, fd, memory=capi.MEM_DEVICE, aye=0.9,
                                  vgrid=(0.01, -0.02, 0.03))
        rc, st = ctx.solve_ppm_de(g, hp, dt, cyc, fd, memory=capi.MEM_DEVICE, accel=accel,
                                  check=False)
        assert rc == capi.OK
        if fallback_cells and cyc == 0:
            assert st["fallbacks"] > 0
        ref = ctx.compute_timestep(g, hp, fd, memory=capi.MEM_DEVICE, aye=0.9,
                                   vgrid=(0.01, -0.02, 0.03))
        assert nxt.item() == ref, (cyc, nxt.item(), ref)
        ctx.set_boundary(g, fd, dual)
    ctx.close()


def test_folded_time_step_of_a_level_with_graphs(torch):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    shapes = [(16, 16, 16), (24, 12, 8), (8, 8, 8), (10, 18, 6)]
    grids = [H.Grid.uniform(s) for s in shapes]
    fs = [_dev(random_state(g, hp, seed=100 + k), torch) for k, g in enumerate(grids)]
    ctx = capi.Context(0)
    ctx.set_graphs(True)
    dt = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.compute_timestep_level(grids, hp, fs, dt_device=dt, want_host=False)
    ctx.set_cfl(dt, courant=hp.cfl)
    for cyc in range(5):  # the solve reads dt and leaves the next one in it
        ctx.solve_level(grids, hp, 0.0, cyc, fs, dt_device=dt)
        ref = ctx.compute_timestep_level(grids, hp, fs)
        assert dt.item() == ref, (cyc, dt.item(), ref)
        ctx.set_boundary_level(grids, fs, True)
    ctx.close()
