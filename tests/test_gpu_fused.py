"""The fused sweep (ppm_b200_set_sweep_mode FUSED: one kernel reconstructs the interface
states and solves the two-shock problem of every face, so the states never reach device
memory) gives the oracle's fields bit for bit, like the split kernels: single grids of
ranks 1-3 with and without dual energy and gravity, the per-cell HLL fallback (planted
negative energies, whose pencils get their states from the flagged-pencil pass), the
single-sweep entry point, batched levels with graph replay and the folded time step."""
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
    c.set_sweep_mode("fused")
    yield c
    c.close()


def _same(a, b, g, what):
    for k, r in compare(a, b, g).items():
        assert r["bitexact"], (what, k, r)


def _dt(g, hp, f):
    return hp.cfl * O.calc_dt(g, hp, f, O.compute_pressure(g, hp, f), g.cellwidth)


@pytest.mark.parametrize("shape,dual,grav,seed", [
    ((16, 16, 16), True, False, 1),
    ((20, 12, 9), False, False, 2),
    ((13, 17, 40), True, True, 3),   # pencils of several 31-face segments
    ((70, 20), True, True, 4),
    ((100,), True, False, 5),
    ((33, 5, 4), False, True, 6),
])
def test_fused_sweep_multistep_matches_oracle(ctx, shape, dual, grav, seed):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=dual, gravity=grav)
    g = H.Grid.uniform(shape)
    f_gpu = random_state(g, hp, seed=seed)
    f_ora = copy_fields(f_gpu)
    accel = None
    if grav:
        rng = np.random.default_rng(seed + 100)
        accel = [0.1 * rng.standard_normal(g.shape) for _ in range(g.rank)]
    for cyc in range(8):
        dt = _dt(g, hp, f_ora)
        rc, st_o = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth, accel=accel)
        assert rc == 0
        rc, st_g = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu, accel=accel)
        _same(f_gpu, f_ora, g, (shape, cyc))
        assert st_g["interfaces"] == st_o["interfaces"]
        assert st_g["newton_iters"] == st_o["newton_iters"]
        H.fill_ghosts(g, f_ora, "periodic")
        H.fill_ghosts(g, f_gpu, "periodic")


def test_fused_sweep_hll_fallback_matches_oracle(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, fallback=True)
    g = H.Grid.uniform((20, 12, 10))
    f = random_state(g, hp, seed=7)
    for (k, j, i) in [(5, 6, 8), (5, 6, 9), (8, 4, 14), (4, 10, 5)]:
        f["te"][k, j, i] = -1e-3
    f_ora, f_gpu = copy_fields(f), copy_fields(f)
    dt = _dt(g, hp, f_ora)
    rc_o, st_o = O.solve_ppm_de(g, hp, dt, 0, f_ora, g.cellwidth)
    rc_g, st_g = ctx.solve_ppm_de(g, hp, dt, 0, f_gpu, check=False)
    assert rc_o == 0 and rc_g == capi.OK
    assert st_o["fallbacks"] == 4 and st_g["fallbacks"] == 4
    _same(f_gpu, f_ora, g, "fallback")


def test_fused_single_sweep_entry_matches_oracle(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    g = H.Grid.uniform((14, 12, 36))
    for dim in range(3):
        f_gpu = random_state(g, hp, seed=20 + dim)
        f_ora = copy_fields(f_gpu)
        p = O.compute_pressure(g, hp, f_ora)
        dt = _dt(g, hp, f_ora)
        rc, _ = O.sweep(dim, g, hp, dt, f_ora, p, g.cellwidth)
        assert rc == 0
        ctx.euler_sweep(dim, g, hp, dt, f_gpu, p)
        _same(f_gpu, f_ora, g, ("sweep", dim))


def test_fused_level_with_graphs_and_folded_timestep_matches_split():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    shapes = [(16, 16, 16), (24, 12, 8), (8, 8, 8), (40, 18, 6), (2, 9, 7), (20, 33, 4)]
    grids, host = [], []
    for k, shp in enumerate(shapes):
        g = H.Grid.uniform(shp, width=tuple(0.25 * s / 8.0 for s in shp))
        grids.append(g)
        host.append(random_state(g, hp, seed=300 + k))
    out = {}
    for mode in ("split", "fused"):
        c = capi.Context(0)
        c.set_sweep_mode(mode)
        c.set_graphs(True)
        f = [{k: torch.from_numpy(v.copy()).cuda() for k, v in fh.items()} for fh in host]
        dtd = torch.zeros(1, dtype=torch.float64, device="cuda")
        c.compute_timestep_level(grids, hp, f, dt_device=dtd, want_host=False)
        c.set_cfl(dtd, courant=hp.cfl)
        for cyc in range(5):
            c.solve_level(grids, hp, 0.0, cyc, f, dt_device=dtd)
            c.set_boundary_level(grids, f, True)
        assert c.synchronize()[0] == capi.OK
        out[mode] = ([{k: v.cpu().numpy() for k, v in fk.items()} for fk in f], dtd.item())
        c.set_cfl(None)
        c.close()
    assert out["split"][1] == out["fused"][1]
    for k, g in enumerate(grids):
        _same(out["fused"][0][k], out["split"][0][k], g, ("level", k))


def test_fused_fast_build_meets_the_bar():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    c = capi.Context(0, variant="fast")
    c.set_sweep_mode("fused")
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((32, 32, 32))
    f_ora = H.turbulence(g, hp, mach=3.0, seed=5)
    f_gpu = {k: torch.from_numpy(v.copy()).cuda() for k, v in f_ora.items()}
    for cyc in range(30):
        dt = _dt(g, hp, f_ora)
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        c.solve_ppm_de(g, hp, dt, cyc, f_gpu, memory=capi.MEM_DEVICE, want_stats=False)
        H.fill_ghosts(g, f_ora, "periodic")
        c.set_boundary(g, f_gpu, True)
        assert c.synchronize()[0] == capi.OK
        tol = 1e-12 if cyc == 0 else 1e-10
        for k, r in compare({k: v.cpu().numpy() for k, v in f_gpu.items()}, f_ora, g).items():
            assert r["maxrel"] <= tol, (cyc, k, r)
    c.close()
