"""RiemannSolver = HLL and HLLC on the GPU (the HLL-family Riemann kernel, ges in the XUB
plane, the density-only check) against the CPU oracle: bit-identical fields after every
step, single grids of rank 1-3, dual energy on and off, colours, slope corrections, the
batched level with and without graphs, HLLC's per-cell HLL fallback, and HLL's stop on
a negative density (ERR_NEGATIVE)."""
import numpy as np
import pytest

import oracle as O
from colour_util import add_colours
from parity_util import compare, copy_fields, random_state
from ppm_b200 import capi
from ppm_b200 import harness as H

pytestmark = pytest.mark.gpu

HLL, HLLC = 1, 4


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return O.calc_dt(g, hp, f, p, g.cellwidth)


def _bitexact(got, ref, g, where=""):
    for k, r in compare(got, ref, g).items():
        assert r["bitexact"], (where, k, r)


def _steps(ctx, g, hp, f, n, bc="periodic"):
    f_gpu, f_ora = copy_fields(f), copy_fields(f)
    for cyc in range(n):
        dt = hp.cfl * _dt(g, hp, f_ora)
        rc, st_o = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        rc, st_g = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu)
        assert rc == capi.OK
        assert st_g["fallbacks"] == st_o["fallbacks"]
        _bitexact(f_gpu, f_ora, g, cyc)
        H.fill_ghosts(g, f_ora, bc)
        H.fill_ghosts(g, f_gpu, bc)


@pytest.mark.parametrize("riemann", [HLL, HLLC])
@pytest.mark.parametrize("dual", [False, True])
def test_random_state_matches_oracle(ctx, riemann, dual):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=dual, riemann=riemann)
    g = H.Grid.uniform((18, 14, 12))
    _steps(ctx, g, hp, random_state(g, hp, seed=51, mach=2.5, contrast=1.0), 4)


@pytest.mark.parametrize("riemann", [HLL, HLLC])
@pytest.mark.parametrize("shape", [(40,), (20, 16)])
def test_low_rank_grids_match_oracle(ctx, riemann, shape):
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=True, riemann=riemann)
    g = H.Grid.uniform(shape)
    _steps(ctx, g, hp, random_state(g, hp, seed=52, mach=1.5), 3)


@pytest.mark.parametrize("riemann", [HLL, HLLC])
def test_colours_and_corrections_match_oracle(ctx, riemann):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True, riemann=riemann, flatten=3,
                       steepen=1)
    g = H.Grid.uniform((20, 18, 16))
    f = H.sedov(g, hp)
    add_colours(g, f, seed=53)
    H.fill_ghosts(g, f, "outflow")
    _steps(ctx, g, hp, f, 4, bc="outflow")


def test_hllc_fallback_matches_oracle(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, fallback=True, riemann=HLLC)
    g = H.Grid.uniform((20, 12, 10))
    f = random_state(g, hp, seed=10, mach=3.0, contrast=1.5)
    add_colours(g, f, seed=54)
    dt = 3.9 * _dt(g, hp, f)  # drains two cells: HLLC falls back to HLL there
    f_ora, f_gpu = copy_fields(f), copy_fields(f)
    rc, st_o = O.solve_ppm_de(g, hp, dt, 0, f_ora, g.cellwidth)
    rc_g, st_g = ctx.solve_ppm_de(g, hp, dt, 0, f_gpu)
    assert rc == 0 and rc_g == capi.OK
    assert st_o["fallbacks"] == 2 and st_g["fallbacks"] == 2
    _bitexact(f_gpu, f_ora, g)


@pytest.mark.parametrize("riemann", [HLL, HLLC])
def test_negative_density_is_fatal(ctx, riemann):
    # HLL stops on it whatever RiemannSolverFallback says; HLLC without the fallback too
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, fallback=(riemann == HLL),
                       riemann=riemann)
    g = H.Grid.uniform((20, 12, 10))
    f = random_state(g, hp, seed=7, mach=3.0, contrast=1.5)
    dt = 5.0 * _dt(g, hp, f)
    rc, st_o = O.solve_ppm_de(g, hp, dt, 0, copy_fields(f), g.cellwidth)
    rc_g, st_g = ctx.solve_ppm_de(g, hp, dt, 0, copy_fields(f), check=False)
    assert rc != 0 and rc_g == capi.ERR_NEGATIVE
    assert st_g["fatal_cells"] > 0 and st_g["fallbacks"] == 0


@pytest.mark.parametrize("graphs", [False, True])
def test_level_batch_matches_oracle(ctx, graphs):
    torch = pytest.importorskip("torch")
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True, riemann=HLLC)
    rng = np.random.default_rng(55)
    grids, host = [], []
    for k in range(6):
        g = H.Grid.uniform(tuple(int(x) for x in rng.integers(8, 20, size=3)))
        f = H.sedov(g, hp) if k % 2 == 0 else random_state(g, hp, seed=60 + k, mach=2.0)
        H.fill_ghosts(g, f, "periodic")
        grids.append(g)
        host.append(f)
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    ora = [copy_fields(f) for f in host]
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.set_graphs(graphs)
    try:
        for cyc in range(3):
            dt = min(hp.cfl * _dt(g, hp, f) for g, f in zip(grids, ora))
            dt_dev.fill_(dt)
            rc, _ = ctx.solve_level(grids, hp, dt, cyc, dev, dt_device=dt_dev if graphs else None)
            assert rc == capi.OK
            torch.cuda.synchronize()
            for k, g in enumerate(grids):
                rc, _ = O.solve_ppm_de(g, hp, dt, cyc, ora[k], g.cellwidth)
                assert rc == 0
                _bitexact({n: v.cpu().numpy() for n, v in dev[k].items()}, ora[k], g, (cyc, k))
                H.fill_ghosts(g, ora[k], "periodic")
                for n, v in dev[k].items():
                    v.copy_(torch.from_numpy(np.ascontiguousarray(ora[k][n])))
    finally:
        ctx.set_graphs(False)


def test_unknown_solver_is_unsupported(ctx):
    hp = H.HydroParams(riemann=2)  # Marquina: not a PPM option
    g = H.Grid.uniform((8, 8, 8))
    rc, _ = ctx.solve_ppm_de(g, hp, 1e-3, 0, random_state(g, hp, seed=1), check=False)
    assert rc == capi.ERR_UNSUPPORTED


@pytest.mark.parametrize("riemann", [5, HLL, HLLC])
def test_gravity_colours_and_options_together(ctx, riemann):
    # the options at once: gravity, colours, flattening + steepening, with each solver
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True, gravity=True, riemann=riemann,
                       flatten=2, steepen=1)
    g = H.Grid.uniform((15, 13, 11))
    f = random_state(g, hp, seed=91, mach=2.0)
    add_colours(g, f, seed=92)
    rng = np.random.default_rng(93)
    accel = [0.1 * rng.standard_normal(g.shape) for _ in range(3)]
    f_gpu, f_ora = copy_fields(f), copy_fields(f)
    for cyc in range(3):
        dt = hp.cfl * _dt(g, hp, f_ora)
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth, accel=accel)
        assert rc == 0
        rc, _ = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu, accel=accel)
        assert rc == capi.OK
        _bitexact(f_gpu, f_ora, g, cyc)
        H.fill_ghosts(g, f_ora, "periodic")
        H.fill_ghosts(g, f_gpu, "periodic")
