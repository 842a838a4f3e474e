"""Colour fields on the GPU (NumberOfColours > 0) against the CPU oracle: every field,
hydro and colour, bit-identical after each step, through the single-grid solve (host and
device memory), the per-direction sweep, the batched level (also replayed from CUDA
graphs), the HLL fallback, the slope corrections, ranks 1-3, and the subgrid capture
of the colour fluxes (Grid_xEulerSweep.C:361-371)."""
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


def _bitexact(got, ref, g, where=""):
    for k, r in compare(got, ref, g).items():
        assert r["bitexact"], (where, k, r)


def _steps(ctx, g, hp, f, n, bc="periodic"):
    f_gpu, f_ora = copy_fields(f), copy_fields(f)
    for cyc in range(n):
        dt = _dt(g, hp, f_ora)
        rc, st_o = O.solve_ppm_de(g, hp, dt, cyc, f_ora, g.cellwidth)
        assert rc == 0
        rc, st_g = ctx.solve_ppm_de(g, hp, dt, cyc, f_gpu)
        assert rc == capi.OK
        assert st_g["fallbacks"] == st_o["fallbacks"]
        _bitexact(f_gpu, f_ora, g, cyc)
        H.fill_ghosts(g, f_ora, bc)
        H.fill_ghosts(g, f_gpu, bc)
    return f_gpu


@pytest.mark.parametrize("dual", [False, True])
def test_random_state_with_colours_matches_oracle(ctx, dual):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=dual)
    g = H.Grid.uniform((18, 14, 12))
    f = random_state(g, hp, seed=41, mach=2.0, contrast=1.0)
    assert add_colours(g, f, seed=42) == 4
    _steps(ctx, g, hp, f, 4)


def test_twelve_colours_matches_oracle(ctx):
    # MultiSpecies = 2 advects 6 + 3 = 9 species colours (Grid_SolveHydroEquations.C:95),
    # plus metals and other tracers
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((13, 11, 9))
    f = random_state(g, hp, seed=5, mach=1.5)
    assert add_colours(g, f, seed=6, fractions=(0.76, 0.24, 0.5, 0.01), extra=7) == 12
    _steps(ctx, g, hp, f, 3)


@pytest.mark.parametrize("shape", [(40,), (20, 16)])
def test_low_rank_grids_with_colours_match_oracle(ctx, shape):
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=True)
    g = H.Grid.uniform(shape)
    f = random_state(g, hp, seed=9, mach=1.5)
    add_colours(g, f, seed=10)
    _steps(ctx, g, hp, f, 3)


def test_corrections_with_colours_match_oracle(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True, flatten=3, steepen=1)
    g = H.Grid.uniform((20, 18, 16))
    f = H.sedov(g, hp)
    add_colours(g, f, seed=3)
    H.fill_ghosts(g, f, "outflow")
    _steps(ctx, g, hp, f, 4, bc="outflow")


def test_hll_fallback_with_colours_matches_oracle(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, fallback=1)
    g = H.Grid.uniform((20, 12, 10))
    f = random_state(g, hp, seed=7)
    for (k, j, i) in [(5, 6, 8), (5, 6, 9), (8, 4, 14), (4, 10, 5)]:
        f["te"][k, j, i] = -1e-3
    add_colours(g, f, seed=8)
    f_ora, f_gpu = copy_fields(f), copy_fields(f)
    dt = _dt(g, hp, f_ora)
    rc, st_o = O.solve_ppm_de(g, hp, dt, 0, f_ora, g.cellwidth)
    rc_g, st_g = ctx.solve_ppm_de(g, hp, dt, 0, f_gpu)
    assert rc == 0 and rc_g == capi.OK
    assert st_o["fallbacks"] == 4 and st_g["fallbacks"] == 4
    _bitexact(f_gpu, f_ora, g)


def test_device_memory_and_sweep_entry_with_colours(ctx):
    torch = pytest.importorskip("torch")
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((16, 12, 10))
    f = random_state(g, hp, seed=13, mach=2.0)
    add_colours(g, f, seed=14)
    dt = _dt(g, hp, f)
    ref = copy_fields(f)
    O.solve_ppm_de(g, hp, dt, 2, ref, g.cellwidth)
    dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()}
    ctx.solve_ppm_de(g, hp, dt, 2, dev, memory=capi.MEM_DEVICE, want_stats=False)
    rc, _ = ctx.synchronize()
    assert rc == capi.OK
    _bitexact({k: v.cpu().numpy() for k, v in dev.items()}, ref, g, "device")
    # one direction at a time (ppm_b200_euler_sweep), host memory
    for dim in range(3):
        a, b = copy_fields(f), copy_fields(f)
        p = O.compute_pressure(g, hp, a)
        rc, _ = O.sweep(dim, g, hp, dt, a, p, g.cellwidth)
        assert rc == 0
        ctx.euler_sweep(dim, g, hp, dt, b, p)
        _bitexact(b, a, g, ("sweep", dim))


def _level(hp, n, seed):
    rng = np.random.default_rng(seed)
    grids, host = [], []
    for k in range(n):
        g = H.Grid.uniform(tuple(int(x) for x in rng.integers(8, 20, size=3)))
        f = H.sedov(g, hp) if k % 3 == 0 else random_state(g, hp, seed=seed + k, mach=2.0)
        add_colours(g, f, seed=seed + 100 + k)
        H.fill_ghosts(g, f, "periodic")
        grids.append(g)
        host.append(f)
    return grids, host


@pytest.mark.parametrize("graphs", [False, True])
def test_level_batch_with_colours_matches_oracle(ctx, graphs):
    torch = pytest.importorskip("torch")
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    grids, host = _level(hp, 7, seed=20)
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    ora = [copy_fields(f) for f in host]
    ctx.set_graphs(graphs)
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    try:
        for cyc in range(3):
            dt = min(_dt(g, hp, f) for g, f in zip(grids, ora))
            dt_dev.fill_(dt)
            rc, _ = ctx.solve_level(grids, hp, dt, cyc, dev, dt_device=dt_dev if graphs else None)
            assert rc == capi.OK
            torch.cuda.synchronize()
            for k, g in enumerate(grids):
                rc, _ = O.solve_ppm_de(g, hp, dt, cyc, ora[k], g.cellwidth)
                assert rc == 0
                got = {n: v.cpu().numpy() for n, v in dev[k].items()}
                _bitexact(got, ora[k], g, (cyc, k))
                H.fill_ghosts(g, ora[k], "periodic")
                for n, v in dev[k].items():
                    v.copy_(torch.from_numpy(np.ascontiguousarray(ora[k][n])))
    finally:
        ctx.set_graphs(False)


def _flux_boxes(lo, hi, ncol, rank=3):
    """Capture boxes (global = local indices) for the GPU and the oracle, with every hydro
    slot and every colour allocated, GPU and oracle arrays distinct."""
    box = {"left_start": [[0] * 3 for _ in range(3)], "left_end": [[0] * 3 for _ in range(3)],
           "right_start": [[0] * 3 for _ in range(3)], "right_end": [[0] * 3 for _ in range(3)],
           "left": [[None] * 3 for _ in range(6)], "right": [[None] * 3 for _ in range(6)],
           "colour_left": [[None] * 3 for _ in range(ncol)],
           "colour_right": [[None] * 3 for _ in range(ncol)]}
    for dim in range(rank):
        for j in range(rank):
            box["left_start"][dim][j] = lo[j]
            box["left_end"][dim][j] = lo[j] if j == dim else hi[j]
            box["right_start"][dim][j] = hi[j] if j == dim else lo[j]
            box["right_end"][dim][j] = hi[j]
        size = 1
        for j in range(rank):
            if j != dim:
                size *= hi[j] - lo[j] + 1
        for side in ("left", "right"):
            for s in range(6):
                box[side][s][dim] = np.zeros(size)
            for n in range(ncol):
                box["colour_" + side][n][dim] = np.zeros(size)
    return box


def _ora_fluxes(box, ncol):
    import ctypes as C
    of = O.OraFluxes()
    for key in ("left_start", "left_end", "right_start", "right_end"):
        arr = getattr(of, key)
        for i in range(3):
            for j in range(3):
                arr[i][j] = int(box[key][i][j])
    dp = C.POINTER(C.c_double)
    for side in ("left", "right"):
        for s in range(6):
            for d in range(3):
                a = box[side][s][d]
                getattr(of, side)[s][d] = a.ctypes.data_as(dp) if a is not None else dp()
        for n in range(ncol):
            for d in range(3):
                a = box["colour_" + side][n][d]
                getattr(of, "colour_" + side)[n][d] = (a.ctypes.data_as(dp) if a is not None
                                                       else dp())
    return of


def test_colour_subgrid_fluxes_match_oracle(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((16, 14, 12))
    f = random_state(g, hp, seed=31, mach=2.0)
    ncol = add_colours(g, f, seed=32)
    lo, hi = (6, 5, 5), (12, 10, 9)
    bg, bo = _flux_boxes(lo, hi, ncol), _flux_boxes(lo, hi, ncol)
    f_gpu, f_ora = copy_fields(f), copy_fields(f)
    dt = _dt(g, hp, f)
    subs = [_ora_fluxes(bo, ncol)]
    rc, _ = O.solve_ppm_de(g, hp, dt, 1, f_ora, g.cellwidth, subgrids=subs, ggs=(0, 0, 0))
    assert rc == 0
    rc, _ = ctx.solve_ppm_de(g, hp, dt, 1, f_gpu, subgrids=[bg], ggs=(0, 0, 0))
    assert rc == capi.OK
    _bitexact(f_gpu, f_ora, g)
    for side in ("left", "right"):
        for dim in range(3):
            for s in range(6):
                assert np.array_equal(bg[side][s][dim], bo[side][s][dim]), (side, s, dim)
            for n in range(ncol):
                a, b = bg["colour_" + side][n][dim], bo["colour_" + side][n][dim]
                assert np.any(a != 0.0)
                assert np.array_equal(a, b), ("colour", side, n, dim)


@pytest.mark.parametrize("bc", ["periodic", "outflow"])
def test_ghost_fill_moves_colours(ctx, bc):
    # SetBoundaryConditions fills every baryon field, colours included
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    grids, host = [], []
    for shape in ((12, 10, 8), (9, 7, 11), (16, 6, 5)):
        g = H.Grid.uniform(shape)
        f = H.new_fields(g, True)
        for k in f:
            f[k][...] = rng.standard_normal(f[k].shape)
        add_colours(g, f, seed=int(rng.integers(1000)), extra=9)  # 12 colours: two chunks
        grids.append(g)
        host.append(f)
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    ctx.set_boundary(grids[0], dev[0], True, (bc,) * 3)
    ctx.set_boundary_level(grids[1:], dev[1:], True, (bc,) * 3)
    torch.cuda.synchronize()
    for g, f, d in zip(grids, host, dev):
        ref = copy_fields(f)
        H.fill_ghosts(g, ref, bc)
        for k in ref:
            assert np.array_equal(d[k].cpu().numpy(), ref[k]), k


def test_zone_copies_move_colours(ctx):
    torch = pytest.importorskip("torch")
    from test_gpu_copy_zones import TILED, copy_zones_host
    domain = (24, 20, 16)
    rng = np.random.default_rng(8)
    grids, left, host = [], [], []
    for box in TILED:
        g = H.Grid.uniform(tuple(hi - lo for lo, hi in box))
        f = H.new_fields(g, True)
        for k in f:
            f[k][...] = rng.standard_normal(f[k].shape)
        add_colours(g, f, seed=int(rng.integers(1000)), extra=5)  # 8 colours
        grids.append(g)
        left.append([box[d][0] - H.NGHOST for d in range(3)])
        host.append(f)
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    ctx.copy_zones_level(grids, dev, left, domain, (1, 1, 1), True)
    torch.cuda.synchronize()
    ref = copy_zones_host(grids, host, left, domain, (1, 1, 1))
    for k in range(len(grids)):
        for name in ref[k]:
            assert np.array_equal(dev[k][name].cpu().numpy(), ref[k][name]), (k, name)
