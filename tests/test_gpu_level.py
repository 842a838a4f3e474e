"""AMR-level batching: every grid of a level advanced by one launch per kernel stage.

The reference advances a level grid by grid (EvolveLevel.C:569-585 calls
grid::SolveHydroEquations -> SolvePPM_DE once per grid; SetLevelTimeStep.C:66 takes
the min of grid::ComputeTimeStep).  The level entry points must give, for every grid,
the fields the single-grid entry point gives, bit for bit, and the oracle's fields.
"""
import numpy as np
import pytest

import oracle as O
from ppm_b200 import capi
from ppm_b200 import harness as H
from parity_util import compare, copy_fields, random_state

pytestmark = pytest.mark.gpu

# patches of one level: ragged sizes, one 2-cell-thin patch, different cell widths;
# (8, 8, 8) before (10, 18, 6) etc. makes later sweep directions need more face scratch
# than the first
LEVEL_SHAPES = [(16, 16, 16), (24, 12, 8), (8, 8, 8), (10, 18, 6), (32, 8, 12),
                (6, 6, 20), (12, 14, 16), (2, 9, 7), (20, 20, 4)]


def _level(hp, seed0, shapes=LEVEL_SHAPES):
    grids, fields = [], []
    for k, shp in enumerate(shapes):
        g = H.Grid.uniform(shp, width=tuple(0.25 * s / 8.0 for s in shp))
        grids.append(g)
        fields.append(random_state(g, hp, seed=seed0 + k))
    return grids, fields


def _dev(f, torch):
    return {k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()}


def _host(f):
    return {k: v.cpu().numpy() for k, v in f.items()}


def _assert_same(a, b, g, what):
    for k, r in compare(a, b, g).items():
        assert r["bitexact"], (what, k, r)


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    t.cuda.set_device(0)
    return t


@pytest.mark.parametrize("dual,grav", [(True, False), (False, False), (True, True)])
def test_level_solve_matches_per_grid_solves_and_oracle(torch, dual, grav):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=dual, gravity=grav)
    grids, host = _level(hp, 100)
    accels = None
    if grav:
        rng = np.random.default_rng(7)
        accels = [[0.1 * rng.standard_normal(g.shape) for _ in range(g.rank)] for g in grids]
    acc_dev = None if accels is None else [[torch.from_numpy(a).cuda() for a in acc]
                                           for acc in accels]
    ctx = capi.Context(0)
    per_grid = [_dev(f, torch) for f in host]
    batched = [_dev(f, torch) for f in host]
    ora = [copy_fields(f) for f in host]
    for cyc in range(4):  # every rotation of the sweep order, and one more
        dt = min(hp.cfl * O.calc_dt(g, hp, f, O.compute_pressure(g, hp, f), g.cellwidth)
                 for g, f in zip(grids, ora))
        for k, g in enumerate(grids):
            acc = None if accels is None else acc_dev[k]
            ctx.solve_ppm_de(g, hp, dt, cyc, per_grid[k], memory=capi.MEM_DEVICE, accel=acc,
                             want_stats=False)
            rc, _ = O.solve_ppm_de(g, hp, dt, cyc, ora[k], g.cellwidth,
                                   accel=None if accels is None else accels[k])
            assert rc == 0
        rc, st = ctx.solve_level(grids, hp, dt, cyc, batched, accels=acc_dev, want_stats=True)
        assert rc == capi.OK
        assert st["interfaces"] > 0
        for k, g in enumerate(grids):
            _assert_same(_host(batched[k]), _host(per_grid[k]), g, ("per-grid", cyc, k))
            _assert_same(_host(batched[k]), ora[k], g, ("oracle", cyc, k))
        for k, g in enumerate(grids):
            H.fill_ghosts(g, ora[k], "periodic")
        ctx.set_boundary_level(grids, batched, dual)
        for k in range(len(grids)):
            ctx.set_boundary(grids[k], per_grid[k], dual)
    ctx.close()


@pytest.mark.parametrize("dual,grav", [(True, False), (False, False), (True, True)])
def test_tolerance_build_level_matches_per_grid_solves(torch, dual, grav):
    # the tolerance build (fused multiply-adds, fast reciprocal and square root) is not
    # bit-identical to the oracle, but a grid still gives the same bits in a level batch
    # as alone: the fast reciprocal and square root have no branches, so what the
    # compiler fuses around them does not depend on the kernel's instantiation (one
    # grid's record in the kernel parameters, a batch's in shared memory)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=dual, gravity=grav)
    grids, host = _level(hp, 300)
    acc_dev = None
    if grav:
        rng = np.random.default_rng(11)
        acc_dev = [[torch.from_numpy(0.1 * rng.standard_normal(g.shape)).cuda()
                    for _ in range(g.rank)] for g in grids]
    ctx = capi.Context(0, variant="fast")
    per_grid = [_dev(f, torch) for f in host]
    batched = [_dev(f, torch) for f in host]
    for cyc in range(4):
        dt = ctx.compute_timestep_level(grids, hp, batched)
        for k, g in enumerate(grids):
            ctx.solve_ppm_de(g, hp, dt, cyc, per_grid[k], memory=capi.MEM_DEVICE,
                             accel=None if acc_dev is None else acc_dev[k], want_stats=False)
        rc, _ = ctx.solve_level(grids, hp, dt, cyc, batched, accels=acc_dev, want_stats=True)
        assert rc == capi.OK
        for k, g in enumerate(grids):
            _assert_same(_host(batched[k]), _host(per_grid[k]), g, ("per-grid", cyc, k))
        ctx.set_boundary_level(grids, batched, dual)
        for k in range(len(grids)):
            ctx.set_boundary(grids[k], per_grid[k], dual)
    ctx.close()


def test_level_solve_in_a_fresh_context(torch):
    # the first call sizes every scratch buffer for the level at once; the second
    # sweep direction of these patches needs more face scratch than the first
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    grids, host = _level(hp, 150, shapes=[(6, 24, 24), (8, 20, 30), (4, 16, 16)])
    ora = [copy_fields(f) for f in host]
    dt = min(hp.cfl * O.calc_dt(g, hp, f, O.compute_pressure(g, hp, f), g.cellwidth)
             for g, f in zip(grids, ora))
    ctx = capi.Context(0)
    dev = [_dev(f, torch) for f in host]
    rc, _ = ctx.solve_level(grids, hp, dt, 0, dev, want_stats=True)
    assert rc == capi.OK
    for k, g in enumerate(grids):
        rc, _ = O.solve_ppm_de(g, hp, dt, 0, ora[k], g.cellwidth)
        assert rc == 0
        _assert_same(_host(dev[k]), ora[k], g, ("fresh", k))
    ctx.close()


def test_level_stats_are_the_sum_over_grids(torch):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    grids, host = _level(hp, 200)
    dt = 1e-3
    tot = {"interfaces": 0, "newton_iters": 0}
    for g, f in zip(grids, host):
        rc, st = O.solve_ppm_de(g, hp, dt, 1, copy_fields(f), g.cellwidth)
        assert rc == 0
        for key in tot:
            tot[key] += st[key]
    ctx = capi.Context(0)
    rc, st = ctx.solve_level(grids, hp, dt, 1, [_dev(f, torch) for f in host], want_stats=True)
    assert rc == capi.OK
    for key in tot:
        assert st[key] == tot[key], key
    ctx.close()


def test_level_graph_replay_matches_direct_launches(torch):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    grids, host = _level(hp, 300)
    direct = [_dev(f, torch) for f in host]
    graphed = [_dev(f, torch) for f in host]
    a = capi.Context(0)
    b = capi.Context(0)
    b.set_graphs(True)
    dt_a = torch.zeros(1, dtype=torch.float64, device="cuda")
    dt_b = torch.zeros(1, dtype=torch.float64, device="cuda")
    for cyc in range(7):  # two full rotations: the second replays captured graphs
        a.compute_timestep_level(grids, hp, direct, dt_device=dt_a, want_host=False)
        a.solve_level(grids, hp, 0.0, cyc, direct, dt_device=dt_a)
        a.set_boundary_level(grids, direct, True)
        b.compute_timestep_level(grids, hp, graphed, dt_device=dt_b, want_host=False)
        n0 = b.launches()
        b.solve_level(grids, hp, 0.0, cyc, graphed, dt_device=dt_b)
        assert b.launches() - n0 == 1 + 5 * 3
        b.set_boundary_level(grids, graphed, True)
    assert a.synchronize()[0] == capi.OK
    assert b.synchronize()[0] == capi.OK
    assert dt_a.item() > 0.0 and dt_a.item() == dt_b.item()
    for k, g in enumerate(grids):
        _assert_same(_host(graphed[k]), _host(direct[k]), g, ("graph", k))
    a.close()
    b.close()


def test_level_timestep_and_boundary_match_single_grid_calls(torch):
    for dual in (False, True):
        hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.6, dual=dual)
        grids, host = _level(hp, 400)
        ctx = capi.Context(0)
        dev = [_dev(f, torch) for f in host]
        dts = [ctx.compute_timestep(g, hp, f) for g, f in zip(grids, host)]
        assert ctx.compute_timestep_level(grids, hp, dev) == min(dts)
        rng = np.random.default_rng(3)
        for f in dev:
            for k in f:
                f[k] += torch.from_numpy(rng.standard_normal(tuple(f[k].shape))).cuda()
        ref = [{k: v.clone() for k, v in f.items()} for f in dev]
        bc = ("periodic", "outflow", "periodic")
        ctx.set_boundary_level(grids, dev, dual, bc)
        for g, f in zip(grids, ref):
            ctx.set_boundary(g, f, dual, bc)
        torch.cuda.synchronize()
        for k, g in enumerate(grids):
            for name in dev[k]:
                assert torch.equal(dev[k][name], ref[k][name]), (k, name)
        ctx.close()


def test_level_rejects_mixed_rank(torch):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    grids, host = _level(hp, 500, shapes=[(8, 8, 8), (8, 8)])
    ctx = capi.Context(0)
    rc, _ = ctx.solve_level(grids, hp, 1e-3, 0, [_dev(f, torch) for f in host], check=False)
    assert rc == capi.ERR_INVALID
    ctx.close()


@pytest.mark.parametrize("schedule,threads,persistent,scratch", [
    ("per_grid", 128, 0, 0),
    ("classes", (64, 256, 128, 128), (1, 0, 1, 0), 0),
    ("batched", 64, 1, 0),
    ("batched", 256, 0, 0),
    ("batched", 128, 1, 4_000_000),  # waves: a few grids at a time
    ("classes", 128, 0, 1),          # every grid its own wave
])
@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_level_schedules_are_bit_identical(torch, schedule, threads, persistent, scratch,
                                           variant):
    # the level schedules (one batch, one batch per size class, one grid at a time), the
    # Riemann stage's block size and persistent launch, and waves under a scratch bound
    # change how the level is launched, never its results: the same fields and the same
    # folded time step as the default batch, direct and replayed from graphs
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    grids, host = _level(hp, 600)
    ref = [_dev(f, torch) for f in host]
    a = capi.Context(0, variant=variant)
    dt_a = torch.zeros(1, dtype=torch.float64, device="cuda")
    a.compute_timestep_level(grids, hp, ref, dt_device=dt_a, want_host=False)
    a.set_cfl(dt_a, courant=hp.cfl)
    for graphs in (False, True):
        b = capi.Context(0, variant=variant)
        b.set_graphs(graphs)
        # class bounds inside the test level's range of sizes, so every class has grids
        b.set_level_config(schedule=schedule, riemann_threads=threads, persistent=persistent,
                           class_cells=(700, 2500), max_scratch_bytes=scratch)
        cur = [_dev(f, torch) for f in host]
        dt_b = torch.zeros(1, dtype=torch.float64, device="cuda")
        b.compute_timestep_level(grids, hp, cur, dt_device=dt_b, want_host=False)
        b.set_cfl(dt_b, courant=hp.cfl)
        for cyc in range(4):
            b.solve_level(grids, hp, 0.0, cyc, cur, dt_device=dt_b)
            b.set_boundary_level(grids, cur, True)
            if not graphs:
                a.solve_level(grids, hp, 0.0, cyc, ref, dt_device=dt_a)
                a.set_boundary_level(grids, ref, True)
        assert b.synchronize()[0] == capi.OK
        assert a.synchronize()[0] == capi.OK
        # ref advanced the same 4 cycles in the first pass
        assert dt_b.item() == dt_a.item(), (graphs, dt_b.item(), dt_a.item())
        for k, g in enumerate(grids):
            _assert_same(_host(cur[k]), _host(ref[k]), g, (schedule, graphs, k))
        b.set_cfl(None)
        b.close()
    a.set_cfl(None)
    a.close()


def test_level_autotuner_keeps_a_choice_and_leaves_fields_alone(torch):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    grids, host = _level(hp, 700)
    dev = [_dev(f, torch) for f in host]
    before = [_host(f) for f in dev]
    ctx = capi.Context(0)
    ctx.set_level_config(class_cells=(700, 2500), max_scratch_bytes=0)
    dt = ctx.compute_timestep_level(grids, hp, dev)
    rep = ctx.autotune_level(grids, hp, dev, dt)
    assert sum(rep["class_grids"]) == len(grids)
    assert all(ms > 0.0 for ms in rep["batched_ms"]) and rep["classes_ms"] > 0.0
    assert rep["chosen"] == ctx.level_config().as_dict()
    for k, g in enumerate(grids):  # the tuning ran on copies
        for name in before[k]:
            assert np.array_equal(before[k][name], dev[k][name].cpu().numpy()), (k, name)
    # and a solve under the chosen schedule is the oracle's
    ora = [copy_fields(f) for f in host]
    rc, _ = ctx.solve_level(grids, hp, dt, 0, dev, want_stats=True)
    assert rc == capi.OK
    for k, g in enumerate(grids):
        rc, _ = O.solve_ppm_de(g, hp, dt, 0, ora[k], g.cellwidth)
        assert rc == 0
        _assert_same(_host(dev[k]), ora[k], g, ("tuned", k))
    ctx.close()
