"""Multi-rank host logic on CPU ranks (gloo, world size 2): the z-slab decomposition
of a uniform grid with its halo exchange and global time step reproduces the undivided
grid bit for bit; the AMR-level partition covers every patch once and balances cells.

The ranks advance their slabs with the CPU oracle, so the test runs without a GPU; the
GPU path is the same host code with device tensors and NCCL."""
import os
import socket

import numpy as np
import pytest

from ppm_b200 import harness as H
from ppm_b200 import parallel as PAR
from parity_util import random_state


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _slab_worker(rank, world, port, bc, steps, out_path):
    import torch
    import torch.distributed as dist
    import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
        S = PAR.Slabs((12, 10, 16), world, bc=bc)
        glob = random_state(S.global_grid, hp, seed=21)
        g = S.slab(rank)
        f = S.scatter(glob, rank)
        tf = {k: torch.from_numpy(v) for k, v in f.items()}  # shares memory with f
        for cyc in range(steps):
            S.exchange(tf, rank, dist)
            H.fill_ghosts(g, f, S.local_bc())
            p = O.compute_pressure(g, hp, f)
            dt_local = hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)
            dt = float(PAR.global_min(dt_local, dist).item())
            rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
            assert rc == 0
        # gather the active layers on rank 0
        gathered = {k: np.zeros_like(v) for k, v in glob.items()}
        S.gather_active(f, rank, gathered)
        for k in sorted(gathered):
            t = torch.from_numpy(gathered[k])
            dist.all_reduce(t, op=dist.ReduceOp.SUM)  # disjoint layers: the sum assembles
        if rank == 0:
            np.savez(out_path, **gathered)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bc", [("periodic",) * 3, ("periodic", "periodic", "outflow")])
def test_z_slabs_reproduce_the_undivided_grid(tmp_path, bc):
    import torch.multiprocessing as mp
    import oracle as O

    steps = 4
    out = str(tmp_path / "slabs.npz")
    mp.start_processes(_slab_worker, args=(2, _free_port(), bc, steps, out), nprocs=2,
                       join=True, start_method="spawn")
    got = dict(np.load(out))
    # the same steps on the undivided grid
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    S = PAR.Slabs((12, 10, 16), 2, bc=bc)
    g = S.global_grid
    f = random_state(g, hp, seed=21)
    for cyc in range(steps):
        H.fill_ghosts(g, f, bc)
        p = O.compute_pressure(g, hp, f)
        dt = hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
        assert rc == 0
    act = g.active_slices()
    for k in f:
        assert np.array_equal(got[k][act], f[k][act]), k


def test_single_rank_exchange_is_the_periodic_fill():
    import torch
    hp = H.HydroParams(dual=True)
    S = PAR.Slabs((6, 5, 9), 1)
    g = S.slab(0)
    f = random_state(g, hp, seed=3)
    rng = np.random.default_rng(0)
    for k in f:
        f[k] += rng.standard_normal(f[k].shape)  # scramble the ghosts
    ref = {k: v.copy() for k, v in f.items()}
    H.fill_ghosts(g, ref, "periodic")
    S.exchange({k: torch.from_numpy(v) for k, v in f.items()}, 0, None)
    H.fill_ghosts(g, f, S.local_bc())
    for k in f:
        assert np.array_equal(f[k], ref[k]), k


def test_level_partition_covers_and_balances():
    hp = H.HydroParams(dual=True)
    grids, _ = H.amr_level(hp, npatch=120, seed=7, source_n=32)
    for nr in (1, 2, 3, 8):
        parts = PAR.partition_level(grids, nr)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(grids)))
        loads = [sum(grids[k].size for k in p) for p in parts]
        biggest = max(g.size for g in grids)
        assert max(loads) - min(loads) <= biggest
