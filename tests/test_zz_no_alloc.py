"""ppm_b200_euler_sweep_static: one directional sweep that allocates no device memory.

It exists for callers that cannot call cudaMalloc when they advance a grid -- code
running under a memory arena that owns all device memory, or inside a callback where
an allocation could synchronise the device or deadlock.  Such a caller passes its own
device arrays for the inputs and outputs and must get the same fields as from the
allocating entry point.  The file name sorts last so that, when a run stops at the
first failure, every other test has already run.
"""
import numpy as np
import pytest

from ppm_b200 import capi
from ppm_b200 import harness as H
from parity_util import compare, random_state

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the one-step bar of the parity tests


def _device(fields, torch):
    return {k: torch.from_numpy(v.copy()).cuda() for k, v in fields.items()}


def test_static_sweep_matches_allocating_entry_point_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    g = H.Grid.uniform((24, 20, 16))
    host = random_state(g, hp, seed=77)
    ctx = capi.Context(0)
    pres_host = np.zeros_like(host["d"])
    ctx.compute_pressure(g, hp, host, pres_host)          # host mode: synchronous
    dt = ctx.compute_timestep(g, hp, host)
    pres = torch.from_numpy(pres_host).cuda()
    ref = _device(host, torch)   # advanced by the allocating entry point
    cur = _device(host, torch)   # advanced by the static one
    torch.cuda.synchronize()
    for call, dim in enumerate((0, 1)):
        ctx.euler_sweep(dim, g, hp, dt, ref, pres, memory=capi.MEM_DEVICE)
        out = {k: torch.full_like(v, float("nan")) for k, v in cur.items()}
        rc, st = capi.euler_sweep_static(dim, g, hp, dt, cur, pres, out)
        torch.cuda.synchronize()
        assert rc == capi.OK, capi.error_string(rc)
        assert st["interfaces"] > 0
        a = {k: v.cpu().numpy() for k, v in out.items()}
        b = {k: v.cpu().numpy() for k, v in ref.items()}
        for k, r in compare(a, b, g).items():
            assert r["maxrel"] <= TOL, (call, k, r)
            assert r["bitexact"], (call, k, r)
        cur = out
    ctx.close()


def test_static_sweep_rejects_sizes_beyond_its_limit():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    # pencils longer than 1031 cells
    g = H.Grid.uniform((1034, 1, 1))
    f = _device(H.new_fields(g, True), torch)
    out = {k: torch.zeros_like(v) for k, v in f.items()}
    rc, _ = capi.euler_sweep_static(0, g, hp, 1e-3, f, f["d"], out)
    assert rc == capi.ERR_TOO_LARGE
    # interface planes beyond 48 MiB: 70^3 active cells
    g = H.Grid.uniform((70, 70, 70))
    f = _device(H.new_fields(g, True), torch)
    out = {k: torch.zeros_like(v) for k, v in f.items()}
    rc, _ = capi.euler_sweep_static(1, g, hp, 1e-3, f, f["d"], out)
    assert rc == capi.ERR_TOO_LARGE
    assert capi.error_string(rc).startswith("size exceeds")
