"""ppm_b200_euler_sweep_static: one directional sweep that allocates no device memory.

It exists for callers that cannot call cudaMalloc when they advance a grid -- code
running under a memory arena that owns all device memory, or inside a callback where
an allocation could synchronise the device or deadlock.  Such a caller passes its own
device arrays for the inputs and outputs and must get the same fields as from the
allocating entry point (and the oracle).  The file name sorts last so that, when a run
stops at the first failure, every other test has already run.
"""
import numpy as np
import pytest

import oracle as O
from ppm_b200 import capi
from ppm_b200 import harness as H
from parity_util import compare, copy_fields, random_state

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the one-step bar of the parity tests


def _device(fields, torch):
    return {k: torch.from_numpy(v.copy()).cuda() for k, v in fields.items()}


def _host(fields):
    return {k: v.cpu().numpy() for k, v in fields.items()}


def _assert_same(a, b, g, what):
    for k, r in compare(a, b, g).items():
        assert r["maxrel"] <= TOL, (what, k, r)
        assert r["bitexact"], (what, k, r)


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
    for call, dim in enumerate((0, 1, 2)):
        ctx.euler_sweep(dim, g, hp, dt, ref, pres, memory=capi.MEM_DEVICE)
        out = {k: torch.full_like(v, float("nan")) for k, v in cur.items()}
        rc, st = capi.euler_sweep_static(dim, g, hp, dt, cur, pres, out)
        torch.cuda.synchronize()
        assert rc == capi.OK, capi.error_string(rc)
        assert st["interfaces"] > 0
        _assert_same(_host(out), _host(ref), g, call)
        cur = out
    ctx.close()


@pytest.mark.parametrize("shape,dual,grav", [
    ((20, 14, 12), True, False),
    ((18, 16, 10), False, True),
    ((15, 13, 11), True, True),
    ((22, 18), True, True),
    ((40,), False, False),
    ((40,), True, True),
])
def test_static_sweep_every_direction_matches_oracle_without_allocating(shape, dual, grav):
    # every sweep direction of ranks 1-3, dual energy on and off, gravity on and off:
    # the static entry point against the allocating one and against the oracle, bit for
    # bit; then a second call with the same inputs gives the same fields (the shared
    # scratch keeps the first call's contents) and leaves the device's free memory as it
    # was (no allocation by the library, torch's allocator or anything else)
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=dual, gravity=grav)
    g = H.Grid.uniform(shape)
    ctx = capi.Context(0)
    for dim in range(g.rank):
        host = random_state(g, hp, seed=90 + 7 * dim + len(shape))
        accel = None
        if grav:
            rng = np.random.default_rng(5 + dim)
            accel = [0.1 * rng.standard_normal(g.shape) for _ in range(g.rank)]
        p = O.compute_pressure(g, hp, host)
        dt = hp.cfl * O.calc_dt(g, hp, host, p, g.cellwidth)
        ora = copy_fields(host)
        rc, _ = O.sweep(dim, g, hp, dt, ora, p, g.cellwidth, accel=accel)
        assert rc == 0
        pres = torch.from_numpy(p).cuda()
        acc_d = [torch.from_numpy(a).cuda() for a in accel] if accel else None
        ref = _device(host, torch)
        ctx.euler_sweep(dim, g, hp, dt, ref, pres, memory=capi.MEM_DEVICE, accel=acc_d)
        fin = _device(host, torch)
        outs = []
        for call in range(2):
            out = {k: torch.full_like(v, float("nan")) for k, v in fin.items()}
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc, st = capi.euler_sweep_static(dim, g, hp, dt, fin, pres, out, accel=acc_d)
            torch.cuda.synchronize()
            free1 = torch.cuda.mem_get_info()[0]
            assert rc == capi.OK, (dim, call, capi.error_string(rc))
            if call == 1:  # the first call may load the kernels' code; the second may not
                assert free1 == free0, (dim, free0 - free1)
            outs.append(_host(out))
        _assert_same(outs[0], _host(ref), g, ("allocating", dim))
        _assert_same(outs[0], ora, g, ("oracle", dim))
        _assert_same(outs[1], outs[0], g, ("second call", dim))
    ctx.close()


def test_static_sweep_rejects_sizes_beyond_its_limit():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    # pencils longer than 1031 cells
    g = H.Grid.uniform((1034, 1, 1))
    f = _device(H.new_fields(g, True), torch)
    out = {k: torch.zeros_like(v) for k, v in f.items()}
    rc, _ = capi.euler_sweep_static(0, g, hp, 1e-3, f, torch.zeros_like(f["d"]), out)
    assert rc == capi.ERR_TOO_LARGE
    # interface planes beyond 48 MiB: 70^3 active cells
    g = H.Grid.uniform((70, 70, 70))
    f = _device(H.new_fields(g, True), torch)
    out = {k: torch.zeros_like(v) for k, v in f.items()}
    rc, _ = capi.euler_sweep_static(1, g, hp, 1e-3, f, torch.zeros_like(f["d"]), out)
    assert rc == capi.ERR_TOO_LARGE
    assert capi.error_string(rc).startswith("size exceeds")


def test_static_sweep_rejects_overlapping_outputs_and_stream_capture():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True)
    g = H.Grid.uniform((12, 10, 8))
    host = random_state(g, hp, seed=3)
    f = _device(host, torch)
    pres = torch.from_numpy(O.compute_pressure(g, hp, host)).cuda()
    before = _host(f)
    # in place (outputs are the inputs), and an output that is the pressure array
    rc, _ = capi.euler_sweep_static(1, g, hp, 1e-3, f, pres, f)
    assert rc == capi.ERR_INVALID
    out = {k: torch.zeros_like(v) for k, v in f.items()}
    out["te"] = pres
    rc, _ = capi.euler_sweep_static(1, g, hp, 1e-3, f, pres, out)
    assert rc == capi.ERR_INVALID
    # under stream capture the call returns before it touches the stream
    out = {k: torch.zeros_like(v) for k, v in f.items()}
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        graph.capture_begin()
        rc, _ = capi.euler_sweep_static(1, g, hp, 1e-3, f, pres, out, stream=s.cuda_stream)
        scratch = torch.zeros(1, device="cuda")  # keeps the captured graph non-empty
        graph.capture_end()
    torch.cuda.synchronize()
    assert rc == capi.ERR_INVALID
    del graph, scratch
    after = _host(f)
    for k in before:
        assert np.array_equal(before[k], after[k]), k
