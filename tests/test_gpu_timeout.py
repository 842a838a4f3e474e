"""The bounded device waits: with the test hook ppm_b200_debug_tma_stall every TMA chunk
of the x sweep's update kernel expects more bytes than its copies deliver, so its
barrier never completes.  Each wait gives up after about a second, the kernel drains
and returns, the call reports PPM_B200_ERR_TIMEOUT, and the same context then solves
normally, bit-identical to the oracle.  Nothing faults or hangs."""
import numpy as np
import pytest

import oracle as O
from ppm_b200 import capi
from ppm_b200 import harness as H
from parity_util import compare, copy_fields, random_state

pytestmark = pytest.mark.gpu


def test_stalled_tma_waits_time_out_and_the_context_recovers():
    ctx = capi.Context(0)
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((16, 10, 8))  # even x extent: the x update reads TMA tiles
    f = random_state(g, hp, seed=4)
    p = O.compute_pressure(g, hp, f)
    dt = hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)
    try:
        ctx.debug_tma_stall(16)
        junk = copy_fields(f)
        rc, _ = ctx.solve_ppm_de(g, hp, dt, 0, junk, check=False)
        assert rc == capi.ERR_TIMEOUT
    finally:
        ctx.debug_tma_stall(0)
    f_gpu, f_ora = copy_fields(f), copy_fields(f)
    rc, _ = ctx.solve_ppm_de(g, hp, dt, 0, f_gpu)
    assert rc == capi.OK
    assert O.solve_ppm_de(g, hp, dt, 0, f_ora, g.cellwidth)[0] == 0
    for k, r in compare(f_gpu, f_ora, g).items():
        assert r["bitexact"], (k, r)
    ctx.close()


def test_stall_hook_rejects_bad_sizes():
    ctx = capi.Context(0)
    for bad in (-16, 8, 8192):
        with pytest.raises(capi.PPMError):
            ctx.debug_tma_stall(bad)
    ctx.close()
