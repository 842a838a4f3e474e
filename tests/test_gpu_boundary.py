"""Ghost-zone fill on the device (ppm_b200_set_boundary / _set_boundary_level) against the
host reference fill (harness.fill_ghosts): every boundary kind per axis (periodic,
outflow, left alone for a halo exchange), ranks 1-3, odd and even extents, a single grid
and a level of differently shaped grids in one launch.  Bit-identical (it is a copy)."""
import numpy as np
import pytest

from ppm_b200 import capi
from ppm_b200 import harness as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    t.cuda.set_device(0)
    return t


def _random_fields(g, dual, seed):
    rng = np.random.default_rng(seed)
    f = H.new_fields(g, dual)
    for k in f:
        if f[k] is not None:
            f[k][...] = rng.standard_normal(f[k].shape)
    return f


def _filled(g, dual):
    """The fields a grid of this rank has: velocities beyond the rank are not passed."""
    return ["d", "te"] + ["v1", "v2", "v3"][:g.rank] + (["ge"] if dual else [])


def _dev(f, torch):
    return {k: (torch.from_numpy(v).cuda() if v is not None else None) for k, v in f.items()}


BCS = [("periodic",) * 3, ("outflow",) * 3, ("periodic", "outflow", "none"),
       ("none", "periodic", "outflow")]
SHAPES = [(37,), (16, 9), (12, 7, 5), (32, 30, 33)]


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("shape", SHAPES)
def test_fill_matches_host(torch, shape, bc):
    g = H.Grid.uniform(shape)
    for dual in (False, True):
        host = _random_fields(g, dual, seed=len(shape) * 7 + len(bc[0]))
        dev = _dev(host, torch)
        ctx = capi.Context(0)
        ctx.set_boundary(g, dev, dual, bc)
        torch.cuda.synchronize()
        H.fill_ghosts(g, host, bc)
        for k in _filled(g, dual):
            assert np.array_equal(dev[k].cpu().numpy(), host[k]), (shape, bc, dual, k)
        ctx.close()


def test_level_fill_matches_host(torch):
    bc = ("periodic", "outflow", "periodic")
    rng = np.random.default_rng(11)
    grids = [H.Grid.uniform(tuple(int(x) for x in rng.integers(3, 40, size=3)))
             for _ in range(25)]
    host = [_random_fields(g, True, seed=k) for k, g in enumerate(grids)]
    dev = [_dev(f, torch) for f in host]
    ctx = capi.Context(0)
    ctx.set_boundary_level(grids, dev, True, bc)
    torch.cuda.synchronize()
    for k, g in enumerate(grids):
        H.fill_ghosts(g, host[k], bc)
        for name in _filled(g, True):
            assert np.array_equal(dev[k][name].cpu().numpy(), host[k][name]), (k, name)
    ctx.close()
