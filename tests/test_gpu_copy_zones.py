"""Sibling and periodic-image zone copies of a level on the device
(ppm_b200_copy_zones_level) against a host restatement of grid::CopyZonesFromGrid
(Grid_CopyZonesFromGrid.C:37-300: overlap of this grid's whole region, moved by each
periodic EdgeOffset, with the other grid's active region, in problem-space positions
converted to indices with nint).  Levels that tile a periodic domain, levels with holes,
a non-periodic axis, and the single-grid case, which must equal the periodic ghost fill."""
import itertools

import numpy as np
import pytest

from ppm_b200 import capi
from ppm_b200 import harness as H

pytestmark = pytest.mark.gpu

NG = H.NGHOST


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    t.cuda.set_device(0)
    return t


def _nint(x):
    return int(np.floor(x + 0.5))


def copy_zones_host(grids, fields, left, domain, periodic):
    """The reference's loop: for every grid (this) and every grid (other), for every
    periodic EdgeOffset of this grid, copy other's active zones that overlap this grid's
    whole region.  Positions in units where the level's zone width is h = 1/domain."""
    h = [1.0 / domain[d] for d in range(3)]
    out = [{k: v.copy() for k, v in f.items()} for f in fields]
    rank = grids[0].rank
    offs = [(-1, 0, 1) if (d < rank and periodic[d]) else (0,) for d in range(3)]
    for a, ga in enumerate(grids):
        for b, gb in enumerate(grids):
            for img in itertools.product(*offs):
                edge = [img[d] * 1.0 for d in range(3)]  # EdgeOffset in domain widths
                start, other_start, dim = [0] * 3, [0] * 3, [1] * 3
                skip = False
                for d in range(rank):
                    cell_left0 = left[a][d] * h[d]
                    grid_left = cell_left0 + edge[d]
                    grid_right = (left[a][d] + ga.dims[d] - 1) * h[d] + h[d] + edge[d]
                    o_left = (left[b][d] + gb.start[d]) * h[d]
                    o_right = (left[b][d] + gb.end[d] + 1) * h[d]
                    if grid_left >= o_right or grid_right <= o_left:
                        skip = True
                        break
                    lo, hi = max(grid_left, o_left), min(grid_right, o_right)
                    s = _nint((lo - grid_left) / h[d])
                    e = _nint((hi - grid_left) / h[d]) - 1
                    if e - s < 0:
                        skip = True
                        break
                    start[d], dim[d] = s, e - s + 1
                    other_start[d] = _nint((lo - left[b][d] * h[d]) / h[d])
                if skip:
                    continue
                dst = tuple(slice(start[d], start[d] + dim[d]) for d in (2, 1, 0))
                src = tuple(slice(other_start[d], other_start[d] + dim[d]) for d in (2, 1, 0))
                for k in out[a]:
                    out[a][k][dst] = fields[b][k][src]
    return out


def _level(domain, boxes, dual, seed):
    """Grids from active boxes [(lo, hi) per axis] of a level; random field values."""
    rng = np.random.default_rng(seed)
    grids, left, host = [], [], []
    for box in boxes:
        g = H.Grid.uniform(tuple(hi - lo for lo, hi in box))
        grids.append(g)
        left.append([box[d][0] - NG for d in range(len(box))] + [0] * (3 - len(box)))
        f = H.new_fields(g, dual)
        for k in f:
            f[k][...] = rng.standard_normal(f[k].shape)
        host.append(f)
    return grids, left, host


def _filled(g, dual):
    return ["d", "te"] + ["v1", "v2", "v3"][:g.rank] + (["ge"] if dual else [])


def _run(torch, grids, left, host, domain, periodic, dual):
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in host]
    ctx = capi.Context(0)
    ctx.copy_zones_level(grids, dev, left, domain, periodic, dual)
    torch.cuda.synchronize()
    ctx.close()
    return [{k: v.cpu().numpy() for k, v in f.items()} for f in dev]


TILED = [((0, 10), (0, 8), (0, 16)), ((10, 24), (0, 8), (0, 16)),
         ((0, 10), (8, 20), (0, 7)), ((0, 10), (8, 20), (7, 16)),
         ((10, 24), (8, 20), (0, 16))]


@pytest.mark.parametrize("periodic", [(1, 1, 1), (1, 1, 0), (0, 1, 1)])
@pytest.mark.parametrize("holes", [False, True])
def test_level_copies_match_reference(torch, periodic, holes):
    domain = (24, 20, 16)
    boxes = TILED[:3] + TILED[4:] if holes else TILED
    grids, left, host = _level(domain, boxes, True, seed=3)
    got = _run(torch, grids, left, host, domain, periodic, True)
    ref = copy_zones_host(grids, host, left, domain, periodic)
    for k, g in enumerate(grids):
        for name in _filled(g, True):
            assert np.array_equal(got[k][name], ref[k][name]), (k, name)


def test_tiled_periodic_level_reproduces_the_global_field(torch):
    domain = (24, 20, 16)
    grids, left, host = _level(domain, TILED, False, seed=8)
    rng = np.random.default_rng(1)
    glob = {k: rng.standard_normal(domain[::-1]) for k in host[0]}
    for g, lf, f in zip(grids, left, host):  # active zones from the global field
        sl = tuple(slice(lf[d] + NG, lf[d] + NG + g.dims[d] - 2 * NG) for d in (2, 1, 0))
        act = g.active_slices()
        for k in f:
            f[k][act] = glob[k][sl]
    got = _run(torch, grids, left, host, domain, (1, 1, 1), False)
    for g, lf, f in zip(grids, left, got):  # every zone, ghosts included, is the global one
        idx = [np.arange(lf[d], lf[d] + g.dims[d]) % domain[d] for d in range(3)]
        for k in _filled(g, False):
            assert np.array_equal(f[k], glob[k][np.ix_(idx[2], idx[1], idx[0])]), k


@pytest.mark.parametrize("shape", [(19,), (12, 9), (10, 8, 7)])
def test_single_grid_equals_periodic_fill(torch, shape):
    g = H.Grid.uniform(shape)
    f = H.new_fields(g, True)
    rng = np.random.default_rng(2)
    for k in f:
        f[k][...] = rng.standard_normal(f[k].shape)
    domain = list(shape) + [1] * (3 - len(shape))
    left = [[-NG] * len(shape) + [0] * (3 - len(shape))]
    got = _run(torch, [g], left, [f], domain, (1, 1, 1), True)[0]
    ref = {k: v.copy() for k, v in f.items()}
    H.fill_ghosts(g, ref, "periodic")
    for k in _filled(g, True):
        assert np.array_equal(got[k], ref[k]), k
