"""Comoving expansion terms (grid::ComovingExpansionTerms with expand_terms.F,
ENERGY_METHOD3 / VELOCITY_METHOD3) against the CPU oracle: bit-identical fields, with
the time-centred (interpolated) pressure and with the current-time pressure, single
grids and a batched level."""
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
    yield c
    c.close()


@pytest.mark.parametrize("shape,dual,with_old", [
    ((12, 10, 8), True, True),
    ((12, 10, 8), False, True),
    ((12, 10, 8), True, False),
    ((16, 9), False, True),
    ((30,), True, True),
])
def test_expansion_terms_match_oracle(ctx, shape, dual, with_old):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=dual)
    g = H.Grid.uniform(shape)
    f = random_state(g, hp, seed=70)
    old = random_state(g, hp, seed=71) if with_old else None
    f_ora = copy_fields(f)
    # Time, OldTime and dt * adot / a of a cosmological step
    t, t_old, coef = 0.8125, 0.8, 0.0123
    O.expansion_terms(g, hp, f_ora, old, t, t_old, coef)
    ctx.expansion_terms(g, hp, f, old, t, t_old, coef)
    for k, r in compare(f, f_ora, g).items():
        assert r["bitexact"], (k, r)
    assert not np.array_equal(f["te"], random_state(g, hp, seed=70)["te"])


def test_expansion_terms_level_matches_single_grids(ctx):
    torch = pytest.importorskip("torch")
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    grids = [H.Grid.uniform(s) for s in ((8, 8, 8), (12, 6, 10), (5, 9, 7))]
    cur = [random_state(g, hp, seed=80 + k) for k, g in enumerate(grids)]
    old = [random_state(g, hp, seed=90 + k) for k, g in enumerate(grids)]
    dev = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in cur]
    dold = [{k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()} for f in old]
    torch.cuda.synchronize()
    ctx.expansion_terms_level(grids, hp, dev, dold, 2.0, 1.9, 0.02)
    ctx.synchronize()
    for k, g in enumerate(grids):
        ref = copy_fields(cur[k])
        O.expansion_terms(g, hp, ref, old[k], 2.0, 1.9, 0.02)
        got = {n: v.cpu().numpy() for n, v in dev[k].items()}
        for n, r in compare(got, ref, g).items():
            assert r["bitexact"], (k, n, r)
