"""SUBling flux correction on the GPU (ppm_b200_correct_fluxes_sublings) against the
oracle: bit-identical fields and refined fluxes for right and left contacts along every
axis, a contact across a periodic level boundary, several siblings in turn, and the undo
of corrections that would leave a density or energy non-positive (including the
reference's right-face undo, which subtracts the triggering field's amount,
Grid_CorrectForRefinedFluxes.C:643-645)."""
import numpy as np
import pytest

import oracle as O
from flux_fix_util import ora_fluxes
from parity_util import copy_fields, random_state
from ppm_b200 import capi
from ppm_b200 import harness as H
from subling_util import copy_box, gbox, own_box

pytestmark = pytest.mark.gpu

GGS = (10, 20, 30)  # active global x 13..20, y 23..28, z 33..36 for an 8x6x4 grid


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _compare(ctx, g, hp, f, own, refs, ggs, level, periodic):
    f_ora, f_gpu = copy_fields(f), copy_fields(f)
    r_ora = [copy_box(r) for r in refs]
    r_gpu = [copy_box(r) for r in refs]
    of = ora_fluxes(own)
    rf = [ora_fluxes(r) for r in r_ora]
    assert O.correct_fluxes_sublings(g, hp, f_ora, of, rf, ggs, level, periodic) == 0
    ctx.correct_fluxes_sublings(g, hp, f_gpu, own, r_gpu, ggs, level, periodic)
    for k in f:
        assert np.array_equal(f_gpu[k], f_ora[k]), k
    for a, b in zip(r_gpu, r_ora):
        for side in ("left", "right"):
            for s in range(6):
                for d in range(3):
                    if a[side][s][d] is not None:
                        assert np.array_equal(a[side][s][d], b[side][s][d]), (side, s, d)
    return f_gpu


# sibling regions touching the grid: (lo, hi) in global indices
CONTACTS = {
    "x_right": ((21, 22, 34), (24, 30, 40)),
    "x_left": ((5, 20, 30), (12, 26, 35)),
    "y_right": ((14, 29, 33), (22, 33, 38)),
    "y_left": ((12, 15, 33), (18, 22, 36)),
    "z_right": ((13, 23, 37), (16, 25, 39)),
    "z_left": ((17, 26, 28), (25, 31, 32)),
}


@pytest.mark.parametrize("name", sorted(CONTACTS))
@pytest.mark.parametrize("dual", [False, True])
def test_contacts_match_oracle(ctx, name, dual):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=dual)
    g = H.Grid.uniform((8, 6, 4))
    f = random_state(g, hp, seed=11)
    rng = np.random.default_rng(12)
    own = own_box(g, GGS, rng)
    lo, hi = CONTACTS[name]
    out = _compare(ctx, g, hp, f, own, [gbox(lo, hi, rng)], GGS, (64, 64, 64), (0, 0, 0))
    assert not np.array_equal(out["d"], f["d"])


def test_several_siblings_and_periodic_wrap(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((8, 6, 4))
    f = random_state(g, hp, seed=13)
    ggs = (10, 20, -3)  # the level's lower z boundary
    rng = np.random.default_rng(14)
    own = own_box(g, ggs, rng)
    refs = [gbox((13, 23, 28), (20, 28, 31), rng),  # across the periodic z boundary
            gbox((21, 22, 0), (24, 30, 3), rng),    # right of x
            gbox((12, 15, 1), (18, 22, 2), rng)]    # below y
    _compare(ctx, g, hp, f, own, refs, ggs, (64, 64, 32), (0, 0, 1))


@pytest.mark.parametrize("slot", [0, 1, 5])  # density, total energy, gas energy
@pytest.mark.parametrize("side", ["x_right", "y_left"])
def test_undo_matches_oracle(ctx, slot, side):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((8, 6, 4))
    f = random_state(g, hp, seed=15)
    rng = np.random.default_rng(16)
    own = own_box(g, GGS, rng)
    lo, hi = CONTACTS[side]
    ref = gbox(lo, hi, rng)
    dim = 0 if side.startswith("x") else 1
    # refined fluxes that drain the edge zones of this field well below zero
    arr = ref["left" if side.endswith("right") else "right"][slot][dim]
    arr += 50.0 * (1.0 if side.endswith("right") else -1.0)
    _compare(ctx, g, hp, f, own, [ref], GGS, (64, 64, 64), (0, 0, 0))


def test_species_colours_match_oracle(ctx):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((8, 6, 4))
    f = random_state(g, hp, seed=19)
    rng = np.random.default_rng(20)
    for n in range(3):
        f[f"col{n}"] = (0.2 + 0.3 * n) * f["d"]
    species = [1, 0, 1]
    own = own_box(g, GGS, rng)
    refs = [gbox(*CONTACTS["x_right"], rng), gbox(*CONTACTS["y_left"], rng)]
    f_ora, f_gpu = copy_fields(f), copy_fields(f)
    r_ora, r_gpu = [copy_box(r) for r in refs], [copy_box(r) for r in refs]
    assert O.correct_fluxes_sublings(g, hp, f_ora, ora_fluxes(own),
                                     [ora_fluxes(r) for r in r_ora], GGS, (64, 64, 64),
                                     (0, 0, 0), species=species) == 0
    ctx.correct_fluxes_sublings(g, hp, f_gpu, own, r_gpu, GGS, (64, 64, 64), (0, 0, 0),
                                species=species)
    for k in f:
        assert np.array_equal(f_gpu[k], f_ora[k]), k


@pytest.mark.parametrize("lo,hi", [((21, 22, 0), (24, 30, 0)), ((12, 15, 0), (18, 22, 0))])
def test_rank2_contacts_match_oracle(ctx, lo, hi):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((8, 6))  # active global x 13..20, y 23..28 at GGS
    f = random_state(g, hp, seed=21)
    rng = np.random.default_rng(22)
    ggs = (GGS[0], GGS[1], 0)
    own = own_box(g, ggs, rng, rank=2)
    out = _compare(ctx, g, hp, f, own, [gbox(lo, hi, rng, rank=2)], ggs, (64, 64, 1),
                   (0, 0, 0))
    assert not np.array_equal(out["d"], f["d"])
