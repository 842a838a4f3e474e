"""The oracle's SUBling flux correction (grid::CorrectForRefinedFluxes with
SUBlingGrid == TRUE, Grid_CorrectForRefinedFluxes.C:147-305, :455-656): the grid's edge
layer that touches a sibling subgrid's projected face gets the difference between its own
boundary flux and the subgrid's refined flux on that face.  Pinned by the conservation
statement the reference encodes, computed here independently of the oracle's index
arithmetic: the corrected density of each edge zone is its old density plus
(own right flux - refined left flux) on a right contact, minus (own left flux - refined
right flux) on a left contact; zones outside the contact are untouched; a contact across
a periodic level boundary wraps."""
import numpy as np
import pytest

import oracle as O
from flux_fix_util import ora_fluxes
from parity_util import copy_fields, random_state
from ppm_b200 import harness as H
from subling_util import gbox, own_box

GGS = (10, 20, 30)


def _grid(hp, seed):
    g = H.Grid.uniform((8, 6, 4))  # active global x 13..20, y 23..28, z 33..36 at GGS
    f = random_state(g, hp, seed=seed)
    return g, f


def _run(g, hp, f, own, ref, ggs, level, periodic):
    out = copy_fields(f)
    of = ora_fluxes(own)
    rf = [ora_fluxes(r) for r in ref]
    rc = O.correct_fluxes_sublings(g, hp, out, of, rf, ggs, level, periodic)
    assert rc == 0
    return out


def test_right_contact_along_x():
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g, f = _grid(hp, 1)
    rng = np.random.default_rng(2)
    own = own_box(g, GGS, rng)
    ref = gbox((21, 22, 34), (24, 30, 40), rng)  # the sibling's subgrid, right of x = 20
    out = _run(g, hp, f, own, [ref], GGS, (64, 64, 64), (0, 0, 0))
    ie = g.end[0]
    changed = np.zeros(g.shape, bool)
    for kg in range(34, 37):
        for jg in range(23, 29):
            k, j = kg - GGS[2], jg - GGS[1]
            x = (kg - 33) * 6 + (jg - 23)
            xr = (kg - 34) * 9 + (jg - 22)
            amount = own["right"][0][0][x] - ref["left"][0][0][xr]
            assert out["d"][k, j, ie] == f["d"][k, j, ie] + amount
            changed[k, j, ie] = True
    assert np.array_equal(out["d"][~changed], f["d"][~changed])
    # momentum, in conserved form: (u*d)_new = u_old*d_old + (own - refined)
    for kg, jg in ((34, 23), (36, 28)):
        k, j = kg - GGS[2], jg - GGS[1]
        x, xr = (kg - 33) * 6 + (jg - 23), (kg - 34) * 9 + (jg - 22)
        mom = f["v1"][k, j, ie] * f["d"][k, j, ie] + (own["right"][2][0][x] - ref["left"][2][0][xr])
        assert out["v1"][k, j, ie] == pytest.approx(mom / out["d"][k, j, ie], rel=1e-14)


def test_left_contact_along_y():
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g, f = _grid(hp, 3)
    rng = np.random.default_rng(4)
    own = own_box(g, GGS, rng)
    ref = gbox((12, 15, 33), (18, 22, 36), rng)  # below y = 23
    out = _run(g, hp, f, own, [ref], GGS, (64, 64, 64), (0, 0, 0))
    js = g.start[1]
    changed = np.zeros(g.shape, bool)
    for kg in range(33, 37):
        for ig in range(13, 19):
            k, i = kg - GGS[2], ig - GGS[0]
            x = (kg - 33) * 8 + (ig - 13)
            xr = (kg - 33) * 7 + (ig - 12)
            amount = -(own["left"][0][1][x] - ref["right"][0][1][xr])
            assert out["d"][k, js, i] == f["d"][k, js, i] + amount
            changed[k, js, i] = True
    assert np.array_equal(out["d"][~changed], f["d"][~changed])


def test_periodic_contact_wraps():
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g, f = _grid(hp, 5)
    ggs = (10, 20, -3)  # active z 0..3: the level's lower z boundary
    rng = np.random.default_rng(6)
    own = own_box(g, ggs, rng)
    ref = gbox((13, 23, 28), (20, 28, 31), rng)  # at the upper z boundary of a 32-zone level
    out = _run(g, hp, f, own, [ref], ggs, (64, 64, 32), (0, 0, 1))
    ks = g.start[2]
    for jg in (23, 26, 28):
        for ig in (13, 17, 20):
            j, i = jg - ggs[1], ig - ggs[0]
            x = (jg - 23) * 8 + (ig - 13)
            amount = -(own["left"][0][2][x] - ref["right"][0][2][x])
            assert out["d"][ks, j, i] == f["d"][ks, j, i] + amount
    # without periodicity the sibling does not touch the grid
    out2 = _run(g, hp, f, own, [ref], ggs, (64, 64, 32), (0, 0, 0))
    for k in f:
        assert np.array_equal(out2[k], f[k])


def test_non_touching_sibling_changes_nothing():
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g, f = _grid(hp, 7)
    rng = np.random.default_rng(8)
    own = own_box(g, GGS, rng)
    ref = gbox((22, 22, 34), (24, 30, 40), rng)  # one zone away from x = 20
    out = _run(g, hp, f, own, [ref], GGS, (64, 64, 64), (0, 0, 0))
    for k in f:
        assert np.array_equal(out[k], f[k])
