"""The oracle's grid::CorrectForRefinedFluxes (proper subgrids): the zones just outside
each subgrid face change by exactly the flux difference (density, added once), the
velocities by the conserved-form update, a layer that is the grid's ghost zone gets no
correction, and a correction that would make density or an energy non-positive is
undone with the refined fluxes reset to the initial ones."""
import numpy as np

import oracle as O
from flux_fix_util import copy_box, flux_box, ora_fluxes
from parity_util import random_state
from ppm_b200 import harness as H

GGS = (40, 50, 60)


def _setup(kick, lo=(5, 4, 6), hi=(9, 10, 8), seed=3):
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((16, 14, 12))
    f = random_state(g, hp, seed=seed)
    rng = np.random.default_rng(seed)
    ini = flux_box(lo, hi, GGS, rng, True)
    ref = flux_box(lo, hi, GGS, rng, True, refined_of=ini, kick=kick)
    return hp, g, f, ini, ref


def test_density_changes_by_the_flux_difference():
    hp, g, f, ini, ref = _setup(kick=0.0)
    before = {k: v.copy() for k, v in f.items()}
    rc = O.correct_fluxes(g, hp, f, [ora_fluxes(ini)], [ora_fluxes(ref)], GGS)
    assert rc == 0
    lo, hi = (5, 4, 6), (9, 10, 8)
    expect = before["d"].copy()
    for dim in range(3):
        t = [j for j in range(3) if j != dim]
        shape = [hi[j] - lo[j] + 1 for j in reversed(t)]
        il = ini["left"][0][dim].reshape(shape)
        rl = ref["left"][0][dim].reshape(shape)
        ir = ini["right"][0][dim].reshape(shape)
        rr = ref["right"][0][dim].reshape(shape)
        sl_l = [slice(lo[j], hi[j] + 1) for j in range(3)]
        sl_r = list(sl_l)
        sl_l[dim] = lo[dim] - 1
        sl_r[dim] = hi[dim] + 1
        zl = tuple(sl_l[::-1])
        zr = tuple(sl_r[::-1])
        expect[zl] = expect[zl] + (il - rl)
        expect[zr] = expect[zr] + (-(ir - rr))
    assert np.array_equal(f["d"], expect)
    # zones away from the faces are untouched
    mask = f["d"] != before["d"]
    assert mask.sum() == sum((hi[a] - lo[a] + 1) * (hi[b] - lo[b] + 1) * 2
                             for a, b in ((1, 2), (0, 2), (0, 1)))
    # the dual-energy consistency holds in the corrected zones
    ke = 0.5 * f["v1"] * f["v1"]
    ke = ke + 0.5 * f["v2"] * f["v2"]
    ke = ke + 0.5 * f["v3"] * f["v3"]
    assert np.allclose(f["te"][mask], (f["ge"] + ke)[mask], rtol=1e-13, atol=0)


def test_ghost_layer_is_not_corrected():
    # a subgrid starting at the first active zone along x: its left x-layer is a ghost
    hp, g, f, ini, ref = _setup(kick=0.0, lo=(3, 4, 6), hi=(7, 10, 8))
    before = f["d"].copy()
    assert O.correct_fluxes(g, hp, f, [ora_fluxes(ini)], [ora_fluxes(ref)], GGS) == 0
    assert np.array_equal(f["d"][:, :, 2], before[:, :, 2])


def test_undo_keeps_states_positive_and_resets_refined_fluxes():
    hp, g, f, ini, ref = _setup(kick=50.0)
    ref_before = copy_box(ref)
    assert O.correct_fluxes(g, hp, f, [ora_fluxes(ini)], [ora_fluxes(ref)], GGS) == 0
    assert (f["d"] > 0).all() and (f["ge"] > 0).all()
    undone = 0
    for dim in range(3):
        for side in ("left", "right"):
            now, was, init = ref[side][0][dim], ref_before[side][0][dim], ini[side][0][dim]
            changed = now != was
            undone += changed.sum()
            assert np.array_equal(now[changed], init[changed])
    assert undone > 0


def test_species_keep_their_density_fraction():
    # FluxCorrection = 1: species colours are divided by the density before the
    # corrections and multiplied by the corrected density after them
    # (Grid_CorrectForRefinedFluxes.C:397-421, :849-866); other colours are untouched
    hp, g, f, ini, ref = _setup(kick=0.0, seed=5)
    rng = np.random.default_rng(6)
    f["col0"] = 0.25 * f["d"] * (1.0 + 0.1 * rng.random(f["d"].shape))
    f["col1"] = rng.random(f["d"].shape)
    before = {k: v.copy() for k, v in f.items()}
    rc = O.correct_fluxes(g, hp, f, [ora_fluxes(ini)], [ora_fluxes(ref)], GGS,
                          species=[1, 0])
    assert rc == 0
    changed = f["d"] != before["d"]
    assert changed.any()
    frac0, frac1 = before["col0"] / before["d"], f["col0"] / f["d"]
    assert np.allclose(frac1, frac0, rtol=1e-15, atol=0)
    assert not np.array_equal(f["col0"][changed], before["col0"][changed])
    assert np.array_equal(f["col0"][~changed], before["col0"][~changed])
    assert np.array_equal(f["col1"], before["col1"])
