"""grid::CorrectForRefinedFluxes on the GPU (ppm_b200_correct_fluxes) against the oracle:
bit-identical fields and refined fluxes for several subgrids of one grid -- two of them
one zone apart, so both correct the zones between them; one touching the grid's active
edge, whose layer there is a ghost zone -- with and without undone corrections, host and
device fields, ranks 2 and 3."""
import numpy as np
import pytest

import oracle as O
from flux_fix_util import copy_box, flux_box, ora_fluxes
from parity_util import compare, copy_fields, random_state
from ppm_b200 import capi
from ppm_b200 import harness as H

pytestmark = pytest.mark.gpu

GGS = (40, 50, 60)


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def _subgrids(rank):
    if rank == 3:
        return [((5, 4, 6), (8, 10, 8)), ((10, 5, 4), (13, 9, 10)), ((3, 12, 3), (6, 14, 5))]
    return [((5, 4, 0), (8, 10, 0)), ((10, 5, 0), (13, 9, 0)), ((3, 12, 0), (6, 14, 0))]


@pytest.mark.parametrize("rank", [2, 3])
@pytest.mark.parametrize("kick", [0.0, 50.0])
@pytest.mark.parametrize("memory", [capi.MEM_HOST, capi.MEM_DEVICE])
def test_correction_matches_oracle(ctx, rank, kick, memory):
    import torch
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((16, 15, 12)[:rank])
    f = random_state(g, hp, seed=7)
    rng = np.random.default_rng(11)
    ini, ref = [], []
    for lo, hi in _subgrids(rank):
        a = flux_box(lo, hi, GGS, rng, True, rank=rank)
        ini.append(a)
        ref.append(flux_box(lo, hi, GGS, rng, True, rank=rank, refined_of=a, kick=kick))
    ref_gpu = [copy_box(b) for b in ref]
    f_ora = copy_fields(f)
    assert O.correct_fluxes(g, hp, f_ora, [ora_fluxes(b) for b in ini],
                            [ora_fluxes(b) for b in ref], GGS) == 0
    if memory == capi.MEM_DEVICE:
        dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()}
        ctx.correct_fluxes(g, hp, dev, ini, ref_gpu, GGS, memory=memory)
        got = {k: v.cpu().numpy() for k, v in dev.items()}
    else:
        got = copy_fields(f)
        ctx.correct_fluxes(g, hp, got, ini, ref_gpu, GGS, memory=memory)
    for k, r in compare(got, f_ora, g).items():
        assert r["bitexact"], (k, r)
    for k in got:  # ghost zones too
        assert np.array_equal(got[k], f_ora[k]), k
    for n in range(len(ref)):
        for side in ("left", "right"):
            for s_ in range(6):
                for d in range(rank):
                    a, b = ref_gpu[n][side][s_][d], ref[n][side][s_][d]
                    if b is not None:
                        assert np.array_equal(a, b), (n, side, s_, d)
    assert any(not np.array_equal(got[k], f[k]) for k in got)


@pytest.mark.parametrize("memory", [capi.MEM_HOST, capi.MEM_DEVICE])
def test_species_colours_match_oracle(ctx, memory):
    # colours flagged as species keep their density fraction (FluxCorrection = 1); the
    # others are left alone
    import torch
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((16, 15, 12))
    f = random_state(g, hp, seed=17)
    rng = np.random.default_rng(18)
    for n in range(5):
        f[f"col{n}"] = (0.1 + 0.2 * n) * f["d"] * (1.0 + 0.1 * rng.random(f["d"].shape))
    species = [1, 0, 1, 1, 0]
    ini, ref = [], []
    for lo, hi in _subgrids(3):
        a = flux_box(lo, hi, GGS, rng, True)
        ini.append(a)
        ref.append(flux_box(lo, hi, GGS, rng, True, refined_of=a, kick=50.0))
    ref_gpu = [copy_box(b) for b in ref]
    f_ora = copy_fields(f)
    assert O.correct_fluxes(g, hp, f_ora, [ora_fluxes(b) for b in ini],
                            [ora_fluxes(b) for b in ref], GGS, species=species) == 0
    if memory == capi.MEM_DEVICE:
        dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in f.items()}
        ctx.correct_fluxes(g, hp, dev, ini, ref_gpu, GGS, memory=memory, species=species)
        got = {k: v.cpu().numpy() for k, v in dev.items()}
    else:
        got = copy_fields(f)
        ctx.correct_fluxes(g, hp, got, ini, ref_gpu, GGS, species=species)
    for k in f:
        assert np.array_equal(got[k], f_ora[k]), k
    for a, b in zip(ref_gpu, ref):
        for side in ("left", "right"):
            for s in range(6):
                for d in range(3):
                    if a[side][s][d] is not None:
                        assert np.array_equal(a[side][s][d], b[side][s][d])
