"""The fifth benchmark configuration's structure -- a Zel'dovich pancake on a three-level
nested static hierarchy (refinement 2, each subgrid the middle half of its parent,
centred on the caustic), comoving expansion, dual energy, self-gravity -- advanced by the
library and by the oracle through the same W cycle (ppm_b200.hierarchy: ghost zones from
the parent, SolvePPM_DE with subgrid-flux capture, expansion terms, flux correction,
projection).  With the exact build both sides are bit-identical on every level, from
z = 100 to the caustic's redshift z = 1 on a 32^3 root and for the first root steps on
a 64^3 root; the root keeps its mass to round-off and the caustic forms."""
import os

import pytest

from hierarchy_util import OracleBackend, root_mass
from parity_util import compare
from ppm_b200 import capi
from ppm_b200 import harness as H
from ppm_b200 import hierarchy as N

pytestmark = pytest.mark.gpu

NTHREADS = os.cpu_count() or 1


def _pair(n, z_init=100.0):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, gravity=True)
    ctx = capi.Context(0)
    a = N.NestedRun(N.nested_pancake(n, 3, hp, z_init=z_init), hp, N.LibraryBackend(ctx, hp),
                    N.EdS(z_init))
    b = N.NestedRun(N.nested_pancake(n, 3, hp, z_init=z_init), hp,
                    OracleBackend(hp, NTHREADS), N.EdS(z_init))
    return hp, ctx, a, b


def _assert_same(a, b, what):
    for la, lb in zip(a.levels, b.levels):
        assert la.t == lb.t, (what, la.index)
        for k, r in compare(la.fields, lb.fields, la.grid).items():
            assert r["bitexact"], (what, la.index, k, r)


def test_nested_pancake_to_the_caustic_matches_oracle():
    hp, ctx, gpu, ora = _pair(32)
    m0 = root_mass(gpu.levels)
    d0 = gpu.levels[2].fields["d"].max()
    t_final = gpu.cosmo.time_of(1.0)
    while gpu.levels[0].t < t_final * (1.0 - 1e-14):
        gpu.step(t_final)
        ora.step(t_final)
        if gpu.root_steps % 25 == 0:
            _assert_same(gpu, ora, gpu.root_steps)
    _assert_same(gpu, ora, "z = 1")
    assert gpu.level_steps == ora.level_steps
    assert abs(gpu.cosmo.redshift(gpu.levels[0].t) - 1.0) < 1e-9
    assert abs(root_mass(gpu.levels) - m0) <= 1e-12 * m0
    # the caustic: the finest level's density peak has grown many times over
    assert gpu.levels[2].fields["d"].max() > 5.0 * d0
    ctx.close()


def test_nested_pancake_64cubed_root_first_steps_match_oracle():
    hp, ctx, gpu, ora = _pair(64)
    for _ in range(12):
        gpu.step()
        ora.step()
    _assert_same(gpu, ora, "64^3, 12 root steps")
    # every level reaches the root's time; a finer level takes at least its parent's steps
    assert gpu.level_steps[2] >= gpu.level_steps[1] >= gpu.level_steps[0] == 12
    ctx.close()
