"""The nested-hierarchy driver (ppm_b200.hierarchy) on the CPU with the oracle doing the
hydro work: a three-level Zel'dovich pancake keeps the root's mass to round-off through
the W cycle (flux correction at the subgrid boundaries and projection of the subgrids),
its levels reach the same time, and the flow falls towards the caustic."""
import math

import numpy as np

from hierarchy_util import OracleBackend, root_mass
from ppm_b200 import harness as H
from ppm_b200 import hierarchy as N


def _run(n=8, levels=3, steps=4):
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.5, dual=True, gravity=True)
    lv = N.nested_pancake(n, levels, hp, z_init=20.0, z_collapse=1.0)
    run = N.NestedRun(lv, hp, OracleBackend(hp), N.EdS(20.0))
    return lv, run


def test_nested_pancake_conserves_root_mass_and_subcycles():
    lv, run = _run()
    m0 = root_mass(lv)
    d0 = lv[2].fields["d"].max()
    for _ in range(4):
        run.step()
        m = root_mass(lv)
        assert abs(m - m0) <= 1e-13 * m0, (m, m0)
        assert lv[1].t == lv[0].t and lv[2].t == lv[0].t
    # finer levels take at least as many steps as their parents
    assert run.level_steps[2] >= run.level_steps[1] >= run.level_steps[0] == 4
    assert lv[2].fields["d"].max() > d0


def test_projection_and_flux_projection_factors():
    # a child state that is uniform projects to the same uniform values; projected fluxes
    # of a uniform flux are the flux itself (2x2 faces and two half steps per coarse face
    # and step, over the total refinement 8)
    hp = H.HydroParams(dual=True)
    lv = N.nested_pancake(8, 2, hp)
    for k, v in lv[1].fields.items():
        v[...] = {"d": 2.0, "te": 3.0, "v1": 0.5, "v2": -0.25, "v3": 0.0, "ge": 1.5}[k]
    N.project_solution(lv[0], lv[1], np)
    lo, hi = N.child_box(lv[0], lv[1])
    sl = (slice(lo, hi + 1),) * 3
    for k in lv[0].fields:
        assert np.all(lv[0].fields[k][sl] == lv[1].fields[k][3, 3, 3]), k
    box = N.flux_box_dict(3, 10, lv[1].ggs, np.zeros, True)
    for side in ("left", "right"):
        for slot in range(6):
            for d in range(3):
                box[side][slot][d] += 2.0 * 0.5  # two fine steps of 0.5 (dt/dx_fine units)
    proj = N.project_fluxes(box, 8, True, np)
    assert np.allclose(proj["left"][0][0], 0.5 * 4 * 2.0 * 0.5 / 4)
    assert proj["left_start"][0][0] == box["left_start"][0][0] // 2
