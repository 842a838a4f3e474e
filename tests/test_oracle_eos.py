"""The oracle's isothermal equation of state (EOSType 3, hydro_rk/EOS.h; used by
Grid_ComputePressure.C:112-124 at the start and, to make the energies consistent, the end
of grid::SolvePPM_DE, Grid_SolvePPM_DE.C:155-157): the pressure is rho * EOSSoundSpeed^2
and the total energy is reset to p/((gamma-1) rho) + v^2/2 wherever the pressure is
computed, so after a solve every cell's total energy is that expression exactly."""
import numpy as np

import oracle as O
from parity_util import random_state
from ppm_b200 import harness as H


def _hp(dual):
    return H.HydroParams(gamma=5.0 / 3.0, cfl=0.3, dual=dual, eos_type=3, eos_sound_speed=0.7)


def _eos_energy(hp, f, g):
    ke = 0.5 * (f["v1"] * f["v1"] + f["v2"] * f["v2"] + f["v3"] * f["v3"])
    p = f["d"] * hp.eos_sound_speed * hp.eos_sound_speed
    return p / ((hp.gamma - 1.0) * f["d"]) + ke


def test_pressure_is_isothermal_and_resets_energy():
    hp = _hp(True)
    g = H.Grid.uniform((10, 8, 6))
    f = random_state(g, hp, seed=3)
    p = O.compute_pressure(g, hp, f)
    assert np.array_equal(p, f["d"] * 0.7 * 0.7)
    assert np.array_equal(f["te"], _eos_energy(hp, f, g))


def test_energies_consistent_after_each_solve():
    for dual in (False, True):
        hp = _hp(dual)
        g = H.Grid.uniform((14, 12, 10))
        f = random_state(g, hp, seed=4, mach=1.0)
        for cyc in range(3):
            p = O.compute_pressure(g, hp, f)
            dt = hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)
            rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
            assert rc == 0
            assert np.array_equal(f["te"], _eos_energy(hp, f, g))
            H.fill_ghosts(g, f, "periodic")


def test_uniform_flow_stays_uniform():
    hp = _hp(True)
    g = H.Grid.uniform((12, 10, 8))
    f = H.new_fields(g, True)
    f["d"][...] = 1.3
    f["v1"][...] = 0.2
    f["ge"][...] = 0.5
    f["te"][...] = 0.5 + 0.5 * 0.2 * 0.2
    p = O.compute_pressure(g, hp, f)
    rc, _ = O.solve_ppm_de(g, hp, hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth), 0, f,
                           g.cellwidth)
    assert rc == 0
    act = g.active_slices()
    assert np.allclose(f["d"][act], 1.3, rtol=1e-14) and np.allclose(f["v1"][act], 0.2, rtol=1e-13)
