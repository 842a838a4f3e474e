"""The Zel'dovich-pancake state of the harness (the published one-dimensional solution,
as Grid_ZeldovichPancakeInitializeGrid.C:132-189 sets it up) and the oracle's comoving
cycles on it: the Eulerian positions solve x - A sin(kx)/k = x_L, density and velocity
follow them, and the flow falls towards the caustic (its central density grows)."""
import numpy as np

import oracle as O
from ppm_b200 import harness as H


def test_pancake_state_follows_the_zeldovich_solution():
    hp = H.HydroParams(gamma=5.0 / 3.0, dual=True)
    g = H.Grid.uniform((64,))
    f = H.zeldovich_pancake(g, hp)
    act = g.active_slices()
    rho, u = f["d"][act][0, 0], f["v1"][act][0, 0]
    n, amp = 64, 2.0 / 101.0
    # invert the density for cos(kx) and check the velocity's sin(kx) against it
    cos_kx = (1.0 - 1.0 / rho) / amp
    amp_v = np.sqrt(2.0 / 3.0) * 2.0 / (101.0 * 2.0 * np.pi)
    assert np.allclose(cos_kx ** 2 + (u / amp_v) ** 2, 1.0, atol=1e-10)
    assert np.allclose(rho, rho[::-1], rtol=1e-13) and np.allclose(u, -u[::-1], atol=1e-16)
    # the zones nearest the caustic are the densest, by less than 1/(1 - A)
    assert rho.argmax() in (n // 2 - 1, n // 2) and rho.max() < 1.0 / (1.0 - amp)


def test_comoving_cycles_collapse_towards_the_caustic():
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g = H.Grid.uniform((48,))
    f = H.zeldovich_pancake(g, hp)
    d0 = f["d"].copy()
    t = 1.0
    for cyc in range(20):
        p = O.compute_pressure(g, hp, f)
        dt = hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth)
        O.expansion_terms(g, hp, f, None, t + dt, t, 0.004)  # dt * adot / a
        rc, _ = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
        assert rc == 0
        H.fill_ghosts(g, f, "periodic")
        t += dt
    act = g.active_slices()
    assert f["d"][act].max() > d0[act].max()
