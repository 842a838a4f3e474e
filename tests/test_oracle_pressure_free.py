"""The oracle's PressureFree path (inteuler.F:199 and :556-561, twoshock.F:124-130,
calc_dt.F:78-137): pressureless advection.  Pinned by what it implies: a density profile
carried by a uniform velocity keeps that velocity to round-off and travels at it (the
PPM-advected profile within the scheme's error of the translated one), while the same
state with pressure develops flow; the time step uses a tiny sound speed."""
import dataclasses

import numpy as np

import oracle as O
from ppm_b200 import harness as H


def _advect(pressure_free, n=64, u0=0.5, steps=None):
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=True, pressure_free=pressure_free)
    g = H.Grid.uniform((n,))
    f = H.new_fields(g, True)
    x = g.centers(0)
    rho = 1.0 + 0.5 * np.sin(2 * np.pi * x)
    f["d"][...] = rho[None, None, :]
    f["v1"][...] = u0
    f["ge"][...] = 1.0 / (hp.gamma - 1.0)  # p = rho: a pressure gradient gas dynamics feels
    f["te"][...] = f["ge"] + 0.5 * u0 * u0
    H.fill_ghosts(g, f, "periodic")
    t, cyc = 0.0, 0
    t_end = 0.5  # a quarter of the box at u0 = 0.5
    while t < t_end - 1e-14:
        p = O.compute_pressure(g, hp, f)
        dt = min(hp.cfl * O.calc_dt(g, hp, f, p, g.cellwidth), t_end - t)
        rc, st = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
        assert rc == 0
        H.fill_ghosts(g, f, "periodic")
        t += dt
        cyc += 1
    return g, f, x, cyc


def test_uniform_velocity_advects_density():
    g, f, x, cyc = _advect(True)
    s, e = g.start[0], g.end[0] + 1
    assert np.abs(f["v1"][0, 0, s:e] - 0.5).max() < 1e-13
    exact = 1.0 + 0.5 * np.sin(2 * np.pi * (x[s:e] - 0.25))
    assert np.abs(f["d"][0, 0, s:e] - exact).max() < 1e-2


def test_pressure_free_differs_from_gas_dynamics():
    _, a, _, _ = _advect(True)
    _, b, _, _ = _advect(False)
    assert np.abs(a["v1"] - b["v1"]).max() > 1e-3


def test_time_step_uses_a_tiny_sound_speed():
    hp = H.HydroParams(gamma=1.4, cfl=0.4, dual=True, pressure_free=True)
    g = H.Grid.uniform((16,))
    f = H.new_fields(g, True)
    f["d"][...] = 1.0
    f["v1"][...] = 0.25
    f["ge"][...] = 10.0
    f["te"][...] = 10.0 + 0.5 * 0.25 ** 2
    p = O.compute_pressure(g, hp, f)
    dt_free = O.calc_dt(g, hp, f, p, g.cellwidth)
    dt_gas = O.calc_dt(g, dataclasses.replace(hp, pressure_free=False), f, p, g.cellwidth)
    dx = g.cellwidth[0][3]
    assert dt_free == dx / (1e-20 + 0.25)
    assert dt_gas < dt_free
