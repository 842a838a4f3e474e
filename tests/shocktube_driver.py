"""Runs the reference's 1-D shock-tube answer problems through a solver backend.

Mirrors Enzo's level-0 cycle for these problems: ghost fill (outflow), CFL
timestep (calc_dt x CourantSafetyNumber, last step clipped to StopTime), one
SolvePPM_DE call per cycle with CycleNumber = cycle count.
"""
import json
from pathlib import Path

import numpy as np

from ppm_b200 import harness as H

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "shocktubes.json").read_text())


def run_problem(name, step_fn, dt_fn, dual=False):
    pr = GOLDEN["problems"][name]
    hp = H.HydroParams(gamma=GOLDEN["gamma"], cfl=GOLDEN["cfl"], dual=dual)
    g = H.Grid.uniform((GOLDEN["nzones"],))
    f = H.shock_tube(g, hp, pr["x0"], pr["left"], pr["right"])
    H.fill_ghosts(g, f, "outflow")
    t, cyc = 0.0, 0
    while t < pr["t"] - 1e-14:
        dt = min(hp.cfl * dt_fn(g, hp, f), pr["t"] - t)
        step_fn(g, hp, dt, cyc, f)
        H.fill_ghosts(g, f, "outflow")
        t += dt
        cyc += 1
    return g, hp, f, cyc


def check_against_exact(name, g, hp, f):
    """The reference's ShockTubeTest: fields inside x-windows vs np.interp of the exact
    solution, assert_allclose(rtol, atol). Returns list of (field, window, max_excess)."""
    pr = GOLDEN["problems"][name]
    pos = np.array(GOLDEN["positions"])
    s, e = g.start[0], g.end[0] + 1
    x = g.centers(0)[s:e]
    d = f["d"][0, 0, s:e]
    u = f["v1"][0, 0, s:e]
    ei = f["te"][0, 0, s:e] - 0.5 * u * u
    vals = {"density": d, "velocity_x": u, "pressure": (hp.gamma - 1.0) * d * ei,
            "specific_thermal_energy": ei}
    bad = []
    for fld in pr["fields"]:
        for le, re in zip(pr["les"], pr["res"]):
            m = (x >= le) & (x <= re)
            ex = np.interp(x[m], pos, pr["exact"][fld])
            excess = np.abs(vals[fld][m] - ex) - (pr["atol"] + pr["rtol"] * np.abs(ex))
            if np.any(excess > 0):
                bad.append((fld, (le, re), float(excess.max())))
    return bad
