"""Generate the shock-tube golden fixtures (tests/golden/shocktubes.json).

The reference pins its PPM-DE solver only through analytic answer tests:
run/Hydro/Hydro-1D/SodShockTube and Toro-{1..7}-ShockTube, each a 1-D run on 100
zones (outflow boundaries, CourantSafetyNumber 0.9, Gamma 1.4) compared with an
exact Riemann solution inside given x-windows at a given rtol/atol
(``*__test_*.py``).  This script writes those problem definitions together with
the exact solution computed by ``exact_riemann.py`` at the same 1000 sample
positions the reference's ``*_exact.txt`` files use.

Given the root of an enzo-dev checkout, it also checks the exact solutions
against the reference's own ``*_exact.txt`` files and records the largest
deviation per column in the fixture.

    python tests/golden/make_golden.py --reference <enzo-dev checkout>
"""
from __future__ import annotations

import argparse
import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import exact_riemann  # noqa: E402

# Problem definitions transcribed from the reference's parameter files and
# answer-test scripts (run/Hydro/Hydro-1D/<name>/<name>.enzo and *__test_*.py).
PROBLEMS = {
    "SodShockTube": dict(x0=0.5, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), t=0.25,
                         fields=["density", "specific_thermal_energy"],
                         les=[0.25, 0.85], res=[0.4, 0.9], rtol=1e-2, atol=1e-7,
                         exact="SodShockTube/SodShockTube_t=0.25_exact.txt"),
    "Toro-1-ShockTube": dict(x0=0.3, left=(1.0, 0.75, 1.0), right=(0.125, 0.0, 0.1), t=0.20,
                             fields=["density", "velocity_x", "pressure", "specific_thermal_energy"],
                             les=[0.0, 0.65], res=[0.25, 0.7], rtol=5e-2, atol=1e-7,
                             exact="Toro-1-ShockTube/Toro-1-ShockTube_t=0.2_exact.txt"),
    "Toro-2-ShockTube": dict(x0=0.5, left=(1.0, -2.0, 0.4), right=(1.0, 2.0, 0.4), t=0.15,
                             fields=["density", "pressure"],
                             les=[0.2, 0.7], res=[0.3, 0.8], rtol=1e-1, atol=1e-7,
                             exact="Toro-2-ShockTube/Toro-2-ShockTube_t=0.15_exact.txt"),
    "Toro-3-ShockTube": dict(x0=0.5, left=(1.0, 0.0, 1000.0), right=(1.0, 0.0, 0.01), t=0.012,
                             fields=["density", "velocity_x", "pressure", "specific_thermal_energy"],
                             les=[0.1, 0.6], res=[0.25, 0.7], rtol=1e-1, atol=1e-7,
                             exact="Toro-3-ShockTube/Toro-3-ShockTube_t=0.012_exact.txt"),
    "Toro-4-ShockTube": dict(x0=0.4, left=(5.99924, 19.5975, 460.894),
                             right=(5.99242, -6.19633, 46.0950), t=0.035,
                             fields=["density", "velocity_x", "pressure", "specific_thermal_energy"],
                             les=[0.5, 0.78], res=[0.6, 0.8], rtol=1e-1, atol=1e-7,
                             exact="Toro-4-ShockTube/Toro-4-ShockTube_t=0.035_exact.txt"),
    "Toro-5-ShockTube": dict(x0=0.8, left=(1.0, -19.59745, 1000.0),
                             right=(1.0, -19.59745, 0.01), t=0.012,
                             fields=["density", "pressure", "specific_thermal_energy"],
                             les=[0.25], res=[0.4], rtol=1e-2, atol=1e-7,
                             exact="Toro-5-ShockTube/Toro-5-ShockTube_t=0.012_exact.txt"),
    "Toro-6-ShockTube": dict(x0=0.5, left=(1.4, 0.0, 1.0), right=(1.0, 0.0, 1.0), t=2.0,
                             fields=["density", "velocity_x", "pressure", "specific_thermal_energy"],
                             les=[0.0], res=[1.0], rtol=1e-6, atol=1e-7,
                             exact="Toro-6-ShockTube/Toro-6-ShockTube_t=2.0_exact.txt"),
    "Toro-7-ShockTube": dict(x0=0.5, left=(1.4, 0.1, 1.0), right=(1.0, 0.1, 1.0), t=2.0,
                             fields=["density", "velocity_x", "pressure", "specific_thermal_energy"],
                             les=[0.0, 0.8], res=[0.6, 1.0], rtol=1e-3, atol=1e-7,
                             exact="Toro-7-ShockTube/Toro-7-ShockTube_t=2.0_exact.txt"),
}
GAMMA = 1.4
CFL = 0.9
NZONES = 100
COLS = ["density", "velocity_x", "pressure", "specific_thermal_energy"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="root of the enzo-dev tree holding run/Hydro/Hydro-1D")
    args = ap.parse_args()
    ref = Path(args.reference) / "run" / "Hydro" / "Hydro-1D"
    pos = (np.arange(1000) + 0.5) / 1000.0
    out = {"gamma": GAMMA, "cfl": CFL, "nzones": NZONES, "positions": pos.tolist(), "problems": {}}
    for name, pr in PROBLEMS.items():
        sol = exact_riemann.sample(pos, pr["t"], pr["x0"], pr["left"], pr["right"], GAMMA)
        entry = {k: v for k, v in pr.items() if k != "exact"}
        entry["exact"] = {c: sol[i].tolist() for i, c in enumerate(COLS)}
        f = ref / pr["exact"]
        if f.exists():
            data = np.loadtxt(f)
            assert data.shape[0] == 1000, (name, data.shape)
            assert np.allclose(data[:, 0], pos, atol=1e-6)
            dev = {}
            for i, c in enumerate(COLS):
                a = data[:, i + 1]
                b = sol[i]
                # the reference prints 6 decimals; compare away from jumps
                rel = np.abs(a - b) / np.maximum(np.abs(a), 1e-3)
                dev[c] = float(np.median(rel))
            entry["reference_check"] = dev
            print(f"{name}: median rel deviation vs reference exact file {dev}")
        out["problems"][name] = entry
    (HERE / "shocktubes.json").write_text(json.dumps(out))
    print("wrote", HERE / "shocktubes.json")


if __name__ == "__main__":
    main()
