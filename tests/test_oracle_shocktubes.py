"""Pins the CPU oracle to the reference's own answer tests.

run/Hydro/Hydro-1D/{SodShockTube,Toro-1..7-ShockTube}/*__test_*.py compare a
100-zone PPM-DE run with the exact Riemann solution inside x-windows at the
listed rtol/atol. The oracle must pass every one of them, with and without the
dual-energy formalism.
"""
import pytest

import oracle as O
from shocktube_driver import GOLDEN, check_against_exact, run_problem


def _step(g, hp, dt, cyc, f):
    rc, st = O.solve_ppm_de(g, hp, dt, cyc, f, g.cellwidth)
    assert rc == 0, st


def _dt(g, hp, f):
    p = O.compute_pressure(g, hp, f)
    return O.calc_dt(g, hp, f, p, g.cellwidth)


@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("name", sorted(GOLDEN["problems"]))
def test_oracle_matches_reference_answer_test(name, dual):
    g, hp, f, cycles = run_problem(name, _step, _dt, dual=dual)
    assert cycles > 10
    assert check_against_exact(name, g, hp, f) == []


def test_exact_solver_matches_reference_files():
    # recorded by make_golden.py when the reference tree was present
    for name, pr in GOLDEN["problems"].items():
        dev = pr.get("reference_check")
        assert dev is not None, name
        for col, v in dev.items():
            assert v < 2e-3, (name, col, v)
