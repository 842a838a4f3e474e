"""Exact solution of the 1-D Riemann problem for an ideal gas.

Follows the published algorithm of E. F. Toro, "Riemann Solvers and Numerical
Methods for Fluid Dynamics", 2nd ed., ch. 4 (pressure function, Newton
iteration for p*, sampling of the self-similar solution).  Used to produce the
shock-tube golden fixtures that the reference's answer tests compare against
(run/Hydro/Hydro-1D/*/..._exact.txt were made with the same method).
"""
from __future__ import annotations

import math

import numpy as np


def _fk(p, rho, pk, ck, g):
    if p > pk:  # shock
        a = 2.0 / ((g + 1.0) * rho)
        b = (g - 1.0) / (g + 1.0) * pk
        q = math.sqrt(a / (p + b))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (b + p))
    pr = p / pk  # rarefaction
    f = 2.0 * ck / (g - 1.0) * (pr ** ((g - 1.0) / (2.0 * g)) - 1.0)
    df = 1.0 / (rho * ck) * pr ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(dl, ul, pl, dr, ur, pr, g):
    cl = math.sqrt(g * pl / dl)
    cr = math.sqrt(g * pr / dr)
    du = ur - ul
    # two-rarefaction guess, bounded below
    p = ((cl + cr - 0.5 * (g - 1.0) * du) /
         (cl / pl ** ((g - 1.0) / (2.0 * g)) + cr / pr ** ((g - 1.0) / (2.0 * g)))) ** (
        2.0 * g / (g - 1.0))
    p = max(p, 1e-12)
    for _ in range(200):
        fl, dfl = _fk(p, dl, pl, cl, g)
        fr, dfr = _fk(p, dr, pr, cr, g)
        pn = p - (fl + fr + du) / (dfl + dfr)
        if pn < 0:
            pn = 1e-12
        if abs(pn - p) / (0.5 * (pn + p)) < 1e-14:
            p = pn
            break
        p = pn
    fl, _ = _fk(p, dl, pl, cl, g)
    fr, _ = _fk(p, dr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(x, t, x0, left, right, g):
    """Return (rho, u, p, e_int) at positions x (array) and time t > 0.

    left/right: (rho, u, p)."""
    dl, ul, pl = left
    dr, ur, pr = right
    ps, us = star_state(dl, ul, pl, dr, ur, pr, g)
    cl = math.sqrt(g * pl / dl)
    cr = math.sqrt(g * pr / dr)
    out = np.zeros((4, len(x)))
    for n, xi in enumerate(x):
        s = (xi - x0) / t
        if s <= us:  # left of contact
            if ps > pl:  # left shock
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    d, u, p = dl, ul, pl
                else:
                    d = dl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1))
                    u, p = us, ps
            else:  # left rarefaction
                shl = ul - cl
                if s <= shl:
                    d, u, p = dl, ul, pl
                else:
                    cml = cl * (ps / pl) ** ((g - 1) / (2 * g))
                    stl = us - cml
                    if s > stl:
                        d = dl * (ps / pl) ** (1 / g)
                        u, p = us, ps
                    else:
                        u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                        c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                        d = dl * (c / cl) ** (2 / (g - 1))
                        p = pl * (c / cl) ** (2 * g / (g - 1))
        else:  # right of contact
            if ps > pr:  # right shock
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    d, u, p = dr, ur, pr
                else:
                    d = dr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1))
                    u, p = us, ps
            else:  # right rarefaction
                shr = ur + cr
                if s >= shr:
                    d, u, p = dr, ur, pr
                else:
                    cmr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                    str_ = us + cmr
                    if s <= str_:
                        d = dr * (ps / pr) ** (1 / g)
                        u, p = us, ps
                    else:
                        u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                        c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                        d = dr * (c / cr) ** (2 / (g - 1))
                        p = pr * (c / cr) ** (2 * g / (g - 1))
        out[:, n] = (d, u, p, p / ((g - 1) * d))
    return out
