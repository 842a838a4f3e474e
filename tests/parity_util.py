"""Helpers shared by the GPU parity tests."""
import numpy as np

from ppm_b200 import harness as H

FIELDS = ("d", "te", "v1", "v2", "v3", "ge")


def copy_fields(f):
    return {k: v.copy() for k, v in f.items()}


def max_rel(a, b):
    """max |a-b| / max(|b|) over the field (field-normalised relative error)."""
    scale = float(np.max(np.abs(b)))
    if scale == 0.0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b))) / scale


def compare(fa, fb, grid):
    out = {}
    for k in fb:
        if k in ("v2",) and grid.rank < 2:
            continue
        if k in ("v3",) and grid.rank < 3:
            continue
        a, b = fa[k], fb[k]
        out[k] = {
            "bitexact": bool(np.array_equal(a, b)),
            "ndiff": int(np.count_nonzero(a != b)),
            "maxrel": max_rel(a, b),
        }
    return out


def random_state(grid, hp, seed=0, mach=1.5, contrast=0.5):
    """Smooth-plus-noise random state with periodic ghosts (for small parity grids)."""
    rng = np.random.default_rng(seed)
    f = H.new_fields(grid, hp.dual)
    shp = grid.shape
    act = grid.active_slices()
    def field(amp):
        a = rng.standard_normal(shp)
        # a little smoothing so the PPM limiters see both smooth and steep regions
        for ax in range(3):
            if shp[ax] > 1:
                a = 0.5 * a + 0.25 * (np.roll(a, 1, ax) + np.roll(a, -1, ax))
        return amp * a
    f["d"][...] = np.exp(contrast * field(1.0))
    p = np.exp(0.3 * field(1.0)) / hp.gamma
    names = ("v1", "v2", "v3")
    ke = np.zeros(shp)
    for dd in range(grid.rank):
        f[names[dd]][...] = field(mach)
        ke += f[names[dd]] ** 2
    eint = p / ((hp.gamma - 1.0) * f["d"])
    f["te"][...] = eint + 0.5 * ke
    if hp.dual:
        f["ge"][...] = eint
    H.fill_ghosts(grid, f, "periodic")
    return f
