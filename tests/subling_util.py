"""Flux boxes for the SUBling flux-correction tests, in global (level) zone indices: a
grid's own boundary fluxes and the projected refined fluxes of a sibling's subgrid
(struct fluxes, Fluxes.h:29-37; GetProjectedBoundaryFluxes fills the latter)."""


def gbox(glo, ghi, rng, rank=3, scale=0.05):
    """Flux box of the region glo..ghi (inclusive, global indices) with seeded values in
    the six hydro slots."""
    b = {"left_start": [[0] * 3 for _ in range(3)], "left_end": [[0] * 3 for _ in range(3)],
         "right_start": [[0] * 3 for _ in range(3)], "right_end": [[0] * 3 for _ in range(3)],
         "left": [[None] * 3 for _ in range(6)], "right": [[None] * 3 for _ in range(6)]}
    for dim in range(rank):
        for j in range(3):
            b["left_start"][dim][j] = glo[j]
            b["left_end"][dim][j] = glo[j] if j == dim else ghi[j]
            b["right_start"][dim][j] = ghi[j] if j == dim else glo[j]
            b["right_end"][dim][j] = ghi[j]
        size = 1
        for j in range(3):
            if j != dim:
                size *= ghi[j] - glo[j] + 1
        for s in range(6):
            for side in ("left", "right"):
                b[side][s][dim] = scale * rng.standard_normal(size)
    return b


def copy_box(b):
    out = {k: [list(r) for r in b[k]] for k in ("left_start", "left_end", "right_start",
                                                "right_end")}
    for side in ("left", "right"):
        out[side] = [[(a.copy() if a is not None else None) for a in row] for row in b[side]]
    return out


def own_box(g, ggs, rng, rank=3):
    """The grid's own boundary fluxes: its active region in global indices."""
    lo = [g.start[d] + ggs[d] for d in range(3)]
    hi = [g.end[d] + ggs[d] for d in range(3)]
    return gbox(lo, hi, rng, rank)
