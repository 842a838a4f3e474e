"""The oracle as a backend of the nested-hierarchy driver (ppm_b200.hierarchy): the same
harness steps, with the CPU restatement doing the hydro work of each grid."""
import numpy as np

import oracle as O
from flux_fix_util import ora_fluxes
from ppm_b200 import harness as H
from ppm_b200.hierarchy import LibraryBackend


class OracleBackend(LibraryBackend):
    def __init__(self, hp, nthreads=1):
        super().__init__(None, hp)
        self.nthreads = nthreads

    def timestep(self, lev, aye):
        p = O.compute_pressure(lev.grid, self.hp, lev.fields)
        return O.calc_dt(lev.grid, self.hp, lev.fields, p, lev.grid.cellwidth, aye=aye)

    def solve(self, lev, grid, dt, cycle, accel, boxes):
        subs = [ora_fluxes(b) for b in boxes] if boxes else None
        rc, _ = O.solve_ppm_de(grid, self.hp, dt, cycle, lev.fields, grid.cellwidth,
                               accel=accel, subgrids=subs, ggs=lev.ggs, nthreads=self.nthreads)
        assert rc == 0, ("oracle solve", lev.index, cycle)

    def expansion_terms(self, lev, old, time, old_time, coef):
        O.expansion_terms(lev.grid, self.hp, lev.fields, old, time, old_time, coef)

    def correct_fluxes(self, lev, initial, refined):
        rc = O.correct_fluxes(lev.grid, self.hp, lev.fields, [ora_fluxes(b) for b in initial],
                              [ora_fluxes(b) for b in refined], lev.ggs)
        assert rc == 0, ("oracle flux correction", lev.index)


def root_mass(levels):
    root = levels[0]
    act = root.grid.active_slices()
    return float(np.sum(root.fields["d"][act]))
