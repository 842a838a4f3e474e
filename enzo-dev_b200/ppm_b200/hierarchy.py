"""A static nested hierarchy around the hydro calls, for the Zel'dovich-pancake workload.

Enzo advances a hierarchy with EvolveLevel (EvolveLevel.C): per level step it fills the
ghost zones (SetBoundaryConditions: periodic for the root, interpolated from the parent
in space and time for a subgrid, InterpolateBoundaryFromParent), copies the fields to
OldBaryonField, runs grid::SolveHydroEquations, adds the comoving expansion terms
(EvolveLevel.C:753-754), recurses into the next level until it reaches the same time,
and then updates from the finer level (UpdateFromFinerGrids.C): the subgrid's boundary
fluxes, projected to this level (Grid_GetProjectedBoundaryFluxes.C), correct the zones
around the subgrid (grid::CorrectForRefinedFluxes), and the subgrid's solution is
projected onto the zones it covers (Grid_ProjectSolutionToParentGrid.C: density
averaged, the other fields as density-weighted averages).

The hierarchy code is the reference's and stays out of this library; this module is the
host-side stand-in that the benchmark and the tests drive the library with.  Its own
choices, shared by every backend so that they see the same inputs:

- one grid per level, each subgrid covering the middle half of its parent along every
  axis (refinement factor 2, n^3 active zones on every level, centred on the caustic);
- ghost zones of a subgrid: its parent's zone value (piecewise constant, conservative),
  linear in time between the parent's old and new fields;
- gravity: the pancake's one-dimensional self-gravity from the root level's density
  profile along x, d^2 phi / dx^2 = (rho - 1)/a in comoving coordinates (units with
  4 pi G = 1, as Enzo's GravitationalConstant = 1 for cosmology), the acceleration
  -dphi/dx / a, solved spectrally at the start of every root step and interpolated
  linearly to the finer levels' zone centres;
- the sweeps see proper cell widths, a(t + dt/2) times the comoving ones, as
  grid::SolveHydroEquations passes them (CellWidthTemp = a * CellWidth), and the time
  step takes a through calc_dt's aye;
- an Einstein-de Sitter expansion a(t) = (t / t_i)^(2/3), t_i = sqrt(2/3) (a = 1 at the
  initial redshift), and Enzo's CosmologyMaxExpansionRate limit (da/a <= 0.01 a step).

A backend does the hydro work of one grid: `solve`, `expansion_terms`,
`correct_fluxes`, `timestep` and the periodic ghost fill; `LibraryBackend` runs the
library's C ABI on host fields (bit-identical to the oracle with the exact build),
`DeviceBackend` keeps the fields on the GPU (torch tensors) for timing.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import harness as H

NG = H.NGHOST


# ---------------------------------------------------------------- cosmology (EdS)
class EdS:
    """Einstein-de Sitter expansion in Enzo's comoving code units (Omega_m = 1):
    a(t) = (t / t_i)^(2/3) with a(t_i) = 1 at the initial redshift."""

    def __init__(self, z_init):
        self.z_init = float(z_init)
        self.t_init = math.sqrt(2.0 / 3.0)

    def a(self, t):
        return (t / self.t_init) ** (2.0 / 3.0)

    def adot_over_a(self, t):
        return 2.0 / (3.0 * t)

    def redshift(self, t):
        return (1.0 + self.z_init) / self.a(t) - 1.0

    def time_of(self, z):
        a = (1.0 + self.z_init) / (1.0 + z)
        return self.t_init * a ** 1.5


# ---------------------------------------------------------------- pancake state
def pancake_profile(xc, n_root, gamma, z_init, z_collapse, e_init):
    """The Zel'dovich pancake at zone centres xc (domain coordinates in [0, 1), caustic at
    0.5; the solution of harness.zeldovich_pancake in root-zone units): density,
    x velocity and specific internal energy."""
    amp = (1.0 + z_collapse) / (1.0 + z_init)
    amp_v = -np.sqrt(2.0 / 3.0) * (1.0 + z_collapse) / ((1.0 + z_init) * 2.0 * np.pi)
    k = 2.0 * np.pi / n_root
    x_e = (np.asarray(xc, dtype=np.float64) - 0.5) * n_root  # Eulerian, root zones
    q = x_e.copy()                                            # Lagrangian position
    for _ in range(100):
        step = (x_e - q + amp * np.sin(k * q) / k) / (1.0 - amp * np.cos(k * q))
        q = q + step
        if np.all(np.abs(step) <= 1e-14 * np.maximum(np.abs(q), 1.0)):
            break
    rho = 1.0 / (1.0 - amp * np.cos(k * q))
    u = amp_v * np.sin(k * q)
    e_int = e_init * rho ** (gamma - 1.0) / (gamma - 1.0)
    return rho, u, e_int


class Level:
    """One level of the nested hierarchy: a single grid of n^3 active zones."""

    def __init__(self, index, n, hp):
        self.index = index
        self.n = n
        self.dx = 1.0 / (n * 2 ** index)
        self.left = 0.0 if index == 0 else 0.5 - 0.5 / 2 ** index   # active region's edge
        self.start = n * (2 ** index - 1) // 2    # global index of the first active zone
        self.ggs = (self.start - NG,) * 3         # ... of the first zone, ghosts included
        width = 1.0 / 2 ** index
        self.grid = H.Grid.uniform((n, n, n), width=width)
        self.fields = None
        self.old = None
        self.t = 0.0
        self.t_old = 0.0
        self.cycle = 0
        self.accel = None

    def centres(self):
        """Zone centres along an axis (ghosts included), domain coordinates."""
        return self.left + (np.arange(self.n + 2 * NG) - NG + 0.5) * self.dx


def nested_pancake(n, nlevels, hp, z_init=100.0, z_collapse=1.0, e_init=1e-6):
    """The nested static hierarchy of the pancake: `nlevels` levels of n^3 zones (n a
    multiple of 4), every level from the pancake solution at its zone centres."""
    assert n % 4 == 0 and n >= 8
    levels = []
    for l in range(nlevels):
        lev = Level(l, n, hp)
        rho, u, e_int = pancake_profile(lev.centres(), n, hp.gamma, z_init, z_collapse, e_init)
        f = H.new_fields(lev.grid, hp.dual)
        f["d"][...] = rho[None, None, :]
        f["v1"][...] = u[None, None, :]
        f["te"][...] = (e_int + 0.5 * u * u)[None, None, :]
        if hp.dual:
            f["ge"][...] = e_int[None, None, :]
        lev.fields = f
        levels.append(lev)
    return levels


# ---------------------------------------------------------------- level operations
def parent_index(child, parent):
    """Parent array index of every child array index along an axis."""
    glob = child.ggs[0] + np.arange(child.n + 2 * NG)
    return glob // 2 - parent.ggs[0]


def ghost_mask(level):
    """True on the ghost shell of a level's arrays (z, y, x order)."""
    m = np.ones(level.grid.shape, dtype=bool)
    m[level.grid.active_slices()] = False
    return m


def child_box(parent, child):
    """The parent's array indices (lo, hi inclusive, per axis) of the zones the child
    covers."""
    lo = child.start // 2 - parent.ggs[0]
    hi = (child.start + child.n) // 2 - 1 - parent.ggs[0]
    return lo, hi


def flux_box_dict(lo, hi, ggs, zeros, dual):
    """A struct-fluxes box (Fluxes.h:29-37) around active zones lo..hi (array indices) of a
    grid whose first zone has global index ggs; zeros(size) makes each flux array."""
    b = {"left_start": [[0] * 3 for _ in range(3)], "left_end": [[0] * 3 for _ in range(3)],
         "right_start": [[0] * 3 for _ in range(3)], "right_end": [[0] * 3 for _ in range(3)],
         "left": [[None] * 3 for _ in range(6)], "right": [[None] * 3 for _ in range(6)]}
    for dim in range(3):
        for j in range(3):
            s, e = lo + ggs[j], hi + ggs[j]
            b["left_start"][dim][j] = s
            b["left_end"][dim][j] = s if j == dim else e
            b["right_start"][dim][j] = e if j == dim else s
            b["right_end"][dim][j] = e
        size = (hi - lo + 1) ** 2
        for slot in [0, 1, 2, 3, 4] + ([5] if dual else []):
            for side in ("left", "right"):
                b[side][slot][dim] = zeros(size)
    return b


def project_fluxes(fine, n_fine, dual, xp):
    """Grid_GetProjectedBoundaryFluxes.C for refinement factor 2 in 3-D: each coarse face
    value is the sum of the 2x2 fine faces on it (accumulated over the fine steps) over
    the total refinement 8; the index boxes divided by 2."""
    out = {k: [[v // 2 for v in row] for row in fine[k]]
           for k in ("left_start", "left_end", "right_start", "right_end")}
    m = n_fine // 2
    for side in ("left", "right"):
        out[side] = [[None] * 3 for _ in range(6)]
        for slot in range(6):
            for dim in range(3):
                a = fine[side][slot][dim]
                if a is None:
                    continue
                # transverse axes in (slowest, fastest) order of the flux array
                q = a.reshape(m, 2, m, 2).sum(axis=(1, 3)) * 0.125
                out[side][slot][dim] = q.reshape(m * m)
    return out


def project_solution(parent, child, xp):
    """Grid_ProjectSolutionToParentGrid.C for refinement factor 2: the parent zones the
    child covers take the child's average density and density-weighted averages of the
    other fields."""
    lo, hi = child_box(parent, child)
    act = child.grid.active_slices()
    m = child.n // 2
    d = child.fields["d"][act].reshape(m, 2, m, 2, m, 2)
    dsum = d.sum(axis=(1, 3, 5))
    sl = (slice(lo, hi + 1),) * 3
    for k, v in child.fields.items():
        if k == "d":
            continue
        w = (v[act].reshape(m, 2, m, 2, m, 2) * d).sum(axis=(1, 3, 5))
        parent.fields[k][sl] = w / dsum
    parent.fields["d"][sl] = dsum * 0.125


def ghost_map(parent, child):
    """Flat indices of the child's ghost zones and of the parent zone each one takes its
    value from (x fastest, as the fields are laid out)."""
    idx = parent_index(child, parent)
    m = ghost_mask(child)
    kz, jy, ix = np.nonzero(m)
    pd = parent.grid.dims
    cd = child.grid.dims
    child_flat = (kz * cd[1] + jy) * cd[0] + ix
    parent_flat = (idx[kz] * pd[1] + idx[jy]) * pd[0] + idx[ix]
    return child_flat.astype(np.int64), parent_flat.astype(np.int64)


def fill_child_ghosts(parent, child, t, be):
    """SetBoundaryConditions for a subgrid: each ghost zone takes its parent zone's value,
    linear in time between the parent's old (t_old) and new (t) fields."""
    gi, pi = child.ghosts
    span = parent.t - parent.t_old
    w = 0.0 if span <= 0.0 else (t - parent.t_old) / span
    for k, v in child.fields.items():
        new = parent.fields[k].reshape(-1)[pi]
        old = parent.old[k].reshape(-1)[pi]
        v.reshape(-1)[gi] = old + w * (new - old)


def gravity_profile(root, cosmo, t):
    """The pancake's self-gravity along x from the root's density profile (the mean over
    y and z): d^2 phi/dx^2 = (rho - 1)/a, acceleration -dphi/dx at the root's active zone
    centres (spectral, periodic)."""
    act = root.grid.active_slices()
    d = root.fields["d"][act]
    prof = d.mean(dim=(0, 1)).cpu().numpy() if hasattr(d, "cpu") else d.mean(axis=(0, 1))
    n = prof.size
    k = 2.0 * np.pi * np.fft.rfftfreq(n, d=1.0 / n)
    src = np.fft.rfft(prof - 1.0) / cosmo.a(t)
    phi = np.zeros_like(src)
    phi[1:] = -src[1:] / (k[1:] ** 2)
    acc = np.fft.irfft(-1j * k * phi, n=n) / cosmo.a(t)
    return acc


def level_accel(level, root, acc_root):
    """The root's acceleration profile, linearly interpolated (periodic) to a level's zone
    centres (ghosts included): the x acceleration along the x axis."""
    xr = (np.arange(root.n) + 0.5) / root.n
    x = level.centres()
    xe = np.concatenate([xr - 1.0, xr, xr + 1.0])
    ae = np.concatenate([acc_root, acc_root, acc_root])
    return np.interp(x, xe, ae)


# ---------------------------------------------------------------- the W cycle
class NestedRun:
    """The W cycle of EvolveLevel over a nested static hierarchy with one backend."""

    def __init__(self, levels, hp, backend, cosmo, max_expansion=0.01):
        self.levels = levels
        self.hp = hp
        self.be = backend
        self.cosmo = cosmo
        self.max_expansion = max_expansion
        t0 = cosmo.t_init
        for l, lev in enumerate(levels):
            lev.t = lev.t_old = t0
            if l > 0:
                lev.ghosts = tuple(backend.index(a) for a in ghost_map(levels[l - 1], lev))
        self.root_steps = 0
        self.level_steps = [0] * len(levels)
        # a consistent start: the zones a subgrid covers are its projection (finest first)
        for l in range(len(levels) - 1, 0, -1):
            project_solution(levels[l - 1], levels[l], np)
        backend.adopt(levels)
        # initial ghost zones: periodic root, children from their parents
        backend.fill_periodic(levels[0])
        for l in range(1, len(levels)):
            p = levels[l - 1]
            p.old = backend.copy(p.fields)
            fill_child_ghosts(p, levels[l], levels[l].t, backend)

    def _dt(self, lev, t_end):
        a = self.cosmo.a(lev.t)
        dt = self.hp.cfl * self.be.timestep(lev, a)
        dt = min(dt, self.max_expansion / self.cosmo.adot_over_a(lev.t))
        return min(dt, t_end - lev.t)

    def _evolve(self, l, t_end, acc_root):
        lev = self.levels[l]
        be = self.be
        child = self.levels[l + 1] if l + 1 < len(self.levels) else None
        parent = self.levels[l - 1] if l > 0 else None
        while lev.t < t_end * (1.0 - 1e-14):
            dt = self._dt(lev, t_end)
            if parent is None:
                be.fill_periodic(lev)
            else:
                fill_child_ghosts(parent, lev, lev.t, be)
            lev.old = be.copy(lev.fields)
            lev.t_old = lev.t
            # flux boxes: the child's region on this level, and this level's own boundary
            boxes = []
            if child is not None:
                lo, hi = child_box(lev, child)
                boxes.append(flux_box_dict(lo, hi, lev.ggs, be.zeros, self.hp.dual))
            if parent is not None:
                boxes.append(flux_box_dict(NG, NG + lev.n - 1, lev.ggs, be.zeros, self.hp.dual))
            a_mid = self.cosmo.a(lev.t + 0.5 * dt)
            proper = dataclasses.replace(
                lev.grid, cellwidth=tuple(a_mid * cw for cw in lev.grid.cellwidth))
            be.solve(lev, proper, dt, lev.cycle, lev.accel, boxes)
            coef = dt * self.cosmo.adot_over_a(lev.t + 0.5 * dt)
            be.expansion_terms(lev, lev.old, lev.t + dt, lev.t, coef)
            lev.t += dt
            lev.cycle += 1
            self.level_steps[l] += 1
            if parent is not None:  # accumulate this level's boundary fluxes for the parent
                own = boxes[-1]
                if lev.own_fluxes is None:
                    lev.own_fluxes = own
                else:
                    for side in ("left", "right"):
                        for slot in range(6):
                            for d in range(3):
                                if own[side][slot][d] is not None:
                                    lev.own_fluxes[side][slot][d] += own[side][slot][d]
            if child is not None:
                child.own_fluxes = None
                self._evolve(l + 1, lev.t, acc_root)
                refined = project_fluxes(child.own_fluxes, child.n, self.hp.dual, be.xp)
                be.correct_fluxes(lev, [boxes[0]], [refined])
                project_solution(lev, child, be.xp)

    def step(self, t_final=math.inf):
        """One root step (the finer levels subcycle to the same time), ending at t_final
        at the latest."""
        root = self.levels[0]
        acc = gravity_profile(root, self.cosmo, root.t)
        for lev in self.levels:
            lev.own_fluxes = None
            lev.accel = self.be.accel(lev, level_accel(lev, root, acc))
        t_end = min(root.t + self._dt(root, math.inf), t_final)
        self._evolve(0, t_end, acc)
        self.root_steps += 1

    def run_to(self, z_final, max_root_steps=100000):
        """Root steps until the redshift z_final (or max_root_steps); returns the
        redshift reached."""
        t_final = self.cosmo.time_of(z_final)
        while self.levels[0].t < t_final * (1.0 - 1e-14) and self.root_steps < max_root_steps:
            self.step(t_final)
        return self.cosmo.redshift(self.levels[0].t)


# ---------------------------------------------------------------- backends
class LibraryBackend:
    """The library's C ABI on host fields (numpy; copies in and out inside each call)."""

    xp = np

    def __init__(self, ctx, hp):
        self.ctx = ctx
        self.hp = hp

    def adopt(self, levels):
        pass

    def copy(self, f):
        return {k: v.copy() for k, v in f.items()}

    def zeros(self, size):
        return np.zeros(size)

    def index(self, idx):
        return idx

    def accel(self, lev, prof):
        """The grid's three acceleration arrays from the x profile (kept per level)."""
        shape = lev.grid.shape
        if getattr(lev, "accel_arrays", None) is None:
            lev.accel_arrays = [np.zeros(shape), np.zeros(shape), np.zeros(shape)]
        lev.accel_arrays[0][...] = prof[None, None, :]
        return lev.accel_arrays

    def fill_periodic(self, lev):
        H.fill_ghosts(lev.grid, lev.fields, "periodic")

    def timestep(self, lev, aye):
        return self.ctx.compute_timestep(lev.grid, self.hp, lev.fields, courant=1.0, aye=aye)

    def solve(self, lev, grid, dt, cycle, accel, boxes):
        """SolvePPM_DE of a level; grid: the level's grid with proper cell widths."""
        self.ctx.solve_ppm_de(grid, self.hp, dt, cycle, lev.fields, accel=accel,
                              subgrids=boxes or None, ggs=lev.ggs)

    def expansion_terms(self, lev, old, time, old_time, coef):
        self.ctx.expansion_terms(lev.grid, self.hp, lev.fields, old, time, old_time, coef)

    def correct_fluxes(self, lev, initial, refined):
        self.ctx.correct_fluxes(lev.grid, self.hp, lev.fields, initial, refined, lev.ggs)


class DeviceBackend(LibraryBackend):
    """The library on device fields (torch tensors): the fields stay on the GPU; the ghost
    interpolation and projection run as torch operations, the subgrid flux boxes on the
    host.  For timing: torch's elementwise arithmetic is not the oracle's, so this
    backend agrees with the others to round-off, not bit for bit."""

    def __init__(self, ctx, hp, device="cuda"):
        super().__init__(ctx, hp)
        import torch
        self.torch = torch
        self.device = device
        self.xp = torch

    def adopt(self, levels):
        t = self.torch
        for lev in levels:
            lev.fields = {k: t.from_numpy(v).to(self.device) for k, v in lev.fields.items()}

    def copy(self, f):
        return {k: v.clone() for k, v in f.items()}

    def index(self, idx):
        return self.torch.as_tensor(idx, dtype=self.torch.int64, device=self.device)

    def accel(self, lev, prof):
        t = self.torch
        shape = lev.grid.shape
        if getattr(lev, "accel_arrays", None) is None:
            lev.accel_arrays = [t.zeros(shape, dtype=t.float64, device=self.device)
                                for _ in range(3)]
        lev.accel_arrays[0].copy_(t.from_numpy(prof).to(self.device).view(1, 1, -1).expand(shape))
        return lev.accel_arrays

    def fill_periodic(self, lev):
        self.ctx.set_boundary(lev.grid, lev.fields, self.hp.dual, ("periodic",) * 3)

    def timestep(self, lev, aye):
        from . import capi
        return self.ctx.compute_timestep(lev.grid, self.hp, lev.fields, memory=capi.MEM_DEVICE,
                                         courant=1.0, aye=aye)

    def solve(self, lev, grid, dt, cycle, accel, boxes):
        from . import capi
        self.ctx.solve_ppm_de(grid, self.hp, dt, cycle, lev.fields, memory=capi.MEM_DEVICE,
                              accel=accel, subgrids=boxes or None, ggs=lev.ggs,
                              want_stats=bool(boxes))

    def expansion_terms(self, lev, old, time, old_time, coef):
        from . import capi
        self.ctx.expansion_terms(lev.grid, self.hp, lev.fields, old, time, old_time, coef,
                                 memory=capi.MEM_DEVICE)

    def correct_fluxes(self, lev, initial, refined):
        from . import capi
        self.ctx.correct_fluxes(lev.grid, self.hp, lev.fields, initial, refined, lev.ggs,
                                memory=capi.MEM_DEVICE)
