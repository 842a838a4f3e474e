"""What Enzo does around the hydro call, restated for tests and benchmarks.

Enzo's hierarchy, boundary exchange and initialisers are outside the hot path;
this module provides just enough of them to drive ``grid::SolvePPM_DE``-style
calls: grid geometry with 3 ghost zones, the hydro parameter defaults of
``SetDefaultGlobalValues.C``, ghost-zone fill (outflow = copy of the nearest
active cell, periodic = wrap; ``ExternalBoundary_SetExternalBoundaryIO.C``
:201-209, :378-386), and seeded synthetic initial conditions.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

NGHOST = 3
FIELD_NAMES = ("d", "te", "v1", "v2", "v3", "ge")


@dataclasses.dataclass
class Grid:
    """One Enzo grid: GridRank, GridDimension, GridStartIndex, GridEndIndex."""

    rank: int
    dims: tuple
    start: tuple
    end: tuple
    cellwidth: tuple  # per-dim arrays of length dims[d] (CellWidth)

    @staticmethod
    def uniform(active, width=1.0, ghosts=NGHOST):
        """active: tuple of active cells per dim (len = rank); domain width per dim."""
        rank = len(active)
        dims, start, end, cw = [], [], [], []
        for d in range(3):
            if d < rank:
                n = int(active[d])
                dims.append(n + 2 * ghosts)
                start.append(ghosts)
                end.append(ghosts + n - 1)
                w = width[d] if isinstance(width, (tuple, list)) else width
                cw.append(np.full(n + 2 * ghosts, w / n, dtype=np.float64))
            else:
                dims.append(1)
                start.append(0)
                end.append(0)
                cw.append(np.ones(1, dtype=np.float64))
        return Grid(rank, tuple(dims), tuple(start), tuple(end), tuple(cw))

    @property
    def shape(self):
        """numpy shape (z, y, x) of one field, x fastest."""
        return (self.dims[2], self.dims[1], self.dims[0])

    @property
    def size(self):
        return self.dims[0] * self.dims[1] * self.dims[2]

    @property
    def active_cells(self):
        n = 1
        for d in range(self.rank):
            n *= self.end[d] - self.start[d] + 1
        return n

    def centers(self, d, left=0.0):
        """Cell-centre coordinates along dim d (ghosts included)."""
        w = self.cellwidth[d]
        edges = left + np.concatenate([[0.0], np.cumsum(w)]) - self.start[d] * w[0]
        return 0.5 * (edges[:-1] + edges[1:])

    def active_slices(self):
        return tuple(
            slice(self.start[d], self.end[d] + 1) for d in (2, 1, 0)
        )


@dataclasses.dataclass
class HydroParams:
    """Hydro globals consumed by the PPM-DE path (SetDefaultGlobalValues.C)."""

    gamma: float = 5.0 / 3.0          # Gamma (:194)
    cfl: float = 0.6                  # CourantSafetyNumber (:181)
    dual: bool = False                # DualEnergyFormalism
    eta1: float = 0.001               # DualEnergyFormalismEta1 (:425)
    eta2: float = 0.1                 # DualEnergyFormalismEta2 (:426)
    small_rho: float = 1e-30          # SmallRho (:803)
    tiny_number: float = 1e-20        # tiny_number -> MinimumPressure
    min_support: float = 0.0          # MinimumSupportEnergyCoefficient
    gravity: bool = False             # GravityOn
    pressure_free: bool = False       # PressureFree (:195)
    fallback: bool = True             # RiemannSolverFallback (:809)
    steepen: int = 0                  # PPMSteepeningParameter (:184): 0 or 1
    flatten: int = 0                  # PPMFlatteningParameter (:182): 0, 1 or 3
    eos_type: int = 0                 # EOSType: 0 ideal gas, 3 isothermal
    eos_sound_speed: float = 2.65e4   # EOSSoundSpeed (:814)
    riemann: int = 5                  # RiemannSolver: 5 TwoShock (the PPM default,
                                      # ReadParameterFile.C:1575-1576), 1 HLL, 4 HLLC


def new_fields(grid, dual):
    f = {n: np.zeros(grid.shape, dtype=np.float64) for n in FIELD_NAMES if n != "ge" or dual}
    return f


def _index_map(grid, d, bc):
    n = grid.dims[d]
    s, e = grid.start[d], grid.end[d]
    idx = np.arange(n)
    if n == 1:
        return idx
    if bc == "periodic":
        return s + (idx - s) % (e - s + 1)
    if bc == "outflow":
        return np.clip(idx, s, e)
    if bc == "none":  # ghosts filled elsewhere (e.g. a halo exchange)
        return idx
    raise ValueError(bc)


def fill_ghosts(grid, fields, bc="periodic"):
    """Ghost-zone fill on host arrays (in place); bc per dim or one string."""
    bcs = bc if isinstance(bc, (tuple, list)) else (bc,) * 3
    ix = _index_map(grid, 0, bcs[0])
    iy = _index_map(grid, 1, bcs[1])
    iz = _index_map(grid, 2, bcs[2])
    for k, a in fields.items():
        if a is None:
            continue
        a[...] = a[np.ix_(iz, iy, ix)]


# ---------------------------------------------------------------- initial conditions

def shock_tube(grid, hp, x0, left, right, dim=0):
    """Grid_HydroShockTubesInitializeGrid.C:72-116 (x <= x0 takes the left state).

    left/right: (rho, v, p) with v along `dim`."""
    f = new_fields(grid, hp.dual)
    xc = grid.centers(dim)
    shp = [1, 1, 1]
    shp[2 - dim] = grid.dims[dim]
    mask = (xc <= x0).reshape(shp)
    vel = ("v1", "v2", "v3")[dim]
    for (rho, v, p), m in ((left, mask), (right, ~mask)):
        etot = p / ((hp.gamma - 1.0) * rho) + 0.5 * (v * v)
        mb = np.broadcast_to(m, grid.shape)
        f["d"][mb] = rho
        f[vel][mb] = v
        f["te"][mb] = etot
        if hp.dual:
            f["ge"][mb] = etot - 0.5 * (v * v)
    return f


def _grf(n, slope, rng):
    """Unit-variance periodic Gaussian random field on n^3 with P(k) ~ k^slope."""
    k = np.fft.fftfreq(n) * n
    kx, ky, kz = np.meshgrid(k, k, k[: n // 2 + 1], indexing="ij")
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    amp = np.zeros_like(kk)
    nz = kk > 0
    amp[nz] = kk[nz] ** (slope / 2.0)
    noise = rng.standard_normal(kk.shape) + 1j * rng.standard_normal(kk.shape)
    g = np.fft.irfftn(noise * amp, s=(n, n, n), axes=(0, 1, 2))
    g -= g.mean()
    g /= g.std()
    return g


def _solenoidal(n, slope, rng):
    k = np.fft.fftfreq(n) * n
    kx, ky, kz = np.meshgrid(k, k, k[: n // 2 + 1], indexing="ij")
    kk2 = kx * kx + ky * ky + kz * kz
    kk = np.sqrt(kk2)
    amp = np.zeros_like(kk)
    nz = kk > 0
    amp[nz] = kk[nz] ** (slope / 2.0)
    comps = [
        (rng.standard_normal(kk.shape) + 1j * rng.standard_normal(kk.shape)) * amp
        for _ in range(3)
    ]
    kv = (kx, ky, kz)
    div = sum(c * kc for c, kc in zip(comps, kv))
    safe = np.where(nz, kk2, 1.0)
    comps = [c - kc * div / safe for c, kc in zip(comps, kv)]
    out = [np.fft.irfftn(c, s=(n, n, n), axes=(0, 1, 2)) for c in comps]
    return out


def turbulence(grid, hp, mach=3.0, sigma_lnrho=0.5, seed=1234):
    """Decaying supersonic turbulence IC on a periodic cube.

    Density lognormal (sigma_ln rho) from a seeded GRF with P(k) ~ k^-2, normalised to
    <rho> = 1; velocity a solenoidal GRF with P(k) ~ k^-4 scaled to rms Mach `mach`
    at c_s = 1; uniform pressure p = 1/gamma."""
    assert grid.rank == 3
    n = grid.end[0] - grid.start[0] + 1
    assert all(grid.end[d] - grid.start[d] + 1 == n for d in range(3))
    rng = np.random.default_rng(seed)
    g = _grf(n, -2.0, rng)
    rho = np.exp(sigma_lnrho * g - 0.5 * sigma_lnrho ** 2)
    rho /= rho.mean()
    vx, vy, vz = _solenoidal(n, -4.0, rng)
    vrms = np.sqrt(np.mean(vx * vx + vy * vy + vz * vz))
    scale = mach / vrms
    # fields are stored (z, y, x); the generator's axes are (x, y, z)
    to_zyx = lambda a: np.ascontiguousarray(np.transpose(a, (2, 1, 0)))
    p0 = 1.0 / hp.gamma
    f = new_fields(grid, hp.dual)
    act = grid.active_slices()
    f["d"][act] = to_zyx(rho)
    f["v1"][act] = to_zyx(vx * scale)
    f["v2"][act] = to_zyx(vy * scale)
    f["v3"][act] = to_zyx(vz * scale)
    eint = p0 / ((hp.gamma - 1.0) * f["d"][act])
    ke = 0.5 * (f["v1"][act] ** 2 + f["v2"][act] ** 2 + f["v3"][act] ** 2)
    f["te"][act] = eint + ke
    if hp.dual:
        f["ge"][act] = eint
    fill_ghosts(grid, f, "periodic")
    return f


def turbulence_device(grid, hp, mach=3.0, sigma_lnrho=0.5, seed=1234, device="cuda"):
    """`turbulence` generated on the GPU with torch (for grids of 512^3 and more, where
    the host FFTs take minutes): the same spectra, normalisations and uniform pressure,
    from torch's seeded generator (a different realisation than the numpy one).
    Returns device float64 tensors with periodic ghosts, in the BaryonField layout."""
    import torch

    assert grid.rank == 3
    n = grid.end[0] - grid.start[0] + 1
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    k = torch.fft.fftfreq(n, device=device, dtype=torch.float64) * n
    kz = torch.fft.rfftfreq(n, device=device, dtype=torch.float64) * n
    kx, ky, kzz = torch.meshgrid(k, k, kz, indexing="ij")
    kk2 = kx * kx + ky * ky + kzz * kzz
    nz = kk2 > 0

    def amp(slope):
        a = torch.zeros_like(kk2)
        a[nz] = kk2[nz] ** (slope / 4.0)  # |k|^(slope/2)
        return a

    def noise():
        re = torch.randn(kk2.shape, generator=gen, device=device, dtype=torch.float64)
        im = torch.randn(kk2.shape, generator=gen, device=device, dtype=torch.float64)
        return torch.complex(re, im)

    g = torch.fft.irfftn(noise() * amp(-2.0), s=(n, n, n), dim=(0, 1, 2))
    g = (g - g.mean()) / g.std()
    rho = torch.exp(sigma_lnrho * g - 0.5 * sigma_lnrho ** 2)
    rho = rho / rho.mean()
    del g
    a4 = amp(-4.0)
    comps = [noise() * a4 for _ in range(3)]
    kv = (kx, ky, kzz)
    div = sum(c * kc for c, kc in zip(comps, kv))
    safe = torch.where(nz, kk2, torch.ones_like(kk2))
    vel = []
    for c, kc in zip(comps, kv):
        vel.append(torch.fft.irfftn(c - kc * div / safe, s=(n, n, n), dim=(0, 1, 2)))
    del comps, div, safe, kx, ky, kzz, kk2, a4
    vrms = torch.sqrt(torch.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2))
    scale = mach / vrms
    p0 = 1.0 / hp.gamma
    shape = grid.shape
    f = {}
    for name in ("d", "te", "v1", "v2", "v3") + (("ge",) if hp.dual else ()):
        f[name] = torch.zeros(shape, dtype=torch.float64, device=device)
    act = grid.active_slices()
    to_zyx = lambda a: a.permute(2, 1, 0).contiguous()
    f["d"][act] = to_zyx(rho)
    for name, v in zip(("v1", "v2", "v3"), vel):
        f[name][act] = to_zyx(v * scale)
    eint = p0 / ((hp.gamma - 1.0) * f["d"][act])
    ke = 0.5 * (f["v1"][act] ** 2 + f["v2"][act] ** 2 + f["v3"][act] ** 2)
    f["te"][act] = eint + ke
    if hp.dual:
        f["ge"][act] = eint
    # periodic ghosts
    gz = grid.start[0]
    for ax in range(3):
        dim = 2 - ax
        s, e = grid.start[dim], grid.end[dim]
        for name in f:
            t = f[name]
            lo = [slice(None)] * 3
            hi = [slice(None)] * 3
            src_lo = [slice(None)] * 3
            src_hi = [slice(None)] * 3
            lo[ax] = slice(0, s)
            src_lo[ax] = slice(e + 1 - gz, e + 1)
            hi[ax] = slice(e + 1, e + 1 + gz)
            src_hi[ax] = slice(s, s + gz)
            t[tuple(lo)] = t[tuple(src_lo)]
            t[tuple(hi)] = t[tuple(src_hi)]
    return f


def zeldovich_pancake(grid, hp, z_init=100.0, z_collapse=1.0, e_init=1e-6, offset=0.0):
    """A Zel'dovich pancake along x in code units (the published one-dimensional
    solution that Grid_ZeldovichPancakeInitializeGrid.C:132-189 sets up): zone q of the
    N active zones has the Lagrangian position q + 1/2 - offset - N/2 (in zones), mapped
    to its Eulerian x by Newton's method on x - A sin(kx)/k = x_L with A = (1+z_c)/(1+z_i)
    and k = 2 pi / N; the density is 1/(1 - A cos kx), the x velocity
    -sqrt(2/3) (1+z_c)/((1+z_i) 2 pi) sin kx, the specific internal energy e_init times
    rho^(gamma-1) (adiabatic from a uniform start).  Ghost zones periodic."""
    f = new_fields(grid, hp.dual)
    n = grid.end[0] - grid.start[0] + 1
    amp = (1.0 + z_collapse) / (1.0 + z_init)
    amp_v = -np.sqrt(2.0 / 3.0) * (1.0 + z_collapse) / ((1.0 + z_init) * 2.0 * np.pi)
    k = 2.0 * np.pi / n
    x_l = np.arange(n) + (0.5 - offset) - 0.5 * n
    x_e = x_l.copy()
    for _ in range(100):  # Newton iteration, converged well before the bound
        step = (x_l - x_e + amp * np.sin(k * x_e) / k) / (1.0 - amp * np.cos(k * x_e))
        x_e = x_e + step
        if np.all(np.abs(step) <= 1e-14 * np.maximum(np.abs(x_e), 1.0)):
            break
    rho = 1.0 / (1.0 - amp * np.cos(k * x_e))
    u = amp_v * np.sin(k * x_e)
    e_int = e_init * rho ** (hp.gamma - 1.0) / (hp.gamma - 1.0)
    act = grid.active_slices()
    f["d"][act] = rho[None, None, :]
    f["v1"][act] = u[None, None, :]
    if hp.dual:
        f["ge"][act] = e_int[None, None, :]
    f["te"][act] = (e_int + 0.5 * u * u)[None, None, :]
    fill_ghosts(grid, f, "periodic")
    return f


def sedov(grid, hp, e_blast=1.0, rho0=1.0, p0=1e-5):
    """Point blast: E deposited as thermal energy in the central 2^3 active cells."""
    assert grid.rank == 3
    f = new_fields(grid, hp.dual)
    f["d"][...] = rho0
    eint0 = p0 / ((hp.gamma - 1.0) * rho0)
    f["te"][...] = eint0
    if hp.dual:
        f["ge"][...] = eint0
    c = [grid.start[d] + (grid.end[d] - grid.start[d] + 1) // 2 for d in range(3)]
    vol = grid.cellwidth[0][0] * grid.cellwidth[1][0] * grid.cellwidth[2][0]
    e_spec = e_blast / (8.0 * vol * rho0)
    sl = (slice(c[2] - 1, c[2] + 1), slice(c[1] - 1, c[1] + 1), slice(c[0] - 1, c[0] + 1))
    f["te"][sl] += e_spec
    if hp.dual:
        f["ge"][sl] += e_spec
    return f


def amr_level(hp, npatch=600, lo=16, hi=128, seed=2024, sedov_fraction=0.5, source_n=128,
              mach=3.0):
    """One AMR level of `npatch` patches for batched solves.

    Edge lengths are drawn independently per axis, log-uniform in [lo, hi] (non-cubic
    patches), every patch with 3 ghost zones and the level's cell width 1/source_n.
    A patch holds either a Sedov blast (E = 1 in its central 2^3 cells, rho = 1,
    p = 1e-5) or a periodic crop, ghosts included, of one turbulence field of
    source_n^3 cells (the generator of `turbulence`, rms Mach `mach`).
    Returns (grids, fields) lists."""
    rng = np.random.default_rng(seed)
    src_grid = Grid.uniform((source_n,) * 3)
    src = turbulence(src_grid, hp, mach=mach, seed=seed + 1)
    act = src_grid.active_slices()
    src = {k: np.ascontiguousarray(v[act]) for k, v in src.items()}
    grids, fields = [], []
    for _ in range(npatch):
        edges = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=3))).astype(int)
        edges = np.clip(edges, lo, hi)
        g = Grid.uniform(tuple(int(e) for e in edges),
                         width=tuple(float(e) / source_n for e in edges))
        if rng.random() < sedov_fraction:
            f = sedov(g, hp)
        else:
            off = rng.integers(0, source_n, size=3)
            idx = [(off[d] - NGHOST + np.arange(g.dims[d])) % source_n for d in range(3)]
            f = new_fields(g, hp.dual)
            for k in f:
                f[k][...] = src[k][np.ix_(idx[2], idx[1], idx[0])]
        grids.append(g)
        fields.append(f)
    return grids, fields


def pressure_np(grid, hp, fields):
    """grid::ComputePressure (time == Time) in numpy, for diagnostics."""
    g = hp.gamma
    if hp.dual:
        ge = fields["ge"]
    else:
        v2 = fields["v1"] ** 2
        if grid.rank > 1:
            v2 = v2 + fields["v2"] ** 2
        if grid.rank > 2:
            v2 = v2 + fields["v3"] ** 2
        ge = fields["te"] - 0.5 * v2
    p = (g - 1.0) * fields["d"] * ge
    return np.maximum(p, hp.tiny_number)


def max_signal_dt(grid, hp, fields):
    """CFL dt (calc_dt.F, ihydro=0) times the Courant factor, numpy version."""
    p = pressure_np(grid, hp, fields)
    act = grid.active_slices()
    cs = np.maximum(np.sqrt(hp.gamma * p[act] / fields["d"][act]), 1e-20)
    s = 0.0
    names = ("v1", "v2", "v3")
    for d in range(grid.rank):
        s = s + (cs + np.abs(fields[names[d]][act])) / grid.cellwidth[d][0]
    return hp.cfl / float(np.max(s))
