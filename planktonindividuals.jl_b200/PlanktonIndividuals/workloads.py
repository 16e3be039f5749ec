"""Seeded synthetic workloads with the shapes of the benchmark configurations.

config1: 2D horizontal, 128×128×1, dx=dy=1 km, dz=10 m, 1 species × 16384 individuals,
         steady double-gyre velocity (peak 0.1 m/s), dt = 60 s.
config2: 3D 256×256×64, dx=dy=50 m, dz=2 m, 2 species × 2,097,152 individuals seeded in the top
         40 m, divergence-free random-Fourier velocity (256 modes, k^-5/3, rms 0.05 m/s) refreshed
         every 60 steps, linear NO3 gradient with depth, dt = 30 s.
config3: 3D 512×512×128, 4 species × 16,777,216 individuals, lognormal sizes with
         μ ∈ {-0.5, 0, 0.5, 1}, σ = 0.25, random-Fourier velocity, dt = 20 s.
Every size can be scaled down for tests with the keyword arguments.

Individuals: positions uniform in the seeded region; size Sz ~ LogNormal(μ, σ);
Bm = Cquota·Sz·Nsuper; quotas at half their maximum (the mean of the reference's uniform
initialisation, plankton_generation.jl:64-68) times U(0.8, 1.2); Chl = Chl2Cint·Bm; gen = 1,
age = 0; capacity = 2 × initial population. Tracers: DIC 20, NH4 0.5, NO3 0.8, PO4 0.10,
DOC 10, DON 0.1, DOP 0.05, POC/PON/POP 0, each × U(0.9, 1.1); DFe, PFe_inorg, PFe_bio and Dust
are 0. Light: 1000·max(0, sin(2π(t/86400 − 1/4))) µmol m⁻² s⁻¹ sampled at the middle of each
hour (ΔT_PAR = 3600 s). Temperature: default_temperature (param_default.jl:22-38).
"""
from dataclasses import dataclass, field

import numpy as np

from ._abi import tracer_names
from .grids import Bounded, LatLonGrid, Periodic, RectilinearGrid, fill_halo_tracer
from .init import empty_individuals
from .parameters import default_temperature, update_bgc_params, update_phyt_params


@dataclass
class Workload:
    name: str
    grid: RectilinearGrid
    bgc: dict
    phyt: dict
    nsp: int
    capacity: int
    N: list
    individuals: list
    tracers: list
    dT: float
    steps: int
    dT_vel: float
    n_vel: int
    vel_fn: object            # vel_fn(snapshot_index) -> (u, v, w)
    parf: np.ndarray          # (Nx, Ny, npar)
    dT_PAR: float
    temp: np.ndarray          # (Nx, Ny, Nz, ntemp)
    dT_temp: float
    seed: int
    meta: dict = field(default_factory=dict)
    mode: str = "quota"           # physiology: "quota" (QuotaMode), "carbon" (CarbonMode) or "macro"

    def velocity(self, t):
        return self.vel_fn(t)

    def snapshots_needed(self, iterations):
        """Velocity snapshots that `iterations` steps from t = 0 read (update.jl:18)."""
        return int(np.floor((iterations - 1) * self.dT / self.dT_vel)) + 1 if iterations > 0 else 1


def diel_parf(Nx, Ny, hours, peak=1000.0, phase=0.0):
    h = np.arange(hours, dtype=np.float64)
    t = (h + 0.5) * 3600.0 + phase
    val = peak * np.maximum(0.0, np.sin(2.0 * np.pi * (t / 86400.0 - 0.25)))
    return np.asfortranarray(np.broadcast_to(val[None, None, :], (Nx, Ny, hours)).copy(order="F"))


def make_individuals(grid, phyt, s, N, C, rng, zmax=None, mu=0.0, sigma=0.2):
    p = {k: (v[s] if hasattr(v, "__len__") else v) for k, v in phyt.items()}
    d = empty_individuals(C)
    zmax = grid.Nz if zmax is None else zmax
    d["ac"][:N] = True
    d["x"][:N] = rng.random(N) * grid.Nx
    d["y"][:N] = rng.random(N) * grid.Ny
    d["z"][:N] = rng.random(N) * zmax
    Sz = np.exp(rng.normal(mu, sigma, N))
    Bm = float(p["Cquota"]) * Sz * float(p["Nsuper"])
    Cq = 0.5 * float(p["Cqmax"]) * Bm * rng.uniform(0.8, 1.2, N)
    Nq = 0.5 * (float(p["Nqmax"]) * (Bm + Cq) - Bm * float(p["R_NC"])) * rng.uniform(0.8, 1.2, N)
    Pq = 0.5 * (float(p["Pqmax"]) * (Bm + Cq) - Bm * float(p["R_PC"])) * rng.uniform(0.8, 1.2, N)
    d["Sz"][:N] = Sz
    d["Bm"][:N] = Bm
    d["Cq"][:N] = Cq
    d["Nq"][:N] = Nq
    d["Pq"][:N] = Pq
    d["Chl"][:N] = float(p["Chl2Cint"]) * Bm
    d["gen"][:N] = 1.0
    return d


TRACER_INIT = dict(DIC=20.0, NH4=0.5, NO3=0.8, PO4=0.10, DOC=10.0, DON=0.1, DOP=0.05,
                   POC=0.0, PON=0.0, POP=0.0)


def make_tracers(grid, rng, no3_gradient_depth=None):
    out = []
    shape = grid.total_size
    zc = -np.asarray(grid.zC, dtype=np.float64)   # depth of cell centres, with halos
    for name in tracer_names:
        v0 = TRACER_INIT.get(name, 0.0)
        a = np.asfortranarray(v0 * rng.uniform(0.9, 1.1, shape))
        if name == "NO3" and no3_gradient_depth:
            a *= (1.0 + zc / no3_gradient_depth)[None, None, :]
        a *= grid.landmask
        fill_halo_tracer(a, grid)
        out.append(np.asfortranarray(a))
    return out


def double_gyre(grid, peak=0.1):
    """Steady double gyre on the C-grid from a corner streamfunction, following the recipe of the
    reference's examples/helper_functions.jl:38-59: ψ = 0.3 sin(πx/L) sin(2πy/L) +
    0.7 sin(2πx/L) sin(πy/L), u = -δyψ, v = δxψ, w = 0; scaled so max(|u|, |v|) = peak."""
    Nx, Ny, Nz = grid.Nx, grid.Ny, grid.Nz
    xs = np.arange(Nx + 1, dtype=np.float64)[:, None]
    ys = np.arange(Ny + 1, dtype=np.float64)[None, :]
    phi = 0.3 * np.sin(np.pi * xs / Nx) * np.sin(2 * np.pi * ys / Ny) + \
        0.7 * np.sin(2 * np.pi * xs / Nx) * np.sin(np.pi * ys / Ny)
    uu = -(phi[:, 1:] - phi[:, :-1])[:-1, :]
    vv = (phi[1:, :] - phi[:-1, :])[:, :-1]
    s = peak / max(np.abs(uu).max(), np.abs(vv).max())
    u = np.asfortranarray(np.repeat((uu * s)[:, :, None], Nz, axis=2))
    v = np.asfortranarray(np.repeat((vv * s)[:, :, None], Nz, axis=2))
    w = np.zeros((Nx, Ny, Nz + 1), order="F")
    return u, v, w


class FourierVelocity:
    """Divergence-free velocity u = ∇×A on the C-grid from a vector potential of `nmodes` random
    Fourier modes per component. Horizontal wavenumbers are integers (periodic in x and y) with
    |k| uniform in [1, kmax]; potential amplitudes scale as |k|^(-11/6), so the velocity energy
    spectrum follows k^(-5/3). A_x and A_y vary as sin(nπ d/H) with depth d so w = 0 at the
    surface and the bottom (Bounded z); A_z varies as cos(nπ d/H). The discrete divergence
    (u[i+1]-u[i])/Δx + (v[j+1]-v[j])/Δy + (w[k]-w[k+1])/Δz is zero up to rounding. Each snapshot
    is scaled to the requested rms speed."""

    def __init__(self, grid, nmodes=256, rms=0.05, seed=0, kmax=None, vert_ratio=0.3):
        self.g = grid
        self.nmodes, self.rms, self.seed = nmodes, rms, seed
        self.kmax = kmax or max(2, min(grid.Nx, grid.Ny) // 8)
        self.vert_ratio = vert_ratio

    def _modes(self, snap, comp):
        rng = np.random.default_rng([self.seed, snap, comp])
        M = self.nmodes
        kabs = rng.uniform(1.0, self.kmax, M)
        ang = rng.uniform(0, 2 * np.pi, M)
        nx = np.rint(kabs * np.cos(ang)).astype(int)
        ny = np.rint(kabs * np.sin(ang)).astype(int)
        zero = (nx == 0) & (ny == 0)
        nx[zero] = 1
        nz = rng.integers(1, 4, M) if comp < 2 else rng.integers(0, 3, M)
        amp = np.hypot(nx, ny) ** (-11.0 / 6.0)
        phase = rng.uniform(0, 2 * np.pi, M)
        return nx, ny, nz, amp, phase

    def _potential(self, snap, comp, xpos, ypos, dpos):
        """Σ_m a_m sin(kx x + ky y + φ) Z_m(d) at x (cells), y (cells), depth d (cells)."""
        g = self.g
        nx, ny, nz, amp, phase = self._modes(snap, comp)
        X = np.exp(1j * (2 * np.pi * np.outer(nx, xpos) / g.Nx))          # (M, nx)
        Y = np.exp(1j * (2 * np.pi * np.outer(ny, ypos) / g.Ny))          # (M, ny)
        if comp < 2:
            Z = np.sin(np.pi * np.outer(nz, dpos) / g.Nz)                  # (M, nd)
        else:
            Z = np.cos(np.pi * np.outer(nz, dpos) / g.Nz)
        W = (amp * np.exp(1j * phase))[:, None] * Z                        # (M, nd)
        out = np.empty((len(xpos), len(ypos), len(dpos)))
        step = max(1, int(2 ** 22 // max(1, len(xpos) * self.nmodes)))
        for j0 in range(0, len(ypos), step):
            j1 = min(len(ypos), j0 + step)
            XY = (X[:, :, None] * Y[:, None, j0:j1]).reshape(self.nmodes, -1)   # (M, nx*nyc)
            F = XY.T @ W                                                         # (nx*nyc, nd)
            out[:, j0:j1, :] = F.imag.reshape(len(xpos), j1 - j0, len(dpos))
        return out

    def __call__(self, snap):
        g = self.g
        Nx, Ny, Nz = g.Nx, g.Ny, g.Nz
        dx, dy = g.Δx, g.Δy
        dz = float(np.asarray(g.dzF)[g.Hz])
        xf, xc = np.arange(Nx + 1, dtype=float), np.arange(Nx + 1, dtype=float) + 0.5
        yf, yc = np.arange(Ny + 1, dtype=float), np.arange(Ny + 1, dtype=float) + 0.5
        df, dc = np.arange(Nz + 1, dtype=float), np.arange(Nz, dtype=float) + 0.5
        r = self.vert_ratio
        Ah = self._potential(snap, 2, xf, yf, dc)              # (x face, y face, d centre)
        Ay = r * self._potential(snap, 1, xf, yc, df)          # (x face, y centre, d face)
        Ax = r * self._potential(snap, 0, xc, yf, df)          # (x centre, y face, d face)
        Ay[:, :, 0] = 0.0; Ay[:, :, -1] = 0.0
        Ax[:, :, 0] = 0.0; Ax[:, :, -1] = 0.0
        # u at (x face i, y centre j, d centre k); v at (x centre, y face, d centre); w at d faces
        u = (Ah[:Nx, 1:Ny + 1, :] - Ah[:Nx, :Ny, :]) / dy - (Ay[:Nx, :Ny, :-1] - Ay[:Nx, :Ny, 1:]) / dz
        v = (Ax[:Nx, :Ny, :-1] - Ax[:Nx, :Ny, 1:]) / dz - (Ah[1:Nx + 1, :Ny, :] - Ah[:Nx, :Ny, :]) / dx
        w = (Ay[1:Nx + 1, :Ny, :] - Ay[:Nx, :Ny, :]) / dx - (Ax[:Nx, 1:Ny + 1, :] - Ax[:Nx, :Ny, :]) / dy
        s = self.rms / np.sqrt(np.mean(u ** 2) + np.mean(v ** 2) + np.mean(w[:, :, :Nz] ** 2))
        return (np.asfortranarray(u * s), np.asfortranarray(v * s), np.asfortranarray(w * s))


def _finish(name, grid, nsp, N, C, phyt_over, bgc_over, dT, steps, rng, vel_fn, n_vel, dT_vel, zmax,
            mus, sigma, seed, no3_grad=None, parf_peak=1000.0):
    FT = np.float64
    bgc = update_bgc_params(bgc_over or {}, FT)
    phyt = update_phyt_params(phyt_over or {}, FT, N=nsp)
    inds = [make_individuals(grid, phyt, s, N[s], C, rng, zmax=zmax, mu=mus[s], sigma=sigma)
            for s in range(nsp)]
    trs = make_tracers(grid, rng, no3_gradient_depth=no3_grad)
    hours = int(np.ceil(steps * dT / 3600.0)) + 1
    parf = diel_parf(grid.Nx, grid.Ny, hours, peak=parf_peak)
    temp = default_temperature(grid, dT, steps)
    return Workload(name, grid, bgc, phyt, nsp, C, list(N), inds, trs, dT, steps, dT_vel, n_vel,
                    vel_fn, parf, 3600.0, temp, 3600.0, seed)


def config1(n=128, N=16384, steps=1440, dT=60.0, seed=1, capacity=None, phyt_over=None):
    """Plain FP64, 2D horizontal (n×n×1, 1 km cells, 10 m deep)."""
    rng = np.random.default_rng(seed)
    grid = RectilinearGrid(size=(n, n, 1), x=(0.0, n * 1000.0), y=(0.0, n * 1000.0), z=(0.0, -10.0),
                           FT=np.float64, topology=(Periodic, Periodic, Bounded))
    u, v, w = double_gyre(grid, 0.1)
    C = capacity or 2 * N
    return _finish("config1", grid, 1, [N], C, phyt_over, None, dT, steps, rng,
                   lambda t: (u, v, w), 1, dT * steps, None, [0.0], 0.2, seed)


def config2(nx=256, nz=64, N_per_species=2_097_152, nsp=2, steps=1000, dT=30.0, seed=2,
            nmodes=256, capacity=None, phyt_over=None):
    """FP64/FP32 3D (nx×nx×nz, 50 m × 50 m × 2 m), individuals in the top 40 m."""
    rng = np.random.default_rng(seed)
    grid = RectilinearGrid(size=(nx, nx, nz), x=(0.0, nx * 50.0), y=(0.0, nx * 50.0),
                           z=(0.0, -2.0 * nz), FT=np.float64, topology=(Periodic, Periodic, Bounded))
    vel = FourierVelocity(grid, nmodes=nmodes, rms=0.05, seed=seed)
    C = capacity or 2 * N_per_species
    zmax = min(nz, 20)
    n_vel = int(np.ceil(steps / 60)) + 1
    return _finish("config2", grid, nsp, [N_per_species] * nsp, C, phyt_over, None, dT, steps, rng,
                   vel, n_vel, 60 * dT, zmax, [0.0] * nsp, 0.2, seed, no3_grad=2.0 * nz)


def carbon(nx=16, nz=8, N_per_species=2000, nsp=2, steps=30, dT=60.0, seed=11, nmodes=16,
           capacity=None, phyt_over=None, temp=None, bd_frac=0.0):
    """CarbonMode workload on a config-2-like 3D grid (nx×nx×nz, 50 m × 50 m × 2 m): individuals
    from CarbonMode's initialize_plankton! rule, optionally with damaged biomass Bd = Bm·U(0,
    bd_frac); `temp` (°C, scalar or interior array) replaces the default temperature so that the
    thermal damage and repair terms (T > Topt) can be exercised."""
    from .architectures import CarbonMode
    from .init import initialize_plankton_carbon
    rng = np.random.default_rng(seed)
    grid = RectilinearGrid(size=(nx, nx, nz), x=(0.0, nx * 50.0), y=(0.0, nx * 50.0),
                           z=(0.0, -2.0 * nz), FT=np.float64, topology=(Periodic, Periodic, Bounded))
    vel = FourierVelocity(grid, nmodes=nmodes, rms=0.05, seed=seed)
    C = capacity or 2 * N_per_species
    bgc = update_bgc_params({}, np.float64)
    phyt = update_phyt_params(phyt_over or {}, np.float64, N=nsp, mode=CarbonMode())
    inds = []
    for s in range(nsp):
        d = initialize_plankton_carbon(grid, phyt, s, N_per_species, C, rng)
        if bd_frac:
            d["Bd"] = d["Bm"] * rng.uniform(0.0, bd_frac, C) * d["ac"]
        inds.append(d)
    trs = make_tracers(grid, rng, no3_gradient_depth=2.0 * nz)
    hours = int(np.ceil(steps * dT / 3600.0)) + 1
    parf = diel_parf(grid.Nx, grid.Ny, hours)
    tmp = default_temperature(grid, dT, steps)
    if temp is not None:
        tmp = np.asfortranarray(np.broadcast_to(np.asarray(temp, dtype=np.float64)[..., None] if np.ndim(temp) == 3
                                                else np.float64(temp), tmp.shape).copy())
    n_vel = int(np.ceil(steps / 60)) + 1
    return Workload("carbon", grid, bgc, phyt, nsp, C, [N_per_species] * nsp, inds, trs, dT, steps,
                    60 * dT, n_vel, vel, parf, 3600.0, tmp, 3600.0, seed, mode="carbon")


def macro(nx=16, nz=8, N_per_species=2000, nsp=2, steps=30, dT=60.0, seed=13, nmodes=16,
          capacity=None, phyt_over=None, bgc_over=None):
    """MacroMolecularMode workload on a config-2-like 3D grid (nx×nx×nz, 50 m × 50 m × 2 m):
    individuals from MacroMolecularMode's initialize_plankton! rule, random-Fourier velocity,
    default temperature and a diel light cycle."""
    from .architectures import MacroMolecularMode
    from .init import initialize_plankton_macro
    rng = np.random.default_rng(seed)
    grid = RectilinearGrid(size=(nx, nx, nz), x=(0.0, nx * 50.0), y=(0.0, nx * 50.0),
                           z=(0.0, -2.0 * nz), FT=np.float64, topology=(Periodic, Periodic, Bounded))
    vel = FourierVelocity(grid, nmodes=nmodes, rms=0.05, seed=seed)
    C = capacity or 2 * N_per_species
    bgc = update_bgc_params(bgc_over or {}, np.float64)
    phyt = update_phyt_params(phyt_over or {}, np.float64, N=nsp, mode=MacroMolecularMode())
    inds = [initialize_plankton_macro(grid, phyt, s, N_per_species, C, rng) for s in range(nsp)]
    trs = make_tracers(grid, rng, no3_gradient_depth=2.0 * nz)
    hours = int(np.ceil(steps * dT / 3600.0)) + 1
    parf = diel_parf(grid.Nx, grid.Ny, hours)
    tmp = default_temperature(grid, dT, steps)
    n_vel = int(np.ceil(steps / 60)) + 1
    return Workload("macro", grid, bgc, phyt, nsp, C, [N_per_species] * nsp, inds, trs, dT, steps,
                    60 * dT, n_vel, vel, parf, 3600.0, tmp, 3600.0, seed, mode="macro")


def iron(nx=16, nz=8, N_per_species=2000, nsp=2, steps=40, dT=120.0, seed=19, nmodes=16,
         capacity=None, phyt_over=None, bgc_over=None, start_hour=17.5, DFe=1.0e-3):
    """IronEnergyMode workload on a config-2-like 3D grid (nx×nx×nz, 50 m × 50 m × 2 m):
    individuals from IronEnergyMode's initialize_plankton! rule, random-Fourier velocity, default
    temperature, DFe ≈ `DFe` (±10 %), and the diel light cycle from `start_hour` (17:30: the
    first hour lit, then night, so that a run of more than 30 steps of 120 s crosses sunset)."""
    from .architectures import IronEnergyMode
    from .init import initialize_plankton_iron
    rng = np.random.default_rng(seed)
    grid = RectilinearGrid(size=(nx, nx, nz), x=(0.0, nx * 50.0), y=(0.0, nx * 50.0),
                           z=(0.0, -2.0 * nz), FT=np.float64, topology=(Periodic, Periodic, Bounded))
    vel = FourierVelocity(grid, nmodes=nmodes, rms=0.05, seed=seed)
    C = capacity or 2 * N_per_species
    bgc = update_bgc_params(bgc_over or {}, np.float64)
    phyt = update_phyt_params(phyt_over or {}, np.float64, N=nsp, mode=IronEnergyMode())
    inds = [initialize_plankton_iron(grid, phyt, s, N_per_species, C, rng) for s in range(nsp)]
    trs = make_tracers(grid, rng, no3_gradient_depth=2.0 * nz)
    trs[tracer_names.index("DFe")] = np.asfortranarray(DFe * rng.uniform(0.9, 1.1, grid.total_size))
    fill_halo_tracer(trs[tracer_names.index("DFe")], grid)
    hours = int(np.ceil(steps * dT / 3600.0)) + 1
    parf = diel_parf(grid.Nx, grid.Ny, hours, phase=(start_hour - 0.5) * 3600.0)
    tmp = default_temperature(grid, dT, steps)
    n_vel = int(np.ceil(steps / 60)) + 1
    return Workload("iron", grid, bgc, phyt, nsp, C, [N_per_species] * nsp, inds, trs, dT, steps,
                    60 * dT, n_vel, vel, parf, 3600.0, tmp, 3600.0, seed, mode="iron")


def latlon_streamfunction_velocity(grid, cfl=0.2, dT=600.0, seed=0):
    """Divergence-free flow on a LatLonGrid from a corner streamfunction ψ of volume transport:
    U = −(ψ[i, j+1] − ψ[i, j]), V = ψ[i+1, j] − ψ[i, j] per level, u = U/Ax and v = V/Ay at the
    faces, w = 0, so every cell's transports sum to zero up to rounding. ψ vanishes on Bounded
    edges (no flow through them) and is periodic in x when x is Periodic. Scaled so the largest
    Courant number |u|ΔT/ΔxC, |v|ΔT/ΔyC is `cfl`."""
    rng = np.random.default_rng(seed)
    Nx, Ny, Nz, Hx, Hy, Hz = grid.Nx, grid.Ny, grid.Nz, grid.Hx, grid.Hy, grid.Hz
    px = grid.topo[0] == Periodic.code
    xs = np.arange(Nx + 1, dtype=np.float64)[:, None]
    ys = np.arange(Ny + 1, dtype=np.float64)[None, :]
    fx = np.sin(2 * np.pi * xs / Nx + rng.uniform(0, 2 * np.pi)) if px else np.sin(np.pi * xs / Nx)
    psi2 = fx * np.sin(np.pi * ys / Ny) + 0.3 * np.sin(2 * np.pi * xs / Nx) * np.sin(2 * np.pi * ys / Ny)
    prof = 1.0 + 0.5 * np.cos(np.pi * (np.arange(Nz) + 0.5) / Nz)
    nxu = Nx + (0 if px else 1)
    U = np.zeros((nxu, Ny, Nz)); V = np.zeros((Nx, Ny + 1, Nz))
    for k in range(Nz):
        psi = psi2 * prof[k]
        U[:, :, k] = -(psi[:nxu, 1:] - psi[:nxu, :-1])
        V[:, :, k] = psi[1:, :] - psi[:-1, :]
    Ax = grid.Ax[Hx:Hx + nxu, Hy:Hy + Ny, Hz:Hz + Nz]
    Ay = grid.Ay[Hx:Hx + Nx, Hy:Hy + Ny + 1, Hz:Hz + Nz]
    u, v = U / Ax, V / Ay
    dxc = grid.dxC[Hx:Hx + nxu, Hy:Hy + Ny][:, :, None]
    dyc = grid.dyC[Hx:Hx + Nx, Hy:Hy + Ny + 1][:, :, None]
    s = cfl / max(np.max(np.abs(u) * dT / dxc), np.max(np.abs(v) * dT / dyc))
    w = np.zeros((Nx, Ny, Nz + 1))
    return np.asfortranarray(u * s), np.asfortranarray(v * s), np.asfortranarray(w)


def latlon(nx=24, ny=20, nz=6, lon=(-10.0, -7.6), lat=(30.0, 32.0), dz=10.0, N_per_species=3000, nsp=2,
           steps=20, dT=600.0, seed=12, capacity=None, phyt_over=None, bgc_over=None, landmask=None, cfl=0.2):
    """QuotaMode on a LatLonGrid (src/Grids/lat_lon_grid.jl): nx×ny×nz cells over `lon` × `lat`
    degrees and nz levels of dz metres, individuals seeded in the top half, a steady
    divergence-free transport streamfunction flow (latlon_streamfunction_velocity)."""
    rng = np.random.default_rng(seed)
    grid = LatLonGrid(size=(nx, ny, nz), lat=lat, lon=lon, z=(0.0, -dz * nz), FT=np.float64, landmask=landmask)
    u, v, w = latlon_streamfunction_velocity(grid, cfl=cfl, dT=dT, seed=seed)
    C = capacity or 2 * N_per_species
    return _finish("latlon", grid, nsp, [N_per_species] * nsp, C, phyt_over, bgc_over, dT, steps, rng,
                   lambda t: (u, v, w), 1, dT * steps, max(1, nz // 2), [0.0] * nsp, 0.2, seed,
                   no3_grad=dz * nz)


def config3(nx=512, nz=128, N_per_species=16_777_216, nsp=4, steps=1000, dT=20.0, seed=3,
            nmodes=256, capacity=None):
    """Mixed precision at scale (nx×nx×nz), 4 species with their own size distributions."""
    rng = np.random.default_rng(seed)
    grid = RectilinearGrid(size=(nx, nx, nz), x=(0.0, nx * 50.0), y=(0.0, nx * 50.0),
                           z=(0.0, -2.0 * nz), FT=np.float64, topology=(Periodic, Periodic, Bounded))
    vel = FourierVelocity(grid, nmodes=nmodes, rms=0.05, seed=seed)
    C = capacity or 2 * N_per_species
    mus = [-0.5, 0.0, 0.5, 1.0][:nsp]
    n_vel = int(np.ceil(steps / 60)) + 1
    return _finish("config3", grid, nsp, [N_per_species] * nsp, C, None, None, dT, steps, rng,
                   vel, n_vel, 60 * dT, min(nz, 20), mus, 0.25, seed, no3_grad=2.0 * nz)


def config4(n_members=64, steps=500, dT=30.0, seed=4, nmodes=32, n_max=None):
    """Batched ensemble: members with grids Nx, Ny ~ U{64..256}, Nz ~ U{16..32} (50 m × 50 m × 2 m
    cells), populations round(2^U(14, 20)) of one species, config-2 physics (random-Fourier velocity
    refreshed every 60 steps, NO3 gradient, individuals in the top 40 m) and their own seeds.
    `nmodes` Fourier modes per member (fewer than config 2's 256 to keep host generation short;
    the device work does not depend on it). `n_max` caps the member count for tests."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n_members if n_max is None else min(n_members, n_max)):
        nx, ny = int(rng.integers(64, 257)), int(rng.integers(64, 257))
        nz = int(rng.integers(16, 33))
        N = int(round(2.0 ** rng.uniform(14, 20)))
        ms = seed * 1000 + m
        r = np.random.default_rng(ms)
        grid = RectilinearGrid(size=(nx, ny, nz), x=(0.0, nx * 50.0), y=(0.0, ny * 50.0),
                               z=(0.0, -2.0 * nz), FT=np.float64, topology=(Periodic, Periodic, Bounded))
        vel = FourierVelocity(grid, nmodes=nmodes, rms=0.05, seed=ms)
        n_vel = int(np.ceil(steps / 60)) + 1
        wl = _finish(f"config4[{m}]", grid, 1, [N], 2 * N, None, None, dT, steps, r, vel, n_vel, 60 * dT,
                     min(nz, 20), [0.0], 0.2, ms, no3_grad=2.0 * nz)
        out.append(wl)
    return out


def config5(n_boxes=4096, steps=2880, dT=60.0, seed=5, n_max=None):
    """Batched 0D boxes (examples/0D_experiment.jl:35): 1×1×1 cells of 128 m × 128 m × 128 m, no
    advection (zero velocity), populations round(2^U(8, 13)), light with a per-box phase offset
    φ ~ U(0, 86400 s). Division by size with dvid_reg = 1.0 and dvid_P = 1.2e-5 s⁻¹ (≈ 1 d⁻¹ for
    cells at nominal size); nitrate and ammonium start at 0.01 mmol m⁻³ (near their half-saturation
    constants), so growth is nutrient-limited. Capacity 8 × the initial population."""
    rng = np.random.default_rng(seed)
    out = []
    over = {"dvid_reg": [1.0], "dvid_P": [1.2e-5]}
    for b in range(n_boxes if n_max is None else min(n_boxes, n_max)):
        N = int(round(2.0 ** rng.uniform(8, 13)))
        phase = float(rng.uniform(0.0, 86400.0))
        ms = seed * 100000 + b
        r = np.random.default_rng(ms)
        grid = RectilinearGrid(size=(1, 1, 1), x=(0.0, 128.0), y=(0.0, 128.0), z=(0.0, -128.0),
                               FT=np.float64, topology=(Periodic, Periodic, Bounded))
        zero = (np.zeros((1, 1, 1), order="F"), np.zeros((1, 1, 1), order="F"), np.zeros((1, 1, 2), order="F"))
        wl = _finish(f"config5[{b}]", grid, 1, [N], 8 * N, over, None, dT, steps, r, lambda t: zero, 1,
                     dT * steps, None, [0.0], 0.2, ms)
        for name in ("NO3", "NH4"):
            a = wl.tracers[tracer_names.index(name)]
            a[...] = 0.01
        hours = wl.parf.shape[2]
        wl.parf = diel_parf(1, 1, hours, peak=1000.0, phase=phase)
        out.append(wl)
    return out


def abiotic(nx=16, nz=8, N_per_species=1500, nsp=2, N_abiotic=(2000, 1000), steps=20, dT=60.0, seed=17,
            nmodes=16, capacity=None, Rd=(12.0, 20.0), release_P=(2.0e-3, 1.0e-3), max_ptc=(25.0, 2.0),
            top_flux=2.0e-9, max_candidates=25, topology=None):
    """QuotaMode with abiotic particles on a config-2-like 3D grid (nx×nx×nz, 50 m × 50 m × 2 m):
    two abiotic species from initialize_abiotic_particle!, interaction pairs (sp1, sa1) and
    (sp2, sa2), release pair (sp1, sa1), particle fluxes into sa2 through the top (constant), the
    east face (a face array) and the south face (a time series). Interaction radii and release
    probabilities are raised from the defaults (Rd = 1e-4 m) so that merges and releases happen
    every step; max_ptc is given per phytoplankton species as IronEnergyMode's parameter would be.
    The abiotic setup is in `wl.abiotic` (see configure_abiotics)."""
    from .init import initialize_abiotic_particle
    rng = np.random.default_rng(seed)
    topology = topology or (Periodic, Periodic, Bounded)
    grid = RectilinearGrid(size=(nx, nx, nz), x=(0.0, nx * 50.0), y=(0.0, nx * 50.0),
                           z=(0.0, -2.0 * nz), FT=np.float64, topology=topology)
    vel = FourierVelocity(grid, nmodes=nmodes, rms=0.05, seed=seed)
    C = capacity or 2 * N_per_species
    n_vel = int(np.ceil(steps / 60)) + 1
    vel_fn = vel
    if grid.topo[0] == Bounded.code or grid.topo[1] == Bounded.code:
        def vel_fn(t, _v=vel, _bx=grid.topo[0] == Bounded.code, _by=grid.topo[1] == Bounded.code):
            u, v, w = _v(t)                  # the periodic field, its first face repeated on Bounded axes
            if _bx:
                u = np.asfortranarray(np.concatenate([u, u[:1]], axis=0))
            if _by:
                v = np.asfortranarray(np.concatenate([v, v[:, :1]], axis=1))
            return u, v, w
    wl = _finish("abiotic", grid, nsp, [N_per_species] * nsp, C, None, None, dT, steps, rng, vel_fn, n_vel, 60 * dT,
                 nz, [0.0] * nsp, 0.2, seed, no3_grad=2.0 * nz)
    nsa = len(N_abiotic)
    params = {"Nsuper": [1.0] * nsa, "Rd": list(Rd)[:nsa], "release_P": list(release_P)[:nsa],
              "sz_min": [1.0e-3] * nsa, "Ktr": [0.0] * nsa}
    from ._abi import FACES, PI_BC_ARRAY2D, PI_BC_ARRAY3D, PI_BC_CONST
    sa_bc = min(1, nsa - 1)
    bcs = [(sa_bc, FACES["top"], PI_BC_CONST, [top_flux], 0),
           (sa_bc, FACES["east"], PI_BC_ARRAY2D, np.asfortranarray(rng.random((grid.Ny, grid.Nz)) * 5.0e-8), 0),
           (sa_bc, FACES["south"], PI_BC_ARRAY3D, np.asfortranarray(rng.random((grid.Nx, grid.Nz, steps + 1)) * 5.0e-8),
            steps + 1)]
    wl.abiotic = dict(params=params, nsa=nsa,
                      intac=[(s, min(s, nsa - 1)) for s in range(nsp)], release=[(0, 0)],
                      max_candidates=max_candidates, max_ptc=list(max_ptc)[:nsp],
                      particles=[initialize_abiotic_particle(grid, N_abiotic[a], C, rng) for a in range(nsa)],
                      bcs=bcs)
    return wl


def configure_abiotics(model, wl):
    """Applies `wl.abiotic` to a model handle (the oracle's or the library's)."""
    a = wl.abiotic
    model.set_abiotics(a["params"], a["nsa"], a["intac"], a["release"], a["max_candidates"], a["max_ptc"])
    for s, d in enumerate(a["particles"]):
        model.set_abiotic_particles(s, d)
    for (sa, face, kind, values, nt) in a["bcs"]:
        model.set_abiotic_bc(sa, face, kind, values, nt)
    return model
