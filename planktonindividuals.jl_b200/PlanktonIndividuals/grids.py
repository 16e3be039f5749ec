"""RectilinearGrid and halo rules, host side (src/Grids/rectilinear_grid.jl, src/Grids/utils.jl,
src/Biogeochemistry/HaloRegions/halo_regions.jl).

Arrays use Julia's column-major order: a grid field is a numpy array of shape (Gx, Gy, Gz) in
Fortran order, so `a[i-1, j-1, k-1]` is the reference's `a[i, j, k]` and the raw memory matches
what the C ABI expects.
"""
from fractions import Fraction

import numpy as np

from ._abi import PI_BOUNDED, PI_PERIODIC


class Periodic:
    """Periodic topology (src/Grids/Grids.jl)."""
    code = PI_PERIODIC


class Bounded:
    """Bounded topology (src/Grids/Grids.jl)."""
    code = PI_BOUNDED


def _topo_code(T):
    if T is Periodic or isinstance(T, Periodic):
        return PI_PERIODIC
    if T is Bounded or isinstance(T, Bounded):
        return PI_BOUNDED
    raise ValueError(f"{T} is not a valid topology!Valid topologies are: Periodic and Bounded.")


def _linspace_exact(a, b, n):
    """collect(range(a, b, length=n)) for Float64: each point is the correctly rounded value of
    a + (i-1)(b-a)/(n-1) computed exactly (Julia's ranges carry extended precision)."""
    fa, fb = Fraction(float(a)), Fraction(float(b))
    if n == 1:
        return np.array([float(fa)])
    return np.array([float(fa + (fb - fa) * i / (n - 1)) for i in range(n)], dtype=np.float64)


class RectilinearGrid:
    """RectilinearGrid(; size, x, y, z, FT, topology, landmask, halo)
    (src/Grids/rectilinear_grid.jl:57-122). x and y are uniform, z is a 2-tuple or the Nz+1
    face positions (surface first, negative downward)."""

    def __init__(self, *, size, x, y, z, FT=np.float32, topology=(Periodic, Periodic, Bounded),
                 landmask=None, halo=(2, 2, 2)):
        Nx, Ny, Nz = (int(v) for v in size)
        Hx, Hy, Hz = (int(v) for v in halo)
        self.topology = tuple(topology)
        self.topo = tuple(_topo_code(T) for T in topology)
        assert isinstance(x, tuple) and len(x) == 2
        assert isinstance(y, tuple) and len(y) == 2
        x1, x2 = x
        y1, y2 = y
        assert x1 < x2
        assert y1 < y2
        FT = np.dtype(FT).type
        self.FT = FT
        dx = (x2 - x1) / Nx
        dy = (y2 - y1) / Ny
        self.Δx = float(FT(dx))
        self.Δy = float(FT(dy))
        self.xF = _linspace_exact(-Hx * dx, (Nx + Hx - 1) * dx, Nx + 2 * Hx).astype(FT)
        self.yF = _linspace_exact(-Hy * dy, (Ny + Hy - 1) * dy, Ny + 2 * Hy).astype(FT)
        self.xC = _linspace_exact((0.5 - Hx) * dx, (Nx + Hx - 0.5) * dx, Nx + 2 * Hx).astype(FT)
        self.yC = _linspace_exact((0.5 - Hy) * dy, (Ny + Hy - 0.5) * dy, Ny + 2 * Hy).astype(FT)
        if isinstance(z, tuple) and len(z) == 2:
            z1, z2 = z
            zf = _linspace_exact(z1, z2, Nz + 1).astype(FT)
        elif hasattr(z, "__len__"):
            zf = np.asarray(z, dtype=FT)
            z1, z2 = zf[0], zf[-1]
        else:
            raise ValueError("z must be a 2-tuple or 1D array")
        assert z1 > z2
        assert len(zf) == Nz + 1
        zF = np.zeros(Nz + 2 * Hz, dtype=FT)
        zC = np.zeros(Nz + 2 * Hz, dtype=FT)
        dzF = np.zeros(Nz + 2 * Hz, dtype=FT)
        dzC = np.zeros(Nz + 2 * Hz, dtype=FT)
        # 0-based views of the reference's 1-based ranges
        zF[Hz:Nz + Hz + 1] = zf
        zC[Hz:Nz + Hz] = (zF[Hz:Nz + Hz] + zF[Hz + 1:Nz + Hz + 1]) / FT(2.0)
        dzF[Hz:Nz + Hz] = zF[Hz:Nz + Hz] - zF[Hz + 1:Nz + Hz + 1]
        dzC[Hz:Nz + Hz - 1] = zC[Hz:Nz + Hz - 1] - zC[Hz + 1:Nz + Hz]
        dzF[0:Hz] = dzF[Hz]
        dzC[0:Hz] = dzF[Hz]
        dzF[Nz + Hz:Nz + 2 * Hz] = dzF[Nz + Hz - 1]
        dzC[Nz + Hz - 1:Nz + 2 * Hz] = dzF[Nz + Hz - 1]
        zF[0:Hz] = zF[Hz:2 * Hz] + dzF[0] * Hz
        if Hz >= 2:
            zF[Nz + Hz + 1:Nz + 2 * Hz] = zF[Nz + 1:Nz + Hz] - dzF[-1] * Hz
        for i in range(1, Hz + 1):
            zC[Nz + Hz + i - 1] = zC[Nz + Hz + i - 2] - dzF[-1]
        for i in range(Hz, 0, -1):
            zC[i - 1] = zC[i] + dzF[0]
        self.zF, self.zC, self.dzF, self.dzC = zF, zC, dzF, dzC
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.Hx, self.Hy, self.Hz = Hx, Hy, Hz
        self.landmask = landmask_validation(landmask, Nx, Ny, Nz, Hx, Hy, Hz, self.topo[0], self.topo[1])

    @property
    def size(self):
        return (self.Nx, self.Ny, self.Nz)

    @property
    def total_size(self):
        return (self.Nx + 2 * self.Hx, self.Ny + 2 * self.Hy, self.Nz + 2 * self.Hz)

    def __repr__(self):
        t = tuple("Periodic" if c == PI_PERIODIC else "Bounded" for c in self.topo)
        return (f"RegularRectilinearGrid{{{np.dtype(self.FT).name}, {t[0]}, {t[1]}, {t[2]}}}"
                f"(Nx={self.Nx}, Ny={self.Ny}, Nz={self.Nz})")


def landmask_validation(landmask, Nx, Ny, Nz, Hx, Hy, Hz, TX, TY):
    """src/Grids/utils.jl:92-129: land mask with halos (Bool, shape (Gx, Gy, Gz))."""
    if landmask is None:
        landmask = np.ones((Nx, Ny, Nz), dtype=bool)
    else:
        landmask = np.asarray(landmask)
        if landmask.dtype != np.bool_ or landmask.ndim != 3:
            raise ValueError("landmask: type mismatch, typeof(landmask) must be Array{Bool, 3}.")
        if landmask.shape != (Nx, Ny, Nz):
            raise ValueError("landmask: grid mismatch, size(landmask) must equal to (grid.Nx, grid.Ny, grid.Nz).")
    lh = np.zeros((Nx + 2 * Hx, Ny + 2 * Hy, Nz + 2 * Hz), dtype=bool, order="F")
    lh[Hx:Hx + Nx, Hy:Hy + Ny, Hz:Hz + Nz] = landmask
    if TX == PI_PERIODIC:
        lh[0:Hx] = lh[Nx:Nx + Hx].copy()
        lh[Nx + Hx:Nx + 2 * Hx] = lh[Hx:2 * Hx].copy()
    else:
        lh[0:Hx] = lh[Hx:Hx + 1].copy()
        lh[Nx + Hx:Nx + 2 * Hx] = lh[Nx + Hx - 1:Nx + Hx].copy()
    if TY == PI_PERIODIC:
        lh[:, 0:Hy] = lh[:, Ny:Ny + Hy].copy()
        lh[:, Ny + Hy:Ny + 2 * Hy] = lh[:, Hy:2 * Hy].copy()
    else:
        lh[:, 0:Hy] = lh[:, Hy:Hy + 1].copy()
        lh[:, Ny + Hy:Ny + 2 * Hy] = lh[:, Ny + Hy - 1:Ny + Hy].copy()
    lh[:, :, 0:Hz] = lh[:, :, Hz:Hz + 1].copy()
    lh[:, :, Nz + Hz:Nz + 2 * Hz] = lh[:, :, Nz + Hz - 1:Nz + Hz].copy()
    return lh


# Grid metrics with 1-based halo-inclusive indices (src/Grids/areas_volumes_spacings.jl:9-22)
def ΔxC(i, j, k, g): return g.Δx
def ΔyC(i, j, k, g): return g.Δy
def ΔzC(i, j, k, g): return g.dzC[k - 1]
def ΔxF(i, j, k, g): return g.Δx
def ΔyF(i, j, k, g): return g.Δy
def ΔzF(i, j, k, g): return g.dzF[k - 1]
def Ax(i, j, k, g): return g.Δy * g.dzF[k - 1]
def Ay(i, j, k, g): return g.Δx * g.dzF[k - 1]
def Az(i, j, k, g): return g.Δx * g.Δy
def volume(i, j, k, g): return g.Δx * g.Δy * g.dzF[k - 1]


# ---- halo rules (halo_regions.jl:2-62); each fill reads its source before writing -----------

def _face(c, axis, lo, N, H, topo, rule="tracer"):
    sl = [slice(None)] * 3

    def put(dst, src_vals):
        s = list(sl); s[axis] = dst; c[tuple(s)] = src_vals

    def get(src):
        s = list(sl); s[axis] = src; return c[tuple(s)].copy()

    if lo:
        if topo == PI_PERIODIC:
            put(slice(0, H), get(slice(N, N + H)))
        else:
            put(slice(0, H), get(slice(H, H + 1)))
    else:
        if rule == "vel" and topo == PI_BOUNDED:
            put(slice(N + H + 1, N + 2 * H), get(slice(N + H, N + H + 1)))
        elif rule == "Gc" and topo == PI_BOUNDED:
            put(slice(N + H, N + 2 * H), 0.0)
        elif topo == PI_PERIODIC:
            put(slice(N + H, N + 2 * H), get(slice(H, 2 * H)))
        else:
            put(slice(N + H, N + 2 * H), get(slice(N + H - 1, N + H)))


def fill_halo_west_east(c, g, rule="tracer"):
    _face(c, 0, True, g.Nx, g.Hx, g.topo[0])
    _face(c, 0, False, g.Nx, g.Hx, g.topo[0], rule)


def fill_halo_tracer(c, g):
    """fill_halo_tracer! for one field (halo_regions.jl:37-47)."""
    for ax, N, H in ((0, g.Nx, g.Hx), (1, g.Ny, g.Hy), (2, g.Nz, g.Hz)):
        _face(c, ax, True, N, H, g.topo[ax])
        _face(c, ax, False, N, H, g.topo[ax])
    return c


def fill_halo_vel(u, v, w, g):
    """fill_halo_vel! (halo_regions.jl:64-99)."""
    _face(u, 0, False, g.Nx, g.Hx, g.topo[0], "vel")
    _face(u, 0, True, g.Nx, g.Hx, g.topo[0])
    for ax, N, H in ((1, g.Ny, g.Hy), (2, g.Nz, g.Hz)):
        _face(u, ax, True, N, H, g.topo[ax]); _face(u, ax, False, N, H, g.topo[ax])
    _face(v, 1, False, g.Ny, g.Hy, g.topo[1], "vel")
    _face(v, 0, True, g.Nx, g.Hx, g.topo[0]); _face(v, 0, False, g.Nx, g.Hx, g.topo[0])
    _face(v, 1, True, g.Ny, g.Hy, g.topo[1])
    _face(v, 2, True, g.Nz, g.Hz, g.topo[2]); _face(v, 2, False, g.Nz, g.Hz, g.topo[2])
    _face(w, 2, False, g.Nz, g.Hz, g.topo[2], "vel")
    _face(w, 0, True, g.Nx, g.Hx, g.topo[0]); _face(w, 0, False, g.Nx, g.Hx, g.topo[0])
    _face(w, 1, True, g.Ny, g.Hy, g.topo[1]); _face(w, 1, False, g.Ny, g.Hy, g.topo[1])
    _face(w, 2, True, g.Nz, g.Hz, g.topo[2])


def fill_halo_Gc(c, g):
    """fill_halo_Gcs! for one field (halo_regions.jl:49-56)."""
    for ax, N, H in ((0, g.Nx, g.Hx), (1, g.Ny, g.Hy), (2, g.Nz, g.Hz)):
        _face(c, ax, False, N, H, g.topo[ax], "Gc")
    return c


def interior(c, g):
    """interior(c, grid) (tracer_fields.jl:16)."""
    return c[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz]
