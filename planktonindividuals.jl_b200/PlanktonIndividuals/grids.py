"""RectilinearGrid, LatLonGrid and halo rules, host side (src/Grids/rectilinear_grid.jl,
src/Grids/lat_lon_grid.jl, src/Grids/utils.jl, src/Biogeochemistry/HaloRegions/halo_regions.jl).

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
        self.zF, self.zC, self.dzF, self.dzC = _z_axis(z, Nz, Hz, FT)
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


class LatLonGrid:
    """LatLonGrid(; size, lat, lon, z, FT, radius, landmask, halo) (src/Grids/lat_lon_grid.jl:57-170).
    lat and lon are 2-tuples in degrees (−80 ≤ lat ≤ 80, −180 ≤ lon ≤ 180), z as for
    RectilinearGrid. x is Periodic when lon spans −180..180, Bounded otherwise; y and z are
    Bounded. Spacings dxC, dyC, dxF, dyF and the face area Az are (Gx, Gy) arrays, Ax, Ay and
    Vol (Gx, Gy, Gz) arrays, in metres, halos included; the model reads them through the C ABI's
    pi_grid_metrics (FP64 form)."""

    is_latlon = True

    def __init__(self, *, size, lat, lon, z, FT=np.float32, radius=6370.0e3, landmask=None, halo=(2, 2, 2)):
        Nx, Ny, Nz = (int(v) for v in size)
        Hx, Hy, Hz = (int(v) for v in halo)
        lat1, lat2 = lat
        lon1, lon2 = lon
        FT = np.dtype(FT).type
        self.FT = FT
        zF, zC, dzF, dzC = _z_axis(z, Nz, Hz, FT)
        assert -180 <= lon1 < lon2 <= 180
        assert -80 <= lat1 < lat2 <= 80
        TX = Periodic if (lon1 == -180 and lon2 == 180) else Bounded
        self.topology = (TX, Bounded, Bounded)
        self.topo = tuple(_topo_code(T) for T in self.topology)
        dlon = (lon2 - lon1) / Nx
        dlat = (lat2 - lat1) / Ny
        self.Δx, self.Δy = float(FT(dlon)), float(FT(dlat))
        self.xF = _linspace_exact(lon1 - Hx * dlon, lon1 + (Nx + Hx - 1) * dlon, Nx + 2 * Hx).astype(FT)
        self.yF = _linspace_exact(lat1 - Hy * dlat, lat1 + (Ny + Hy - 1) * dlat, Ny + 2 * Hy).astype(FT)
        self.xC = _linspace_exact(lon1 + (0.5 - Hx) * dlon, lon1 + (Nx + Hx - 0.5) * dlon, Nx + 2 * Hx).astype(FT)
        self.yC = _linspace_exact(lat1 + (0.5 - Hy) * dlat, lat1 + (Ny + Hy - 0.5) * dlat, Ny + 2 * Hy).astype(FT)
        self.zF, self.zC, self.dzF, self.dzC = zF, zC, dzF, dzC
        Gx, Gy, Gz = Nx + 2 * Hx, Ny + 2 * Hy, Nz + 2 * Hz
        # degree to metre (lat_lon_grid.jl:141-163): deg2rad(x) = x·(π/180); cos(y·π/180)
        d2r = lambda x: x * (np.pi / 180)
        r = float(radius)
        cy = np.array([np.cos(float(y) * np.pi / 180) for y in self.yC])
        sy = np.array([np.sin(float(y) * np.pi / 180) for y in self.yF])
        dxc = np.empty((Gx, Gy), dtype=FT, order="F")
        dxc[:, :] = (r * cy * d2r(dlon))[None, :]
        dyc = np.full((Gx, Gy), FT(r * d2r(dlat)), dtype=FT, order="F")
        self.dxC, self.dyC = dxc, dyc
        self.dxF, self.dyF = dxc.copy(order="F"), dyc.copy(order="F")
        Az = np.zeros((Gx, Gy), dtype=FT, order="F")
        Az[:Gx - 1, :Gy - 1] = ((r * r) * d2r(dlon) * (sy[1:] - sy[:-1]))[None, :]
        Az[Gx - 1, :] = Az[Gx - 2, :]              # the corner (Gx, Gy) keeps the 0 of row Gy
        Az[:Gx - 1, Gy - 1] = Az[:Gx - 1, Gy - 2]
        self.Az = Az
        self.Ax = np.asfortranarray(dzF[None, None, :] * self.dyF[:, :, None]).astype(FT)
        self.Ay = np.asfortranarray(dzF[None, None, :] * self.dxF[:, :, None]).astype(FT)
        self.Vol = np.asfortranarray(self.Az[:, :, None] * dzF[None, None, :]).astype(FT)
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.Hx, self.Hy, self.Hz = Hx, Hy, Hz
        self.landmask = landmask_validation(landmask, Nx, Ny, Nz, Hx, Hy, Hz, self.topo[0], self.topo[1])

    size = RectilinearGrid.size
    total_size = RectilinearGrid.total_size

    def __repr__(self):
        t = tuple("Periodic" if c == PI_PERIODIC else "Bounded" for c in self.topo)
        return (f"LatLonGrid{{{np.dtype(self.FT).name}, {t[0]}, {t[1]}, {t[2]}}}"
                f"(Nx={self.Nx}, Ny={self.Ny}, Nz={self.Nz})")


def LoadLatLonGrid(*, grid_info, size, lat, lon, FT=np.float32, landmask=None, halo=(2, 2, 2)):
    """LoadLatLonGrid(; grid_info, size, lat, lon, FT, landmask, halo)
    (src/Grids/lat_lon_grid.jl:196-316): a LatLonGrid whose metrics come from an external model
    grid. grid_info maps RF, RC, DRF, DRC (vertical), DXC, DXG, DYC, DYG, RAC (Nx×Ny) and hFacC,
    hFacW, hFacS (Nx×Ny×Nz) to arrays, as MITgcm names them."""
    Nx, Ny, Nz = (int(v) for v in size)
    Hx, Hy, Hz = (int(v) for v in halo)
    lat1, lat2 = lat
    lon1, lon2 = lon
    assert -180 <= lon1 < lon2 <= 180
    assert -80 <= lat1 < lat2 <= 80
    FT = np.dtype(FT).type
    g = LatLonGrid.__new__(LatLonGrid)
    g.FT = FT
    TX = Periodic if (lon1 == -180 and lon2 == 180) else Bounded
    g.topology = (TX, Bounded, Bounded)
    g.topo = tuple(_topo_code(T) for T in g.topology)
    dlon, dlat = (lon2 - lon1) / Nx, (lat2 - lat1) / Ny
    g.Δx, g.Δy = float(FT(dlon)), float(FT(dlat))
    g.xF = _linspace_exact(lon1 - Hx * dlon, lon1 + (Nx + Hx - 1) * dlon, Nx + 2 * Hx).astype(FT)
    g.yF = _linspace_exact(lat1 - Hy * dlat, lat1 + (Ny + Hy - 1) * dlat, Ny + 2 * Hy).astype(FT)
    g.xC = _linspace_exact(lon1 + (0.5 - Hx) * dlon, lon1 + (Nx + Hx - 0.5) * dlon, Nx + 2 * Hx).astype(FT)
    g.yC = _linspace_exact(lat1 + (0.5 - Hy) * dlat, lat1 + (Ny + Hy - 0.5) * dlat, Ny + 2 * Hy).astype(FT)
    Gx, Gy, Gz = Nx + 2 * Hx, Ny + 2 * Hy, Nz + 2 * Hz
    gi = {k: np.asarray(v) for k, v in dict(grid_info).items()}
    zF = np.zeros(Gz, dtype=FT); zC = np.zeros(Gz, dtype=FT)
    dzF = np.zeros(Gz, dtype=FT); dzC = np.zeros(Gz, dtype=FT)
    zF[Hz:Nz + Hz + 1] = gi["RF"].astype(FT)
    zC[Hz:Nz + Hz] = gi["RC"].astype(FT)
    dzF[Hz:Nz + Hz] = gi["DRF"].astype(FT)
    dzC[Hz:Nz + Hz] = gi["DRC"].astype(FT)[:Nz]
    dzC[Hz] *= FT(2.0)                       # the first layer only has half of the grid
    arr2 = {}
    for name, key in (("dxC", "DXC"), ("dxF", "DXG"), ("dyC", "DYC"), ("dyF", "DYG"), ("Az", "RAC")):
        a = np.zeros((Gx, Gy), dtype=FT, order="F")
        a[Hx:Nx + Hx, Hy:Ny + Hy] = gi[key].astype(FT)
        arr2[name] = a
    hf = {}
    for name, key in (("hFW", "hFacW"), ("hFS", "hFacS"), ("hFC", "hFacC")):
        a = np.ones((Gx, Gy, Gz), dtype=FT, order="F")
        a[Hx:Nx + Hx, Hy:Ny + Hy, Hz:Nz + Hz] = gi[key].astype(FT)
        hf[name] = a
    dzF[0:Hz] = dzF[Hz]; dzC[0:Hz] = dzC[Hz]
    dzF[Nz + Hz:] = dzF[Nz + Hz - 1]; dzC[Nz + Hz:] = dzC[Nz + Hz - 1]
    zF[0:Hz] = zF[Hz:2 * Hz] + dzF[0] * 2
    zC[0:Hz] = zC[Hz:2 * Hz] + dzC[0] * 2
    zF[Nz + Hz + 1:Nz + 2 * Hz] = zF[Nz + 1:Nz + Hz] - dzF[-1] * 2
    zC[Nz + Hz:Nz + 2 * Hz] = zC[Nz:Nz + Hz] - dzC[-1] * 2
    for a in arr2.values():
        if g.topo[0] == PI_PERIODIC:
            a[0:Hx, :] = a[Nx:Nx + Hx, :]; a[Nx + Hx:, :] = a[Hx:2 * Hx, :]
        else:
            a[0:Hx, :] = a[Hx:Hx + 1, :]; a[Nx + Hx:, :] = a[Nx + Hx - 1:Nx + Hx, :]
        a[:, 0:Hy] = a[:, Hy:Hy + 1]; a[:, Ny + Hy:] = a[:, Ny + Hy - 1:Ny + Hy]
    for a in hf.values():
        if g.topo[0] == PI_PERIODIC:
            a[0:Hx] = a[Nx:Nx + Hx]; a[Nx + Hx:] = a[Hx:2 * Hx]
        else:
            a[0:Hx] = a[Hx:Hx + 1]; a[Nx + Hx:] = a[Nx + Hx - 1:Nx + Hx]
        a[:, 0:Hy] = a[:, Hy:Hy + 1]; a[:, Ny + Hy:] = a[:, Ny + Hy - 1:Ny + Hy]
        a[:, :, 0:Hz] = a[:, :, Hz:Hz + 1]; a[:, :, Nz + Hz:] = a[:, :, Nz + Hz - 1:Nz + Hz]
    g.zF, g.zC, g.dzF, g.dzC = zF, zC, dzF, dzC
    g.dxC, g.dxF, g.dyC, g.dyF, g.Az = arr2["dxC"], arr2["dxF"], arr2["dyC"], arr2["dyF"], arr2["Az"]
    g.Ax = np.asfortranarray(dzF[None, None, :] * g.dyF[:, :, None] * hf["hFW"]).astype(FT)
    g.Ay = np.asfortranarray(dzF[None, None, :] * g.dxF[:, :, None] * hf["hFS"]).astype(FT)
    g.Vol = np.asfortranarray(dzF[None, None, :] * g.Az[:, :, None] * hf["hFC"]).astype(FT)
    g.Nx, g.Ny, g.Nz = Nx, Ny, Nz
    g.Hx, g.Hy, g.Hz = Hx, Hy, Hz
    g.landmask = landmask_validation(landmask, Nx, Ny, Nz, Hx, Hy, Hz, g.topo[0], g.topo[1])
    return g


def _z_axis(z, Nz, Hz, FT):
    """Vertical faces, centers and spacings with halos, as both grid constructors build them
    (rectilinear_grid.jl:82-111, lat_lon_grid.jl:105-139)."""
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
    return zF, zC, dzF, dzC


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


# Grid metrics with 1-based halo-inclusive indices (src/Grids/areas_volumes_spacings.jl:9-38):
# a RectilinearGrid forms them from Δx, Δy and dzF, a LatLonGrid reads its arrays
def _ll(g): return getattr(g, "is_latlon", False)
def ΔxC(i, j, k, g): return g.dxC[i - 1, j - 1] if _ll(g) else g.Δx
def ΔyC(i, j, k, g): return g.dyC[i - 1, j - 1] if _ll(g) else g.Δy
def ΔzC(i, j, k, g): return g.dzC[k - 1]
def ΔxF(i, j, k, g): return g.dxF[i - 1, j - 1] if _ll(g) else g.Δx
def ΔyF(i, j, k, g): return g.dyF[i - 1, j - 1] if _ll(g) else g.Δy
def ΔzF(i, j, k, g): return g.dzF[k - 1]
def Ax(i, j, k, g): return g.Ax[i - 1, j - 1, k - 1] if _ll(g) else g.Δy * g.dzF[k - 1]
def Ay(i, j, k, g): return g.Ay[i - 1, j - 1, k - 1] if _ll(g) else g.Δx * g.dzF[k - 1]
def Az(i, j, k, g): return g.Az[i - 1, j - 1] if _ll(g) else g.Δx * g.Δy
def volume(i, j, k, g): return g.Vol[i - 1, j - 1, k - 1] if _ll(g) else g.Δx * g.Δy * g.dzF[k - 1]


def cell_volumes(g):
    """volume(i, j, k, g) for every halo-inclusive cell, shape (Gx, Gy, Gz) in Fortran order."""
    if _ll(g):
        return np.asfortranarray(g.Vol, dtype=np.float64)
    Gx, Gy, _ = g.total_size
    return np.asfortranarray(np.broadcast_to((g.Δx * g.Δy) * np.asarray(g.dzF, dtype=np.float64), (Gx, Gy, len(g.dzF))))


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
