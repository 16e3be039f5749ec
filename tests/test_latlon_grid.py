"""LatLonGrid (src/Grids/lat_lon_grid.jl) on the host and in the CPU oracle: the reference's grid
tests (test/grid_test.jl:69-135) re-run against the host grid, the metric identities of the
constructor, the loader of external grids, and a phosphorus budget that closes to rounding when the
flow is divergence-free in the grid's own face areas."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import (Bounded, LatLonGrid, LoadLatLonGrid, Periodic, Ax, Ay, Az, volume, ΔxC,
                                 ΔxF, ΔyC, ΔyF, ΔzC, ΔzF)
from PlanktonIndividuals import _abi
from PlanktonIndividuals import grids as G
from PlanktonIndividuals import workloads as W


def test_lat_lon_grid():                             # grid_test.jl:69-82
    grid = LatLonGrid(size=(360, 160, 10), lat=(-80, 80), lon=(-180, 180), z=(0, -20))
    assert (grid.Nx, grid.Ny, grid.Nz) == (360, 160, 10)
    for a, n in ((grid.xC, 360), (grid.yC, 160), (grid.zC, 10), (grid.xF, 360), (grid.yF, 160), (grid.zF, 10)):
        assert len(a) == n + 2 * 2
    assert grid.topology == (Periodic, Bounded, Bounded)
    assert "LatLonGrid" in repr(grid)


def test_lat_lon_areas_volumes():                    # grid_test.jl:115-131
    grid = LatLonGrid(size=(360, 160, 10), lat=(-80, 80), lon=(-180, 180), z=(0, -20))
    assert ΔxC(1, 1, 1, grid) == grid.dxC[0, 0]
    assert ΔyC(1, 1, 1, grid) == grid.dyC[0, 0]
    assert ΔzC(1, 1, 1, grid) == grid.dzC[0]
    assert ΔxF(1, 1, 1, grid) == grid.dxF[0, 0]
    assert ΔyF(1, 1, 1, grid) == grid.dyF[0, 0]
    assert ΔzF(1, 1, 1, grid) == grid.dzF[0]
    assert Ax(1, 1, 1, grid) == grid.Ax[0, 0, 0]
    assert Ay(1, 1, 1, grid) == grid.Ay[0, 0, 0]
    assert Az(1, 1, 1, grid) == grid.Az[0, 0]
    assert volume(1, 1, 1, grid) == grid.Vol[0, 0, 0]


def test_lat_lon_metric_identities():
    """The constructor's formulas (lat_lon_grid.jl:141-163) in Float64: zonal spacing shrinks with
    cos(latitude), the meridional one is constant, areas and volumes are the products of the
    spacings with dzF, the face area Az is the band area between the y faces."""
    r = 6370.0e3
    g = LatLonGrid(size=(24, 20, 6), lat=(30, 32), lon=(-10, -7.6), z=(0, -60), FT=np.float64)
    assert g.topology == (Bounded, Bounded, Bounded)
    d2r = np.pi / 180
    dlon, dlat = (-7.6 - -10.0) / 24, (32 - 30) / 20         # (lon₂ − lon₁)/Nx, (lat₂ − lat₁)/Ny
    for j in (0, 7, 23):
        assert g.dxC[3, j] == r * np.cos(g.yC[j] * np.pi / 180) * (dlon * d2r)
    assert np.all(g.dyC == r * (dlat * d2r)) and np.all(g.dxF == g.dxC) and np.all(g.dyF == g.dyC)
    assert np.all(np.diff(g.dxC[0, :]) < 0)                    # northern hemisphere: shrinks poleward
    Gx, Gy, Gz = g.total_size
    j = 5
    assert g.Az[2, j] == (r * r) * (dlon * d2r) * (np.sin(g.yF[j + 1] * np.pi / 180) - np.sin(g.yF[j] * np.pi / 180))
    assert g.Az[Gx - 1, Gy - 1] == 0.0                         # the corner the reference leaves at zero
    assert np.array_equal(g.Az[Gx - 1, :Gy - 1], g.Az[Gx - 2, :Gy - 1])
    k = 4
    assert np.array_equal(g.Ax[:, :, k], g.dzF[k] * g.dyF)
    assert np.array_equal(g.Ay[:, :, k], g.dzF[k] * g.dxF)
    assert np.array_equal(g.Vol[:, :, k], g.Az * g.dzF[k])
    # volumes sum to the shell segment between the faces (to the accuracy of the sine differences)
    Hx, Hy, Hz = g.Hx, g.Hy, g.Hz
    V = g.Vol[Hx:Hx + 24, Hy:Hy + 20, Hz:Hz + 6].sum()
    exact = r * r * (24 * dlon * d2r) * (np.sin(32 * d2r) - np.sin(30 * d2r)) * 60.0
    assert abs(V - exact) <= 1e-9 * exact


def test_load_lat_lon_grid():                        # grid_test.jl:84-113, with a synthetic grid_info
    """The reference loads MITgcm's one-degree channel (MeshArrays, not available here); the same
    loader is driven with arrays of those shapes whose level thicknesses span 10 .. 456.5 m."""
    Nx, Ny, Nz = 36, 16, 5
    drf = np.array([10.0, 50.0, 120.0, 300.0, 456.5])
    rf = np.concatenate([[0.0], -np.cumsum(drf)])
    rc = 0.5 * (rf[:-1] + rf[1:])
    drc = np.concatenate([[-rc[0]], rc[:-1] - rc[1:]])
    rng = np.random.default_rng(3)
    info = dict(RF=rf, RC=rc, DRF=drf, DRC=drc,
                DXC=1e5 * rng.uniform(0.9, 1.1, (Nx, Ny)), DXG=1e5 * rng.uniform(0.9, 1.1, (Nx, Ny)),
                DYC=np.full((Nx, Ny), 1.1e5), DYG=np.full((Nx, Ny), 1.1e5),
                RAC=1.1e10 * rng.uniform(0.9, 1.1, (Nx, Ny)),
                hFacC=np.ones((Nx, Ny, Nz)), hFacW=np.ones((Nx, Ny, Nz)), hFacS=np.ones((Nx, Ny, Nz)))
    mask = np.ones((Nx, Ny, Nz), dtype=bool)
    g = LoadLatLonGrid(grid_info=info, size=(Nx, Ny, Nz), lat=(-80, 80), lon=(-180, 180), landmask=mask, FT=np.float64)
    assert (g.Nx, g.Ny, g.Nz) == (Nx, Ny, Nz)
    for a, n in ((g.xC, Nx), (g.yC, Ny), (g.zC, Nz), (g.xF, Nx), (g.yF, Ny), (g.zF, Nz)):
        assert len(a) == n + 4
    assert g.dzF.min() == 10.0 and g.dzF.max() == 456.5
    assert g.dzC[2] == 2.0 * drc[0]                            # the first layer only has half of the grid
    Hx, Hy = g.Hx, g.Hy
    assert np.array_equal(g.dxF[Hx:Hx + Nx, Hy:Hy + Ny], info["DXG"])
    assert np.array_equal(g.dxC[0:Hx, :], g.dxC[Nx:Nx + Hx, :])  # periodic in x
    assert np.array_equal(g.Vol[:, :, 3], g.dzF[3] * g.Az)


def _tot_mass(c, g):
    vol = G.cell_volumes(g)
    return float(np.sum(G.interior(c, g) * G.interior(vol, g)))


@pytest.mark.parametrize("lon", [(-10.0, -7.6), (-180.0, 180.0)])
def test_latlon_phosphorus_budget_divergence_free_tight(lon):
    """With a flow whose face transports cancel in every cell and no divisions, P moves between
    individuals, PO4, DOP and POP without loss on a LatLonGrid (Bounded or Periodic in x): the
    budget with the grid's own cell volumes closes to rounding after 20 steps."""
    nx = 24 if lon[0] != -180.0 else 36
    lat = (30.0, 32.0) if lon[0] != -180.0 else (-60.0, 60.0)
    wl = W.latlon(nx=nx, lon=lon, lat=lat, N_per_species=800, steps=20,
                  phyt_over={"dvid_P": [0.0, 0.0], "mort_P": [2e-4, 2e-4], "mort_reg": [0.9, 0.9]})
    m = oracle.from_workload(wl)
    g = wl.grid

    def TP():
        t = sum(_tot_mass(m.get_tracer(n), g) for n in (3, 7, 11))
        for s in range(wl.nsp):
            d = m.get_individuals(s)
            a = d["ac"]
            t += float(np.sum((d["Pq"] + d["Bm"] * wl.phyt["R_PC"][s])[a]))
        return t

    tp0 = TP()
    u, v, w = wl.velocity(0)
    for it in range(wl.steps):
        m.set_velocity(u, v, w)
        m.set_PARF(wl.parf[:, :, int(it * wl.dT // 3600)])
        m.set_temp(wl.temp[:, :, :, int(it * wl.dT // 3600)])
        m.time_step(wl.dT)
    x = m.get_individuals(0)["x"]
    assert np.any(np.abs(x - wl.individuals[0]["x"]) > 0.05)     # the flow moved them
    assert abs(TP() - tp0) <= 1e-12 * tp0


def test_latlon_refused_by_the_fp32_form():
    """The FP32 form has no LatLonGrid path: pi_create(..., PI_FP32) refuses the grid before any
    device call, and PlanktonModel asks for FT = Float64."""
    from PlanktonIndividuals import GPU, PlanktonModel, _lib
    from PlanktonIndividuals._native import CModel, PIError
    wl = W.latlon(N_per_species=50, steps=1)
    lib = _lib.load()
    with pytest.raises(PIError) as e:
        CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP32)
    assert e.value.code == _abi.PI_ERR_ARG and "LatLonGrid" in str(e.value)
    with pytest.raises(NotImplementedError):
        PlanktonModel(GPU(), wl.grid, FT=np.float32)
