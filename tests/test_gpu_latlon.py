"""LatLonGrid (src/Grids/lat_lon_grid.jl) through the FP64 step on the GPU against the CPU oracle
with tolerance 0: per-cell spacings in the particle interpolation and diffusion, face areas and
volumes in DST3FL, tracer diffusion, flux boundary conditions, light and the consumption terms
(Grids/areas_volumes_spacings.jl:27-38), on a Bounded regional grid with land and on a Periodic
global band, and through PlanktonModel → PlanktonSimulation → update!."""
import math

import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel
from helpers import VelCache, compare_states, drive, same

pytestmark = pytest.mark.gpu

OVER2 = {"dvid_P": [1e-3, 8e-4], "dvid_reg": [1.0, 1.0], "mort_P": [5e-4, 3e-4], "mort_reg": [0.9, 0.9],
         "grz_P": [2e-4, 1e-4]}
DIFFUSION = {"κh": 50.0, "κv": 1e-3, "κhP": 20.0, "κvP": 2e-4}


def pair(lib, wl):
    ref = oracle.from_workload(wl)
    gpu = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    gpu.set_state(wl.individuals, wl.tracers)
    return ref, gpu


def daylight(wl):
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    return wl


def test_latlon_bounded_with_land_bcs_and_diffusion_bitexact(gpu_lib):
    nx, ny, nz = 24, 20, 6
    lm = np.ones((nx, ny, nz), dtype=bool)
    lm[3:7, 4:15, :] = False                       # an island through every level
    lm[15:, 12:, 4:] = False                       # a shelf in the north-east
    wl = daylight(W.latlon(nx=nx, ny=ny, nz=nz, N_per_species=1500, steps=20, landmask=lm,
                           phyt_over=OVER2, bgc_over=DIFFUSION))
    # no individual starts on land: move those that do to the nearest water column's position
    for d in wl.individuals:
        a = d["ac"]
        land = a & ~lm[np.minimum(d["x"].astype(int), nx - 1), np.minimum(d["y"].astype(int), ny - 1),
                       np.minimum(d["z"].astype(int), nz - 1)]
        d["x"][land] = 12.5
        d["y"][land] = 2.5
    ref, gpu = pair(gpu_lib, wl)
    g = wl.grid
    rng = np.random.default_rng(0)
    for m in (ref, gpu):
        m.set_flux_bc(_abi.tracer_names.index("NO3"), _abi.FACES["top"], _abi.PI_BC_CONST, [1e-4])
        m.set_flux_bc(_abi.tracer_names.index("DIC"), _abi.FACES["west"], _abi.PI_BC_ARRAY2D,
                      np.asfortranarray(rng.uniform(0, 1e-3, (g.Ny, g.Nz))))
        m.set_flux_bc(_abi.tracer_names.index("PO4"), _abi.FACES["south"], _abi.PI_BC_CONST, [2e-5])
        m.set_flux_bc(_abi.tracer_names.index("DON"), _abi.FACES["bottom"], _abi.PI_BC_ARRAY3D,
                      np.asfortranarray(rng.uniform(0, 1e-5, (g.Nx, g.Ny, 25))), 25)
        rng = np.random.default_rng(0)
    vel = VelCache(wl)
    drive(ref, wl, 20, vel)
    drive(gpu, wl, 20, vel)
    assert compare_states(ref, gpu, 2) == []
    assert ref.count_active(0) != 1500 or ref.count_active(1) != 1500     # divisions or deaths happened
    gpu.close()


def test_latlon_periodic_global_band_bitexact(gpu_lib):
    """lon = (−180, 180) makes x Periodic (lat_lon_grid.jl:98); 10° × 6° cells whose zonal
    spacing varies by a factor of two between the equator and 60°."""
    wl = daylight(W.latlon(nx=36, ny=20, nz=4, lon=(-180.0, 180.0), lat=(-60.0, 60.0), N_per_species=2000,
                           steps=16, phyt_over=OVER2, bgc_over=DIFFUSION))
    assert wl.grid.topo[0] == _abi.PI_PERIODIC
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 16, vel)
    drive(gpu, wl, 16, vel)
    assert compare_states(ref, gpu, 2) == []
    gpu.close()


def test_latlon_drop_in_api_bitexact(gpu_lib):
    """PlanktonModel(GPU(), LatLonGrid(...); FT = Float64) → PlanktonSimulation → update!, with
    diagnostics, against the oracle from the model's own initial state."""
    from PlanktonIndividuals import (GPU, LatLonGrid, PlanktonDiagnostics, PlanktonModel, PlanktonSimulation,
                                     default_PARF, phyto_setup, tracer_names, update_b)
    grid = LatLonGrid(size=(16, 12, 4), lat=(-20.0, -17.0), lon=(140.0, 144.0), z=(0.0, -40.0), FT=np.float64)
    params = {"dvid_P": 1e-3, "mort_P": 5e-4, "grz_P": 2e-5}
    model = PlanktonModel(GPU(), grid, FT=np.float64, max_individuals=4000,
                          phyto=phyto_setup(dict(params), [1500], 1), seed=9)
    diags = PlanktonDiagnostics(model, tracer=("NO3",), phytoplankton=("num", "PS"))
    u, v, w = W.latlon_streamfunction_velocity(grid, cfl=0.2, dT=300.0, seed=4)
    vels = {"u": u[..., None], "v": v[..., None], "w": w[..., None]}
    parf = np.asfortranarray(np.roll(default_PARF(grid, 300.0, 20), -10, axis=2))
    ref = oracle.OracleModel(grid, model.bgc_params, model.phyto.params, 1, 4000, 9)
    ref.set_state([dict(model.individuals.phytos.sp1.data)], [model.tracers[n].data for n in tracer_names])
    ref.set_diags(1 << tracer_names.index("NO3"), 1 << 0)
    sim = PlanktonSimulation(model, ΔT=300.0, iterations=20, PARF=parf, vels=vels, ΔT_vel=300.0 * 20, diags=diags)
    inp = sim.input
    for _ in range(20):
        _, t = ref.get_time()
        tv, tp, tt = (int(math.floor(t / inp[k])) for k in ("ΔT_vel", "ΔT_PAR", "ΔT_temp"))
        ref.set_velocity(*(np.asfortranarray(np.asarray(inp["vels"][c])[..., tv]) for c in "uvw"))
        ref.set_PARF(inp["PARF"][:, :, tp])
        ref.set_temp(inp["temp"][:, :, :, tt])
        ref.time_step(300.0)
    update_b(sim)
    assert compare_states(ref, model._native, 1) == []
    assert same(ref.get_diag(_abi.PI_DIAG_PROC + 0, 0), diags.phytos.sp1.PS)
    assert same(ref.get_diag(_abi.PI_DIAG_TRACER + tracer_names.index("NO3"), 0), diags.tracer.NO3)
    b = model._native.budget()
    from PlanktonIndividuals.grids import cell_volumes, interior
    vol = interior(cell_volumes(grid), grid)
    P = sum(float(np.sum(interior(model.tracers[n].data, grid) * vol)) for n in ("PO4", "DOP", "POP"))
    assert abs(b[2] - P) <= 1e-12 * P                          # pi_get_budget uses the cell volumes
