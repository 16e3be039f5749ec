"""Edge cases of the FP64 step, GPU vs oracle with tolerance 0: land mask (2D and 3D), Bounded
x/y, flux boundary conditions, tracer and individual diffusion, per-species grazing, the Timer and Sizer_Timer division types, capacity
overflow, N steps = N/2 + N/2 (checkpoint/resume), and the device-resident update! path."""
import ctypes as ct

import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel, CapacityError
from PlanktonIndividuals.grids import Bounded, Periodic, RectilinearGrid, fill_halo_tracer
from helpers import VelCache, compare_states, drive, forcing_indices

pytestmark = pytest.mark.gpu


def pair(lib, wl):
    ref = oracle.from_workload(wl)
    gpu = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    gpu.set_state(wl.individuals, wl.tracers)
    return ref, gpu


def daylight(wl):
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    return wl


def regrid(wl, grid, seed=3):
    """Same physics on another grid (topology/land mask): rebuild individuals and tracers."""
    rng = np.random.default_rng(seed)
    wl.grid = grid
    wl.individuals = [W.make_individuals(grid, wl.phyt, s, wl.N[s], wl.capacity, rng) for s in range(wl.nsp)]
    wl.tracers = W.make_tracers(grid, rng)
    u, v, w = W.double_gyre(grid, 0.1)
    if grid.topo[0] == _abi.PI_BOUNDED:
        u = np.concatenate([u, u[:1]], axis=0)
    if grid.topo[1] == _abi.PI_BOUNDED:
        v = np.concatenate([v, v[:, :1]], axis=1)
    wl.vel_fn = lambda t: (np.asfortranarray(u), np.asfortranarray(v), w)
    wl.parf = W.diel_parf(grid.Nx, grid.Ny, wl.parf.shape[2])
    from PlanktonIndividuals.parameters import default_temperature
    wl.temp = default_temperature(grid, wl.dT, wl.steps)
    return daylight(wl)


OVER = {"dvid_P": [1e-3], "dvid_reg": [1.0], "mort_P": [5e-4], "mort_reg": [0.9], "grz_P": [2e-4]}


def test_landmask_bitexact(gpu_lib):
    wl = W.config1(n=24, N=1200, steps=30, capacity=4000, phyt_over=OVER)
    lm = np.ones((24, 24, 1), dtype=bool)
    lm[5:9, 3:20, :] = False
    lm[15:17, 10:12, :] = False
    g = RectilinearGrid(size=(24, 24, 1), x=(0.0, 24e3), y=(0.0, 24e3), z=(0.0, -10.0), FT=np.float64,
                        landmask=lm)
    wl = regrid(wl, g)
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 30, vel); drive(gpu, wl, 30, vel)
    assert compare_states(ref, gpu, 1) == []


def test_bounded_xy_bitexact(gpu_lib):
    wl = W.config1(n=20, N=900, steps=25, capacity=3000, phyt_over=OVER)
    g = RectilinearGrid(size=(20, 20, 1), x=(0.0, 20e3), y=(0.0, 20e3), z=(0.0, -10.0), FT=np.float64,
                        topology=(Bounded, Bounded, Bounded))
    wl = regrid(wl, g)
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 25, vel); drive(gpu, wl, 25, vel)
    assert compare_states(ref, gpu, 1) == []


def test_flux_bcs_bitexact(gpu_lib):
    wl = daylight(W.config2(nx=12, nz=6, N_per_species=500, nsp=1, steps=12, nmodes=12))
    ref, gpu = pair(gpu_lib, wl)
    g = wl.grid
    rng = np.random.default_rng(0)
    for m in (ref, gpu):
        m.set_flux_bc(_abi.tracer_names.index("NO3"), _abi.FACES["top"], _abi.PI_BC_CONST, [1e-4])
        m.set_flux_bc(_abi.tracer_names.index("DIC"), _abi.FACES["west"], _abi.PI_BC_ARRAY2D,
                      np.asfortranarray(rng.uniform(0, 1e-3, (g.Ny, g.Nz))))
        m.set_flux_bc(_abi.tracer_names.index("DON"), _abi.FACES["bottom"], _abi.PI_BC_ARRAY3D,
                      np.asfortranarray(rng.uniform(0, 1e-5, (g.Nx, g.Ny, 20))), 20)
        rng = np.random.default_rng(0)
    vel = VelCache(wl)
    drive(ref, wl, 12, vel); drive(gpu, wl, 12, vel)
    assert compare_states(ref, gpu, 1) == []


def landmask_3d(wl, seed=5):
    """The workload on the same geometry with land: a sloping bottom (deep cells of the western
    columns) and a block of land through the upper levels; tracers rebuilt on the masked grid."""
    g = wl.grid
    lm = np.ones((g.Nx, g.Ny, g.Nz), dtype=bool)
    for i in range(g.Nx // 2):
        lm[i, :, g.Nz - 1 - (g.Nx // 2 - i) * g.Nz // g.Nx:] = False
    lm[g.Nx // 2:g.Nx // 2 + 3, 2:g.Ny - 3, :g.Nz // 2] = False
    wl.grid = RectilinearGrid(size=(g.Nx, g.Ny, g.Nz), x=(0.0, g.Nx * float(g.Δx)), y=(0.0, g.Ny * float(g.Δy)),
                              z=(0.0, -float(np.sum(np.asarray(g.dzF)[g.Hz:g.Hz + g.Nz]))), FT=np.float64,
                              topology=(Periodic, Periodic, Bounded), landmask=lm)
    wl.tracers = W.make_tracers(wl.grid, np.random.default_rng(seed), no3_gradient_depth=2.0 * g.Nz)
    return wl


DIFFUSION = {"κh": 1.0, "κv": 1e-3, "κhP": 0.5, "κvP": 2e-4}

IRON_INIT = {"DFe": 2e-4, "PFe_inorg": 1e-4, "PFe_bio": 5e-5, "Dust": 1e-3}


def with_iron(wl, seed=7, lm=None):
    """Non-zero iron tracers and dust (the workloads start them at zero), so the iron forcing,
    the sinking of PFe_inorg, PFe_bio and Dust, and the DFe ligand threshold all act."""
    rng = np.random.default_rng(seed)
    g = wl.grid
    for name, v0 in IRON_INIT.items():
        a = np.asfortranarray(v0 * rng.uniform(0.2, 1.8, g.total_size)) * g.landmask
        fill_halo_tracer(a, g)
        wl.tracers[_abi.tracer_names.index(name)] = np.asfortranarray(a)
    wl.bgc["ligand"] = 2e-4      # DFe above and below the threshold of the scavenging term
    return wl


def test_iron_and_sinking_bitexact(gpu_lib):
    wl = with_iron(daylight(W.config2(nx=12, nz=10, N_per_species=600, nsp=1, steps=15, nmodes=12, phyt_over=OVER)))
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 15, vel); drive(gpu, wl, 15, vel)
    assert compare_states(ref, gpu, 1) == []


def test_landmask_3d_bitexact(gpu_lib):
    wl = landmask_3d(daylight(W.config2(nx=16, nz=10, N_per_species=900, nsp=1, steps=15, nmodes=12,
                                        phyt_over=OVER)))
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 15, vel); drive(gpu, wl, 15, vel)
    assert compare_states(ref, gpu, 1) == []


def test_diffusion_bitexact(gpu_lib):
    """tracer_diffusion! (κh, κv) and the individuals' random walk (κhP, κvP) switched on."""
    wl = daylight(W.config2(nx=12, nz=8, N_per_species=700, nsp=1, steps=15, nmodes=12, phyt_over=OVER))
    wl.bgc.update(DIFFUSION)
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 15, vel); drive(gpu, wl, 15, vel)
    assert compare_states(ref, gpu, 1) == []


def test_per_species_grazing_and_division_types(gpu_lib):
    over = {"dvid_type": [2, 3], "dvid_P": [2e-3, 2e-3], "dvid_reg": [12.0, 1.5], "dvid_reg2": [12.0, 6.0],
            "grz_P": [3e-4, 3e-4], "mort_P": [3e-4, 3e-4]}
    wl = daylight(W.config2(nx=12, nz=6, N_per_species=700, nsp=2, steps=25, nmodes=12, phyt_over=over))
    wl.bgc["shared_graz"] = 0.0
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 25, vel); drive(gpu, wl, 25, vel)
    assert compare_states(ref, gpu, 2) == []


def test_capacity_overflow_message(gpu_lib):
    over = {"dvid_P": [5e-2], "dvid_reg": [0.5]}
    wl = daylight(W.config1(n=8, N=200, steps=10, capacity=210, phyt_over=over))
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    msgs = []
    for m in (ref, gpu):
        with pytest.raises(CapacityError) as e:
            drive(m, wl, 10, vel)
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1]
    it, t = gpu.get_time()
    assert msgs[1] == f"number of individual exceeds the capacity at timestep {t / 86400.0!r} days"


def test_split_run_equals_full_run(gpu_lib):
    """Checkpoint/resume: download the state after N/2 steps into a fresh model, continue, and
    compare with an uninterrupted run (bit-exact)."""
    wl = daylight(W.config1(n=16, N=500, steps=20, capacity=1500, phyt_over=OVER))
    _, a = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(a, wl, 20, vel)
    _, b = pair(gpu_lib, wl)
    drive(b, wl, 10, vel)
    inds = [b.get_individuals(0)]
    trs = [b.get_tracer(n) for n in range(_abi.NTRACERS)]
    it, t = b.get_time()
    c = CModel(gpu_lib, "pi_", wl.grid, wl.bgc, wl.phyt, 1, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    c.set_state(inds, trs)
    c.set_time(it, t)
    # vel₀ is part of the timestepper state: the velocity of step 10
    c.set_velocity0(*vel(forcing_indices(t - wl.dT, wl)[0]))
    drive(c, wl, 10, vel)
    for k, va in a.get_individuals(0).items():
        assert np.array_equal(va, c.get_individuals(0)[k]), k
    for n in range(_abi.NTRACERS):
        assert np.array_equal(a.get_tracer(n), c.get_tracer(n))


def test_simulation_update_path_bitexact(gpu_lib):
    """pi_sim_create/pi_sim_update (series resident on the device) equals step-by-step uploads."""
    wl = daylight(W.config2(nx=12, nz=8, N_per_species=600, nsp=1, steps=24, nmodes=12, phyt_over=OVER))
    wl.dT_vel = 8 * wl.dT
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 24, vel)
    snaps = [vel(i) for i in range(3)]
    u = np.asfortranarray(np.stack([s[0] for s in snaps], axis=3))
    v = np.asfortranarray(np.stack([s[1] for s in snaps], axis=3))
    w = np.asfortranarray(np.stack([s[2] for s in snaps], axis=3))
    dp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    lib = gpu_lib
    sim = ct.c_void_p()
    assert lib.pi_sim_create(gpu.h, wl.dT, 24, dp(u), dp(v), dp(w), 3, wl.dT_vel, dp(wl.parf), wl.parf.shape[2],
                             wl.dT_PAR, dp(wl.temp), wl.temp.shape[3], wl.dT_temp, ct.byref(sim)) == 0
    assert lib.pi_sim_update(sim, 0, 1) == 0
    lib.pi_sim_destroy(sim)
    assert compare_states(ref, gpu, 1) == []
