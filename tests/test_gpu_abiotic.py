"""Abiotic particles (src/Individuals/Abiotic/) in the FP64 form on the GPU against the CPU oracle
with tolerance 0: particles created from constant, face-array and time-series particle fluxes,
advected and diffused, merged into phytoplankton through the cell-binned interaction (candidate
collisions, the max_ptc cap) and released again, with the ptc and abiotic num diagnostics; the
error paths; and the drop-in API (PlanktonModel(...; abiotic = abiotic_setup(...)),
set_bc_particle!, PlanktonSimulation, update!)."""
import math

import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CapacityError, CModel, PIError
from PlanktonIndividuals.grids import Bounded
from helpers import VelCache, compare_states, drive, same

pytestmark = pytest.mark.gpu


def pair(lib, wl):
    ref = W.configure_abiotics(oracle.from_workload(wl), wl)
    gpu = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    gpu.set_state(wl.individuals, wl.tracers)
    W.configure_abiotics(gpu, wl)
    return ref, gpu


def compare_abiotics(ref, gpu, nsa):
    bad = []
    for a in range(nsa):
        A, B = ref.get_abiotic_particles(a), gpu.get_abiotic_particles(a)
        bad += [f"sa{a + 1}.{k}" for k in A if not same(A[k], B[k])]
        if not same(ref.get_diag(_abi.PI_DIAG_ABIO_NUM, a), gpu.get_diag(_abi.PI_DIAG_ABIO_NUM, a)):
            bad.append(f"sa{a + 1}.num")
    return bad


def tracers_equal(ref, gpu):
    return [n for n in range(_abi.NTRACERS) if not same(ref.get_tracer(n), gpu.get_tracer(n))]


@pytest.mark.parametrize("topology", ["periodic", "bounded"])
def test_abiotic_creation_interaction_release_fp64_bitexact(gpu_lib, topology):
    topo = None if topology == "periodic" else (Bounded, Bounded, Bounded)
    wl = W.abiotic(steps=20, topology=topo)
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    for chunk in range(4):
        drive(ref, wl, 5, vel)
        drive(gpu, wl, 5, vel)
        assert compare_states(ref, gpu, wl.nsp) == [], chunk
        assert compare_abiotics(ref, gpu, 2) == [], chunk
        assert tracers_equal(ref, gpu) == [], chunk
    for s in range(wl.nsp):
        assert same(ref.get_diag(_abi.PI_DIAG_PTC, s), gpu.get_diag(_abi.PI_DIAG_PTC, s))
    p1 = gpu.get_individuals(1)
    assert gpu.get_individuals(0)["ptc"].sum() > 0 and p1["ptc"].max() == wl.abiotic["max_ptc"][1]
    assert gpu.count_abiotic(1) > 1000                                # boundary creation
    assert [gpu.count_abiotic(a) for a in range(2)] == [ref.count_abiotic(a) for a in range(2)]
    gpu.close()


def test_abiotic_errors_match_the_oracle(gpu_lib):
    wl = W.abiotic(steps=4, N_abiotic=(2000, 2900), top_flux=1.0)   # the top fills 256 cells a step
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    msgs = []
    for m in (ref, gpu):
        with pytest.raises(CapacityError) as ei:
            drive(m, wl, 4, vel)
        msgs.append(str(ei.value))
    assert msgs[0] == msgs[1] and "number of abiotic particles exceeds the capacity" in msgs[1]
    wl = W.abiotic(steps=2, max_ptc=(25.0, math.nan))                 # sp2 without max_ptc
    ref, gpu = pair(gpu_lib, wl)
    vel = VelCache(wl)
    for m in (ref, gpu):
        with pytest.raises(PIError, match="no field max_ptc"):
            drive(m, wl, 2, vel)
    with pytest.raises(PIError):
        CModel(gpu_lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed,
               precision=_abi.PI_FP32).set_abiotics(wl.abiotic["params"], 2)
    gpu.close()


def test_abiotic_drop_in_api_bitexact(gpu_lib):
    """PlanktonModel(GPU(), grid; FT = Float64, abiotic = abiotic_setup(nothing, N, 2, Palat(...)))
    with set_bc_particle! → PlanktonSimulation → update!, PlanktonDiagnostics with the ptc and
    abiotic num fields, against the oracle from the model's own initial state. QuotaMode has no
    max_ptc and the default Rd = 1e-4 m merges nothing, as in the reference's 2D example."""
    from PlanktonIndividuals import (GPU, Palat, PlanktonDiagnostics, PlanktonModel, PlanktonSimulation,
                                     RectilinearGrid, abiotic_setup, default_PARF, phyto_setup, set_bc_particle_b,
                                     tracer_names, update_b)
    grid = RectilinearGrid(size=(12, 12, 6), x=(0.0, 600.0), y=(0.0, 600.0), z=(0.0, -12.0), FT=np.float64)
    model = PlanktonModel(GPU(), grid, FT=np.float64, max_individuals=4000, phyto=phyto_setup(None, [1500, 800], 2),
                          abiotic=abiotic_setup(None, [1000, 300], 2, Palat([("sp1", "sa1")], [("sp1", "sa1")])),
                          seed=6)
    set_bc_particle_b(model, sa="sa2", pos="top", bc_value=3.0e-9)
    set_bc_particle_b(model, sa="sa2", pos="bottom", bc_value=np.full((12, 12), 2.0e-9))
    diags = PlanktonDiagnostics(model, tracer=("PO4",))
    assert set(diags.abiotics) == {"sa1", "sa2"} and "ptc" in diags.phytos.sp1.keys()
    fv = W.FourierVelocity(grid, nmodes=12, rms=0.02, seed=3)
    snaps = [fv(i) for i in range(2)]
    vels = {c: np.stack([s[q] for s in snaps], axis=-1) for q, c in enumerate("uvw")}
    parf = np.asfortranarray(np.roll(default_PARF(grid, 60.0, 20), -10, axis=2))
    ref = oracle.OracleModel(grid, model.bgc_params, model.phyto.params, 2, 4000, 6)
    ref.set_state([dict(model.individuals.phytos[f"sp{s + 1}"].data) for s in range(2)],
                  [model.tracers[n].data for n in tracer_names])
    ref.set_abiotics(model.abiotic.params, 2, [(0, 0)], [(0, 0)], 25, [math.nan, math.nan])
    for a in range(2):
        ref.set_abiotic_particles(a, dict(model.individuals.abiotics[f"sa{a + 1}"].data))
    ref.set_abiotic_bc(1, _abi.FACES["top"], _abi.PI_BC_CONST, [3.0e-9])
    ref.set_abiotic_bc(1, _abi.FACES["bottom"], _abi.PI_BC_ARRAY2D, np.full((12, 12), 2.0e-9))
    sim = PlanktonSimulation(model, ΔT=60.0, iterations=20, PARF=parf, vels=vels, ΔT_vel=600.0, diags=diags)
    inp = sim.input
    for _ in range(20):
        _, t = ref.get_time()
        tv, tp, tt = (int(math.floor(t / inp[k])) for k in ("ΔT_vel", "ΔT_PAR", "ΔT_temp"))
        ref.set_velocity(*(np.asfortranarray(np.asarray(inp["vels"][c])[..., tv]) for c in "uvw"))
        ref.set_PARF(inp["PARF"][:, :, tp])
        ref.set_temp(inp["temp"][:, :, :, tt])
        ref.time_step(60.0)
    update_b(sim)
    assert compare_states(ref, model._native, 2) == []
    assert compare_abiotics(ref, model._native, 2) == []
    assert same(ref.get_diag(_abi.PI_DIAG_ABIO_NUM, 1), diags.abiotics.sa2.num)
    assert not diags.phytos.sp1.ptc.any()
    assert model.count_abiotic()[1] > 300
    with pytest.raises(NotImplementedError):
        PlanktonModel(GPU(), grid, FT=np.float32, max_individuals=100, phyto=phyto_setup(None, [10], 1),
                      abiotic=abiotic_setup(None, [10], 1))
