"""MacroMolecularMode (src/Individuals/Plankton/MacroMolecularMode/) in the FP64 form on the GPU
against the CPU oracle with tolerance 0: every pool (PRO, DNA, RNA, CH, NST, PST, Chl), gen, age,
decisions, tracers and diagnostics after divisions by DNA, age-dependent mortality and grazing,
including the stale pools of inactive slots, and through PlanktonModel → PlanktonSimulation →
update!."""
import math

import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel, PIError
from helpers import VelCache, compare_states, drive, same

pytestmark = pytest.mark.gpu


def pair(lib, wl):
    ref = oracle.from_workload(wl)
    gpu = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed,
                 precision=_abi.PI_FP64, mode="macro")
    gpu.set_state(wl.individuals, wl.tracers)
    return ref, gpu


def daylight(wl):
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    return wl


def test_macro_divisions_deaths_grazing_fp64_bitexact(gpu_lib):
    over = {"dvid_P": [3e-3, 2e-3], "mort_P": [8e-4, 5e-4], "grz_P": [1e-4, 5e-5], "VDOCmax": [1e-6, 0.0],
            "KsatDOC": [5.0, 0.0]}
    wl = daylight(W.macro(nx=16, nz=8, N_per_species=1500, steps=25, phyt_over=over,
                          bgc_over={"κhP": 0.5, "κvP": 2e-4}))
    C_DNA = wl.phyt["C_DNA"][0]
    for d in wl.individuals:
        d["DNA"][:400] = 2.2 * C_DNA                   # ready to divide
        d["age"][d["ac"]] = 0.8
    ref, gpu = pair(gpu_lib, wl)
    for m in (ref, gpu):
        m.set_diags(1 << _abi.tracer_names.index("DOC"), (1 << len(_abi.MACRO_PROC_NAMES)) - 1)
    vel = VelCache(wl)
    drive(ref, wl, 25, vel)
    drive(gpu, wl, 25, vel)
    assert compare_states(ref, gpu, 2) == []
    for q in range(len(_abi.MACRO_PROC_NAMES)):
        for s in range(2):
            assert same(ref.get_diag(_abi.PI_DIAG_PROC + q, s), gpu.get_diag(_abi.PI_DIAG_PROC + q, s)), q
    assert not np.any(gpu.get_diag(_abi.PI_DIAG_PROC + _abi.MACRO_PROC_NAMES.index("VNH4"), 0))     # listed as :VHN4
    e = gpu.get_individuals(0)
    assert np.sum(e["gen"][e["ac"]] >= 2.0) > 50 and ref.count_active(0) != 1500
    b = gpu.budget()
    assert b[3] > 0 and b[4] > 0 and b[5] > 0
    gpu.close()


def test_macro_fp32_is_refused(gpu_lib):
    wl = W.macro(N_per_species=100, steps=1)
    with pytest.raises(PIError) as ei:
        CModel(gpu_lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP32,
               mode="macro")
    assert "FP64 form only" in str(ei.value)


def test_macro_drop_in_api_bitexact(gpu_lib):
    """PlanktonModel(GPU(), grid; FT = Float64, mode = MacroMolecularMode()) → PlanktonSimulation →
    update!, with diagnostics by name, against the oracle from the model's own initial state."""
    from PlanktonIndividuals import (GPU, MacroMolecularMode, PlanktonDiagnostics, PlanktonModel, PlanktonSimulation,
                                     RectilinearGrid, default_PARF, phyto_setup, tracer_names, update_b)
    grid = RectilinearGrid(size=(12, 12, 6), x=(0.0, 600.0), y=(0.0, 600.0), z=(0.0, -12.0), FT=np.float64)
    params = {"dvid_P": 1e-3, "mort_P": 5e-4, "grz_P": 2e-5}
    model = PlanktonModel(GPU(), grid, FT=np.float64, mode=MacroMolecularMode(), max_individuals=4000,
                          phyto=phyto_setup(dict(params), [1500], 1), seed=5)
    diags = PlanktonDiagnostics(model, tracer=("NO3",), phytoplankton=("num", "PS", "S_PRO", "ρChl", "PRO"))
    fv = W.FourierVelocity(grid, nmodes=12, rms=0.02, seed=3)
    snaps = [fv(i) for i in range(2)]
    vels = {c: np.stack([s[q] for s in snaps], axis=-1) for q, c in enumerate("uvw")}
    parf = np.asfortranarray(np.roll(default_PARF(grid, 60.0, 20), -10, axis=2))
    ref = oracle.OracleModel(grid, model.bgc_params, model.phyto.params, 1, 4000, 5, mode="macro")
    ref.set_state([dict(model.individuals.phytos.sp1.data)], [model.tracers[n].data for n in tracer_names])
    names = _abi.MACRO_PROC_NAMES
    ref.set_diags(1 << tracer_names.index("NO3"), sum(1 << names.index(k) for k in ("PS", "S_PRO", "ρChl", "PRO")))
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
    assert compare_states(ref, model._native, 1) == []
    assert same(ref.get_diag(_abi.PI_DIAG_PROC + names.index("S_PRO"), 0), diags.phytos.sp1.S_PRO)
    assert same(ref.get_diag(_abi.PI_DIAG_PROC + names.index("PRO"), 0), diags.phytos.sp1.PRO)
    with pytest.raises(NotImplementedError):
        PlanktonModel(GPU(), grid, FT=np.float32, mode=MacroMolecularMode(), max_individuals=100,
                      phyto=phyto_setup(None, [10], 1))
