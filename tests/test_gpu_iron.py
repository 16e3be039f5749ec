"""IronEnergyMode (src/Individuals/Plankton/IronEnergyMode/) in the FP64 form on the GPU against the
CPU oracle with tolerance 0: every pool (Sz, Bm, CH, qNO3, qNH4, qP, the four Fe quotas, exEn, Chl,
tdark), gen, age, decisions, tracers (DFe and PFe_bio included) and the 32 process diagnostics
across sunset, with divisions, grazing and a nitrogen-fixing species, including the stale pools
of inactive slots; and through PlanktonModel → PlanktonSimulation → update!."""
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
                 precision=_abi.PI_FP64, mode="iron")
    gpu.set_state(wl.individuals, wl.tracers)
    return ref, gpu


def test_iron_sunset_divisions_grazing_fp64_bitexact(gpu_lib):
    over = {"dvid_P": [2e-4, 2e-4], "dvid_reg": [1.0, 1.0], "grz_P": [1e-4, 5e-5], "mort_P": [5e-4, 3e-4],
            "mort_reg": [1.5, 1.5], "is_nr": [1.0, 0.0], "is_croc": [0.0, 1.0]}
    wl = W.iron(N_per_species=1500, steps=40, capacity=6000, phyt_over=over,
                bgc_over={"κhP": 0.5, "κvP": 2e-4})
    ref, gpu = pair(gpu_lib, wl)
    for m in (ref, gpu):
        m.set_diags(1 << _abi.tracer_names.index("DFe"), (1 << len(_abi.IRON_PROC_NAMES)) - 1)
    vel = VelCache(wl)
    for chunk in range(4):
        drive(ref, wl, 10, vel)
        drive(gpu, wl, 10, vel)
        assert compare_states(ref, gpu, 2) == [], chunk
    for n in range(_abi.NTRACERS):
        assert same(ref.get_tracer(n), gpu.get_tracer(n)), _abi.tracer_names[n]
    for q in range(len(_abi.IRON_PROC_NAMES)):
        for s in range(2):
            assert same(ref.get_diag(_abi.PI_DIAG_PROC + q, s), gpu.get_diag(_abi.PI_DIAG_PROC + q, s)), q
    assert same(ref.get_diag(_abi.PI_DIAG_TRACER + _abi.tracer_names.index("DFe"), 0),
                gpu.get_diag(_abi.PI_DIAG_TRACER + _abi.tracer_names.index("DFe"), 0))
    e = gpu.get_individuals(1)
    a = e["ac"]
    assert np.all(e["tdark"][a] > 0) and np.sum(e["gen"][a] >= 2.0) > 20 and np.any(e["qFeNF"][a])
    b = gpu.budget()
    assert b[3] > 0 and b[4] > 0 and b[5] > 0
    gpu.close()


def test_iron_fp32_is_refused(gpu_lib):
    wl = W.iron(N_per_species=100, steps=1)
    with pytest.raises(PIError) as ei:
        CModel(gpu_lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP32,
               mode="iron")
    assert "FP64 form only" in str(ei.value)


def test_iron_drop_in_api_bitexact(gpu_lib):
    """PlanktonModel(GPU(), grid; FT = Float64, mode = IronEnergyMode()) → PlanktonSimulation →
    update!, with diagnostics by name, against the oracle from the model's own initial state."""
    from PlanktonIndividuals import (GPU, IronEnergyMode, PlanktonDiagnostics, PlanktonModel, PlanktonSimulation,
                                     RectilinearGrid, default_PARF, phyto_setup, tracer_names, update_b)
    grid = RectilinearGrid(size=(12, 12, 6), x=(0.0, 600.0), y=(0.0, 600.0), z=(0.0, -12.0), FT=np.float64)
    params = {"dvid_P": 2e-4, "dvid_reg": 1.0, "grz_P": 5e-5}
    model = PlanktonModel(GPU(), grid, FT=np.float64, mode=IronEnergyMode(), max_individuals=4000,
                          phyto=phyto_setup(dict(params), [1500], 1), seed=5)
    diags = PlanktonDiagnostics(model, tracer=("DFe",), phytoplankton=("num", "PS", "VFe", "qFePS", "tdark"))
    fv = W.FourierVelocity(grid, nmodes=12, rms=0.02, seed=3)
    snaps = [fv(i) for i in range(2)]
    vels = {c: np.stack([s[q] for s in snaps], axis=-1) for q, c in enumerate("uvw")}
    parf = np.asfortranarray(np.roll(default_PARF(grid, 60.0, 20), -10, axis=2))
    ref = oracle.OracleModel(grid, model.bgc_params, model.phyto.params, 1, 4000, 5, mode="iron")
    ref.set_state([dict(model.individuals.phytos.sp1.data)], [model.tracers[n].data for n in tracer_names])
    names = _abi.IRON_PROC_NAMES
    ref.set_diags(1 << tracer_names.index("DFe"), sum(1 << names.index(k) for k in ("PS", "VFe", "qFePS", "tdark")))
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
    assert same(ref.get_diag(_abi.PI_DIAG_PROC + names.index("VFe"), 0), diags.phytos.sp1.VFe)
    assert same(ref.get_diag(_abi.PI_DIAG_PROC + names.index("qFePS"), 0), diags.phytos.sp1.qFePS)
    with pytest.raises(NotImplementedError):
        PlanktonModel(GPU(), grid, FT=np.float32, mode=IronEnergyMode(), max_individuals=100,
                      phyto=phyto_setup(None, [10], 1))
