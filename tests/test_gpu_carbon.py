"""CarbonMode (src/Individuals/Plankton/CarbonMode/) in the FP64 form against the CPU oracle,
tolerance 0: photosynthesis with light and thermal limitation, thermal damage and repair above
Topt, respiration, division that halves the damaged biomass a daughter's slot held before,
grazing and mortality (size-based, and thermal when thermal = 1), the carbon-only consumption and
losses, and the CarbonMode process diagnostics."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel, PIError
from helpers import VelCache, compare_states, drive, same

pytestmark = pytest.mark.gpu

OVER = {"dvid_P": [1e-3, 2e-3], "mort_P": [3e-4, 3e-4], "grz_P": [1e-4, 0.0], "dvid_reg": [1.0, 1.1]}
ALL_CPROC = (1 << len(_abi.CARBON_PROC_NAMES)) - 1
TMASK = sum(1 << _abi.tracer_names.index(n) for n in ("DIC", "DOC", "POC"))


def _run(lib, wl, steps, diags=True):
    ref = oracle.from_workload(wl)
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64,
               mode="carbon")
    m.set_state(wl.individuals, wl.tracers)
    if diags:
        for x in (ref, m):
            x.set_diags(TMASK, ALL_CPROC)
    vel = VelCache(wl)
    drive(ref, wl, steps, vel)
    drive(m, wl, steps, vel)
    return ref, m


def _daylight(wl):
    wl.parf = np.asfortranarray(np.full_like(wl.parf, 600.0))
    return wl


def test_carbon_thermal_fp64_bitexact(gpu_lib):
    """thermal = 1 (default) at 28.6 °C (above Topt = 27): damage, repair and thermal mortality."""
    wl = _daylight(W.carbon(nx=16, nz=8, N_per_species=2500, steps=25, temp=28.6, bd_frac=0.5, phyt_over=OVER))
    ref, m = _run(gpu_lib, wl, 25)
    assert compare_states(ref, m, wl.nsp) == []
    counts = [m.count_active(s) for s in range(2)]
    assert counts != [2500, 2500]
    for s in range(2):
        for q in range(len(_abi.CARBON_PROC_NAMES)):
            a, b = ref.get_diag(_abi.PI_DIAG_PROC + q, s), m.get_diag(_abi.PI_DIAG_PROC + q, s)
            assert same(a, b), (q, s)
        assert np.any(ref.get_diag(_abi.PI_DIAG_PROC + _abi.CARBON_PROC_NAMES.index("TD"), s) != 0.0)
    for n in range(_abi.NTRACERS):
        if TMASK >> n & 1:
            assert same(ref.get_diag(_abi.PI_DIAG_TRACER + n, 0), m.get_diag(_abi.PI_DIAG_TRACER + n, 0))
    b = m.budget()
    d = [m.get_individuals(s) for s in range(2)]
    assert b[3] == pytest.approx(sum(float(np.sum(x["Bm"][x["ac"]])) for x in d), rel=1e-12)
    assert b[4] == 0.0 and b[5] == 0.0


def test_carbon_without_thermal_and_bacteria_fp64_bitexact(gpu_lib):
    """thermal = 0 (size-based mortality, no damage) and a bacterial species (is_bact = 1:
    photosynthesis independent of light), through a night and a day of PAR."""
    over = dict(OVER, thermal=[0.0, 0.0], is_bact=[0.0, 1.0])
    wl = W.carbon(nx=12, nz=6, N_per_species=1500, steps=30, temp=24.0, bd_frac=0.2, phyt_over=over, seed=13)
    wl.parf = np.asfortranarray(np.roll(wl.parf, -5, axis=2))
    ref, m = _run(gpu_lib, wl, 30, diags=False)
    assert compare_states(ref, m, wl.nsp) == []


def test_carbon_fp32_is_refused(gpu_lib):
    wl = W.carbon(nx=8, nz=4, N_per_species=100, steps=2)
    with pytest.raises(PIError) as ei:
        CModel(gpu_lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP32,
               mode="carbon")
    assert "FP64 form only" in str(ei.value)


def test_carbon_drop_in_api_bitexact(gpu_lib):
    """PlanktonModel(GPU(), grid; FT = Float64, mode = CarbonMode()) → PlanktonSimulation →
    update!, with PlanktonDiagnostics of CarbonMode processes by name, against the oracle from the
    model's own initial state; FT = Float32 is refused."""
    import math
    from PlanktonIndividuals import (GPU, CarbonMode, PlanktonDiagnostics, PlanktonModel, PlanktonSimulation,
                                     RectilinearGrid, default_PARF, phyto_setup, tracer_names, update_b)
    grid = RectilinearGrid(size=(12, 12, 6), x=(0.0, 600.0), y=(0.0, 600.0), z=(0.0, -12.0), FT=np.float64)
    params = {"dvid_P": 1e-3, "mort_P": 5e-4, "grz_P": 2e-5}
    model = PlanktonModel(GPU(), grid, FT=np.float64, mode=CarbonMode(), max_individuals=4000,
                          phyto=phyto_setup(dict(params), [1500], 1), seed=5)
    diags = PlanktonDiagnostics(model, tracer=("DIC",), phytoplankton=("num", "PS", "RS", "Bm"))
    fv = W.FourierVelocity(grid, nmodes=12, rms=0.02, seed=3)
    snaps = [fv(i) for i in range(2)]
    vels = {c: np.stack([s[q] for s in snaps], axis=-1) for q, c in enumerate("uvw")}
    parf = np.asfortranarray(np.roll(default_PARF(grid, 60.0, 20), -10, axis=2))
    ref = oracle.OracleModel(grid, model.bgc_params, model.phyto.params, 1, 4000, 5, mode="carbon")
    ref.set_state([dict(model.individuals.phytos.sp1.data)], [model.tracers[n].data for n in tracer_names])
    ref.set_diags(1 << tracer_names.index("DIC"), (1 << 0) | (1 << 3) | (1 << 5))
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
    assert same(ref.get_diag(_abi.PI_DIAG_PROC + 0, 0), diags.phytos.sp1.PS)
    assert same(ref.get_diag(_abi.PI_DIAG_PROC + 3, 0), diags.phytos.sp1.RS)
    assert same(ref.get_diag(_abi.PI_DIAG_TRACER + tracer_names.index("DIC"), 0), diags.tracer.DIC)
    with pytest.raises(NotImplementedError):
        PlanktonModel(GPU(), grid, FT=np.float32, mode=CarbonMode(), max_individuals=100,
                      phyto=phyto_setup(None, [10], 1))
