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
