"""Optional diagnostics on the GPU (PlanktonDiagnostics(model; tracer, phytoplankton),
src/Diagnostics/diagnostics_struct.jl:23-105, diags_spcs! in diagnostics_kernels.jl:14-33, tracer
sums of time_step.jl:168-172), with every QuotaMode process and several tracers enabled, two
species, divisions, deaths and grazing (daughters add at their slot's stale find_inds! cell):
- FP64 form against the CPU oracle, tolerance 0 for every field;
- FP32 form within 1e-4 of each field's largest magnitude (its processes are Float32 values summed
  in 64-bit fixed point, its tracer sums Float32 as the reference's Float32 diagnostics);
- through the Python PlanktonDiagnostics of a PlanktonModel: the same fields by name.
"""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel
from helpers import VelCache, drive, same

pytestmark = pytest.mark.gpu

ALL_PROC = (1 << len(_abi.PROC_NAMES)) - 1
TMASK = sum(1 << _abi.tracer_names.index(n) for n in ("NO3", "DOC", "POC", "Dust"))
OPTIONAL_ZERO = (_abi.PI_DIAG_TRACER + _abi.tracer_names.index("Dust"),
                 _abi.PI_DIAG_PROC + _abi.PROC_NAMES.index("VDOC"), _abi.PI_DIAG_PROC + _abi.PROC_NAMES.index("exu"))


def _wl():
    over = {"dvid_P": [1e-3, 2e-3], "dvid_reg": [1.0, 1.1], "mort_P": [3e-4, 3e-4], "grz_P": [1e-4, 0.0]}
    wl = W.config2(nx=16, nz=10, N_per_species=2500, steps=20, nmodes=16, seed=81, phyt_over=over)
    wl.parf = np.asfortranarray(np.full_like(wl.parf, 400.0))     # daylight: photosynthesis runs
    wl.dT_vel = 10 * wl.dT
    return wl


def _run(lib, wl, precision, steps):
    ref = oracle.from_workload(wl)
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=precision)
    m.set_state(wl.individuals, wl.tracers)
    for x in (ref, m):
        x.set_diags(TMASK, ALL_PROC)
    vel = VelCache(wl)
    drive(ref, wl, steps, vel)
    drive(m, wl, steps, vel)
    return ref, m


def _kinds(wl):
    out = [(_abi.PI_DIAG_TRACER + n, 0) for n in range(_abi.NTRACERS) if TMASK >> n & 1]
    out += [(_abi.PI_DIAG_PROC + q, s) for s in range(wl.nsp) for q in range(len(_abi.PROC_NAMES))]
    return out


def test_optional_diagnostics_fp64_bitexact(gpu_lib):
    wl = _wl()
    ref, m = _run(gpu_lib, wl, _abi.PI_FP64, 20)
    for kind, s in _kinds(wl):
        a, b = ref.get_diag(kind, s), m.get_diag(kind, s)
        assert same(a, b), (kind, s, int(np.sum(a != b)))
        # every field is exercised except dust (none in this workload) and the two processes that
        # can stay zero in a short run (organic uptake and exudation)
        if kind not in OPTIONAL_ZERO:
            assert np.any(a != 0.0), (kind, s)
    assert gpu_lib.pi_reset_diags(m.h) == 0
    assert not np.any(m.get_diag(_abi.PI_DIAG_PROC, 0))


def test_optional_diagnostics_fp32_within_bounds(gpu_lib):
    wl = _wl()
    ref, m = _run(gpu_lib, wl, _abi.PI_FP32, 20)
    for kind, s in _kinds(wl):
        a, b = ref.get_diag(kind, s), m.get_diag(kind, s)
        scale = max(float(np.abs(a).max()), 1e-300)
        assert float(np.abs(a - b).max()) <= 1e-4 * scale, (kind, s, float(np.abs(a - b).max()) / scale)


def test_plankton_diagnostics_by_name(gpu_lib):
    from PlanktonIndividuals import GPU, PlanktonDiagnostics, PlanktonModel, RectilinearGrid, TimeStep_b, phyto_setup
    grid = RectilinearGrid(size=(8, 8, 4), x=(0.0, 400.0), y=(0.0, 400.0), z=(0.0, -8.0), FT=np.float64)
    model = PlanktonModel(GPU(), grid, FT=np.float64, max_individuals=1200, phyto=phyto_setup(None, [400], 1), seed=3)
    d = PlanktonDiagnostics(model, tracer=("NH4", "DOC"), phytoplankton=("num", "PS", "Bm", "Chl"))
    assert d.tracer.keys() == ("NH4", "DOC", "PAR")
    nat = model._native
    u = np.zeros((8, 8, 4)); w = np.zeros((8, 8, 5))
    for _ in range(3):
        nat.set_velocity(u, u, w); nat.set_PARF(np.full((8, 8), 500.0)); nat.set_temp(np.full((8, 8, 4), 20.0))
        TimeStep_b(model, 60.0, d)
    assert np.array_equal(d.tracer.NH4, nat.get_diag(_abi.PI_DIAG_TRACER + _abi.tracer_names.index("NH4"), 0))
    assert np.array_equal(d.phytos.sp1.PS, nat.get_diag(_abi.PI_DIAG_PROC + _abi.PROC_NAMES.index("PS"), 0))
    assert d.phytos.sp1.Bm.sum() > 0 and d.phytos.sp1.num.sum() > 0
    with pytest.raises(ValueError, match="is not one of the diagnostics"):
        PlanktonDiagnostics(model, phytoplankton=("RP",))
