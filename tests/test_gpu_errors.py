"""Error paths of the C ABI on the GPU, with the failure made on the host (no GPU fault):

- pi_check_finite / pi_batch_check_finite: a NaN written into a tracer cell, or an Inf into an
  attribute of an active individual, through the setters is reported as PI_ERR_NAN naming the
  tracer and its (i, j, k) cell, or the individual and its species (1-based), in both precisions;
  a clean state passes.
- PI_ERR_DOMAIN: a velocity far above CFL 1 carries individuals out of the halo-padded grid; the
  step reports PI_ERR_DOMAIN as the oracle does, and the FP64 state after the step (positions
  clamped into the grid) equals the oracle's bit for bit.
"""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel, PIError
from helpers import VelCache, compare_states, drive

pytestmark = pytest.mark.gpu


def _model(lib, wl, precision):
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=precision)
    m.set_state(wl.individuals, wl.tracers)
    return m


@pytest.mark.parametrize("precision", [_abi.PI_FP64, _abi.PI_FP32])
def test_check_finite_names_injected_nan(gpu_lib, precision):
    wl = W.config2(nx=12, nz=6, N_per_species=300, nsp=2, steps=4, nmodes=8, seed=51)
    m = _model(gpu_lib, wl, precision)
    m.check_finite()
    no3 = _abi.tracer_names.index("NO3")
    bad = wl.tracers[no3].copy(order="F")
    bad[4, 6, 3] = np.nan                       # Julia (5, 7, 4)
    m.set_tracer(no3, bad)
    with pytest.raises(PIError) as ei:
        m.check_finite()
    assert ei.value.code == _abi.PI_ERR_NAN
    assert "tracer NO3 at (5, 7, 4)" in str(ei.value)
    m.set_tracer(no3, wl.tracers[no3])
    m.check_finite()
    inds = {k: np.array(v, copy=True) for k, v in wl.individuals[1].items()}
    slot = int(np.nonzero(inds["ac"])[0][17])
    inds["Bm"][slot] = np.inf
    m.set_individuals(1, inds)
    with pytest.raises(PIError) as ei:
        m.check_finite()
    assert ei.value.code == _abi.PI_ERR_NAN
    assert f"individual {slot + 1} of species 2" in str(ei.value)
    m.close()


@pytest.mark.parametrize("precision", [_abi.PI_FP64, _abi.PI_FP32])
def test_domain_error_above_cfl_one(gpu_lib, precision):
    wl = W.config1(n=16, N=400, steps=2, capacity=1200)
    u, v, w = wl.velocity(0)
    fast = (np.asfortranarray(u * 1e5), np.asfortranarray(v * 1e5), w)
    ref, m = oracle.from_workload(wl), _model(gpu_lib, wl, precision)
    for x in (ref, m):
        x.set_velocity(*fast)
        x.set_PARF(wl.parf[:, :, 0])
        x.set_temp(wl.temp[:, :, :, 0])
    with pytest.raises(PIError) as e_ref:
        ref.time_step(wl.dT)
    with pytest.raises(PIError) as e_gpu:
        m.time_step(wl.dT)
    assert e_ref.value.code == e_gpu.value.code == _abi.PI_ERR_DOMAIN
    if precision == _abi.PI_FP64:
        assert compare_states(ref, m, wl.nsp) == []
    m.close()


def test_bounded_wait_gives_up_and_context_stays_usable(gpu_lib):
    """A device-side wait on an mbarrier that nothing arrives on (the helper the tracer kernel's
    staging waits use) gives up after its limit and reports it; the context runs a step afterwards."""
    import ctypes as ct
    gave, waited = ct.c_int32(-1), ct.c_int64(0)
    assert gpu_lib.pi_selftest_bounded_wait(ct.c_int64(20_000_000), ct.byref(gave), ct.byref(waited)) == 0
    assert gave.value == 1
    assert 20_000_000 <= waited.value < 1_000_000_000
    wl = W.config1(n=16, N=256, steps=2)
    m = CModel(gpu_lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP32)
    m.set_state(wl.individuals, wl.tracers)
    drive(m, wl, 2, VelCache(wl))
    assert m.count_active(0) > 0
    m.close()
