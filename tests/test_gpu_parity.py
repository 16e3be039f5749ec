"""FP64 GPU step vs the CPU oracle: identical inputs and draws give identical Float64 bits for
every individual attribute, cell index, tracer and diagnostic (tolerance 0)."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel
from helpers import VelCache, compare_states, drive

pytestmark = pytest.mark.gpu


def gpu_model(lib, wl):
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    m.set_state(wl.individuals, wl.tracers)
    return m


def run_pair(lib, wl, steps):
    ref, gpu = oracle.from_workload(wl), gpu_model(lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, steps, vel)
    drive(gpu, wl, steps, vel)
    return ref, gpu


def daylight(wl):
    # shift the light series so the run starts in daylight
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    return wl


def test_config1_small_bitexact(gpu_lib):
    wl = daylight(W.config1(n=32, N=1024, steps=40))
    ref, gpu = run_pair(gpu_lib, wl, 40)
    assert compare_states(ref, gpu, wl.nsp) == []
    assert gpu.count_active(0) == ref.count_active(0)


def test_divisions_deaths_grazing_bitexact(gpu_lib):
    over = {"dvid_P": [1e-3], "dvid_reg": [1.0], "mort_P": [5e-4], "mort_reg": [0.9], "grz_P": [2e-4]}
    wl = daylight(W.config1(n=24, N=1500, steps=60, capacity=6000, phyt_over=over))
    ref, gpu = run_pair(gpu_lib, wl, 60)
    assert compare_states(ref, gpu, wl.nsp) == []
    n = gpu.count_active(0)
    assert n != 1500      # the population changed: divisions and deaths happened


def test_config2_small_3d_two_species_bitexact(gpu_lib):
    over = {"dvid_P": [1e-3, 2e-3], "dvid_reg": [1.0, 1.1], "mort_P": [3e-4, 3e-4], "grz_P": [1e-4, 0.0]}
    wl = daylight(W.config2(nx=16, nz=12, N_per_species=2500, steps=30, nmodes=24, phyt_over=over))
    wl.dT_vel = 10 * wl.dT      # refresh every 10 steps in this small case
    ref, gpu = run_pair(gpu_lib, wl, 30)
    assert compare_states(ref, gpu, wl.nsp) == []
