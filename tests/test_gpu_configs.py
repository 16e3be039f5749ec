"""Parity at the sizes of the benchmark configurations, GPU against the CPU oracle.

- Config 1 at full size (128×128×1, one species of 16,384 individuals, double-gyre flow, dt = 60 s,
  1440 steps = one day): the FP64 form equals the oracle bit for bit (tolerance 0) in every
  attribute, tracer and diagnostic; the FP32 form stays within the FP32 bounds of
  test_gpu_fp32.py.
- A 3D case of config 2's kind at 64×64×32 with two species of 50,000 individuals each and
  divisions, deaths and grazing switched on, 100 steps (one velocity refresh): FP64 == oracle.
- The vertically stretched grid of the reference's grid test (test/grid_test.jl:27-51: 4×6×4,
  z faces 0, -1, -3, -5, -10 m) and a 24×24×10 grid with a stretched profile, each through
  GPU steps: FP64 == oracle, FP32 within the FP32 bounds.
- Config 2 at full size (256×256×64, 2 × 2,097,152 individuals), 1000 steps: the FP32 batched
  form against the FP64 form (which the tests above tie to the oracle): population counts equal at
  every 100th step and interior tracer mass within 1e-5 relative at the end (marked slow).
"""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel
from PlanktonIndividuals.grids import RectilinearGrid
from helpers import VelCache, compare_states, drive
from test_gpu_fp32 import TRACER_MASS_RTOL, check_errors, errors_vs_oracle

pytestmark = pytest.mark.gpu


def _model(lib, wl, precision):
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=precision)
    m.set_state(wl.individuals, wl.tracers)
    return m


def _three(lib, wl, steps):
    """Oracle, FP64 and FP32 models of the workload after `steps` update! steps."""
    ref, g64, g32 = oracle.from_workload(wl), _model(lib, wl, _abi.PI_FP64), _model(lib, wl, _abi.PI_FP32)
    vel = VelCache(wl)
    for m in (ref, g64, g32):
        drive(m, wl, steps, vel)
    return ref, g64, g32


@pytest.mark.slow
def test_config1_full_size_one_day(gpu_lib):
    wl = W.config1()
    assert (wl.grid.Nx, wl.grid.Ny, wl.grid.Nz, wl.N[0], wl.steps, wl.dT) == (128, 128, 1, 16384, 1440, 60.0)
    ref, g64, g32 = _three(gpu_lib, wl, wl.steps)
    assert compare_states(ref, g64, wl.nsp) == []
    assert g64.count_active(0) != 16384           # a day of divisions changed the population
    # 1440 FP32 steps: pointwise tracer differences grow to a few 1e-5 of the field's maximum while
    # the interior masses stay within TRACER_MASS_RTOL
    check_errors(errors_vs_oracle(ref, g32, wl), tracer_rel=1e-4)


def test_3d_two_species_64x64x32_bitexact(gpu_lib):
    over = {"dvid_P": [1e-4, 2e-4], "dvid_reg": [1.0, 1.1], "mort_P": [5e-5, 5e-5], "grz_P": [2e-6, 0.0]}
    wl = W.config2(nx=64, nz=32, N_per_species=50_000, steps=100, nmodes=64, seed=31, phyt_over=over)
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))          # start in daylight
    ref, g64 = oracle.from_workload(wl), _model(gpu_lib, wl, _abi.PI_FP64)
    vel = VelCache(wl)
    drive(ref, wl, 100, vel)
    drive(g64, wl, 100, vel)
    assert compare_states(ref, g64, wl.nsp) == []
    assert [g64.count_active(s) for s in range(2)] != [50_000, 50_000]


def _stretched(wl, size, zfaces, x, y, seed):
    """The workload's physics on a grid with the given vertical faces; state rebuilt on it, a
    double-gyre flow in x-y and a weak vertical velocity (zero at the surface and the bottom)."""
    rng = np.random.default_rng(seed)
    g = RectilinearGrid(size=size, x=x, y=y, z=np.asarray(zfaces, dtype=np.float64), FT=np.float64)
    wl.grid = g
    wl.individuals = [W.make_individuals(g, wl.phyt, s, wl.N[s], wl.capacity, rng) for s in range(wl.nsp)]
    wl.tracers = W.make_tracers(g, rng)
    u, v, _ = W.double_gyre(g, 0.02)
    w = np.zeros((g.Nx, g.Ny, g.Nz + 1), order="F")
    ii, jj = np.meshgrid(np.arange(g.Nx), np.arange(g.Ny), indexing="ij")
    for k in range(1, g.Nz):
        w[:, :, k] = 2e-4 * np.sin(2 * np.pi * (ii + 0.5) / g.Nx) * np.cos(2 * np.pi * (jj + 0.5) / g.Ny)
    wl.vel_fn = lambda t: (np.asfortranarray(u), np.asfortranarray(v), w)
    wl.parf = np.asfortranarray(np.roll(W.diel_parf(g.Nx, g.Ny, wl.parf.shape[2]), -10, axis=2))
    from PlanktonIndividuals.parameters import default_temperature
    wl.temp = default_temperature(g, wl.dT, wl.steps)
    return wl


OVER = {"dvid_P": [1e-3], "dvid_reg": [1.0], "mort_P": [5e-4], "mort_reg": [0.9], "grz_P": [2e-4]}


def test_reference_stretched_grid_through_steps(gpu_lib):
    wl = W.config1(n=8, N=200, steps=20, capacity=800, phyt_over=OVER)
    wl = _stretched(wl, (4, 6, 4), [0.0, -1.0, -3.0, -5.0, -10.0], (0.0, 12.0), (0.0, 12.0), seed=41)
    g = wl.grid
    assert g.Δx == 3.0 and g.Δy == 2.0
    assert list(g.dzC) == [1.0, 1.0, 1.5, 2.0, 3.5, 5.0, 5.0, 5.0]
    assert list(g.dzF) == [1.0, 1.0, 1.0, 2.0, 2.0, 5.0, 5.0, 5.0]
    ref, g64, g32 = _three(gpu_lib, wl, 20)
    assert compare_states(ref, g64, wl.nsp) == []
    check_errors(errors_vs_oracle(ref, g32, wl))


def test_stretched_3d_grid_through_steps(gpu_lib):
    wl = W.config1(n=8, N=3000, steps=25, capacity=9000, phyt_over=OVER)
    dz = np.linspace(1.0, 6.0, 10)
    zf = -np.concatenate([[0.0], np.cumsum(dz)])
    wl = _stretched(wl, (24, 24, 10), zf, (0.0, 24e2), (0.0, 24e2), seed=42)
    ref, g64, g32 = _three(gpu_lib, wl, 25)
    assert compare_states(ref, g64, wl.nsp) == []
    check_errors(errors_vs_oracle(ref, g32, wl))


@pytest.mark.slow
def test_config2_full_size_1000_steps_fp32_vs_fp64(gpu_lib):
    from PlanktonIndividuals.accuracy import fp32_vs_fp64
    wl = W.config2()
    assert (wl.grid.Nx, wl.grid.Ny, wl.grid.Nz, wl.nsp, wl.N[0], wl.dT) == (256, 256, 64, 2, 2_097_152, 30.0)
    r = fp32_vs_fp64(gpu_lib, wl, 1000, check_every=100)
    print({k: v for k, v in r.items() if k != "counts"})
    assert r["counts_equal_at_every_check"], r["counts"]
    assert r["max_tracer_mass_rel_err"] <= TRACER_MASS_RTOL
