"""The drop-in API on the GPU, used as a user of the reference would use it:

    grid  = RectilinearGrid(size, x, y, z; FT)
    model = PlanktonModel(GPU(), grid; FT, max_individuals, phyto = phyto_setup(params, N, Nsp))
    sim   = PlanktonSimulation(model; ΔT, iterations, PARF, vels, ΔT_vel)
    update!(sim)
    sim.diags (PlanktonDiagnostics), model.individuals.phytos.sp1.data, model.tracers.NO3.data

against the CPU oracle started from the model's initial state and driven with the snapshots that
update! selects (src/Simulation/update.jl:14-26). FT = Float64: identical bits (tolerance 0) for
every attribute, tracer and diagnostic, and model.t / model.iteration; FT = Float32: within the
FP32 bounds of test_gpu_fp32.py.
"""
import math
from types import SimpleNamespace

import numpy as np
import pytest

import oracle
from PlanktonIndividuals import (GPU, PlanktonModel, PlanktonSimulation, RectilinearGrid, default_PARF,
                                 phyto_setup, tracer_names, update_b)
from PlanktonIndividuals import _abi, workloads as W
from helpers import same
from test_gpu_fp32 import check_errors, errors_vs_oracle

pytestmark = pytest.mark.gpu

STEPS = 25
PARAMS = {"dvid_P": 1e-3, "dvid_reg": 1.0, "mort_P": 5e-4, "mort_reg": 0.9, "grz_P": 2e-5}


def _setup(FT):
    grid = RectilinearGrid(size=(16, 16, 8), x=(0.0, 800.0), y=(0.0, 800.0), z=(0.0, -16.0), FT=FT)
    model = PlanktonModel(GPU(), grid, FT=FT, max_individuals=6000,
                          phyto=phyto_setup(dict(PARAMS), [2000], 1), seed=7)
    fv = W.FourierVelocity(grid, nmodes=16, rms=0.02, seed=3)
    snaps = [fv(i) for i in range(3)]
    vels = {c: np.stack([s[q] for s in snaps], axis=-1) for q, c in enumerate("uvw")}
    parf = np.asfortranarray(np.roll(default_PARF(grid, 60.0, STEPS), -10, axis=2))
    # the oracle starts from the model's own initial state
    inds = [dict(model.individuals.phytos.sp1.data)]
    trs = [model.tracers[name].data for name in tracer_names]
    ref = oracle.OracleModel(grid, model.bgc_params, model.phyto.params, 1, 6000, 7)
    ref.set_state(inds, trs)
    sim = PlanktonSimulation(model, ΔT=60.0, iterations=STEPS, PARF=parf, vels=vels, ΔT_vel=600.0)
    return grid, model, sim, ref


def _drive_like_update(ref, sim, steps):
    inp = sim.input
    for _ in range(steps):
        _, t = ref.get_time()
        tv, tp, tt = (int(math.floor(t / inp[k])) for k in ("ΔT_vel", "ΔT_PAR", "ΔT_temp"))
        ref.set_velocity(*(np.asfortranarray(np.asarray(inp["vels"][c])[..., tv]) for c in "uvw"))
        ref.set_PARF(inp["PARF"][:, :, tp])
        ref.set_temp(inp["temp"][:, :, :, tt])
        ref.time_step(sim.ΔT)


def test_api_fp64_bitexact_with_oracle(gpu_lib):
    grid, model, sim, ref = _setup(np.float64)
    update_b(sim)
    _drive_like_update(ref, sim, STEPS)
    assert model.iteration == STEPS and model.t == STEPS * 60.0
    A, B = ref.get_individuals(0), model.individuals.phytos.sp1.data
    for k in A:
        assert same(A[k], B[k]), k
    for n, name in enumerate(tracer_names):
        assert same(ref.get_tracer(n), model.tracers[name].data), name
    d = sim.diags
    assert same(ref.get_diag(_abi.PI_DIAG_PAR, 0), d.tracer.PAR)
    for key, kind in (("num", _abi.PI_DIAG_NUM), ("graz", _abi.PI_DIAG_GRAZ), ("mort", _abi.PI_DIAG_MORT),
                      ("dvid", _abi.PI_DIAG_DVID)):
        assert same(ref.get_diag(kind, 0), getattr(d.phytos.sp1, key)), key
    assert d.phytos.sp1.ptc.shape == grid.total_size and not d.phytos.sp1.ptc.any()
    assert model.count_active() != [2000]
    sim.close()


def test_api_fp32_within_bounds(gpu_lib):
    grid, model, sim, ref = _setup(np.float32)
    update_b(sim)
    _drive_like_update(ref, sim, STEPS)
    assert model.iteration == STEPS
    check_errors(errors_vs_oracle(ref, model._native, SimpleNamespace(grid=grid, nsp=1)))
    sim.close()


def test_simulation_with_output_writer(gpu_lib, tmp_path):
    """update!(sim) with an output writer: a write_output! after every step (update.jl:30); the
    last archived individuals equal the model's, the averaged diagnostics have the interior shape
    and the species log has one line per step. The steps run one pi_sim_update_steps call each and
    give the same state as a single update! call."""
    from PlanktonIndividuals import PlanktonDiagnostics, PlanktonOutputWriter
    from PlanktonIndividuals.output import read_archive
    grid, model, sim, ref = _setup(np.float64)
    w = PlanktonOutputWriter(dir=str(tmp_path / "out"), write_log=True, save_diags=True, save_phytoplankton=True,
                             phytoplankton_include=("x", "y", "z", "Bm", "ac"))
    sim.output_writer = w
    sim.diags = PlanktonDiagnostics(model, tracer=("NO3",), phytoplankton=("num", "PS"), iteration_interval=5)
    update_b(sim)
    _drive_like_update(ref, sim, STEPS)
    A = ref.get_individuals(0)
    for k in A:
        assert same(A[k], model.individuals.phytos.sp1.data[k]), k
    ph = read_archive(w.phytoplankton_file)
    for k in ("x", "y", "z", "Bm", "ac"):
        assert same(ph[f"timeseries/sp1/{k}/{STEPS}"], A[k]), k
    dg = read_archive(w.diags_file)
    assert dg[f"timeseries/NO3/{STEPS}"].shape == (16, 16, 8)
    assert f"timeseries/phyto/sp1/PS/{STEPS}" in dg and f"timeseries/PAR/5" in dg
    lines = open(str(tmp_path / "out" / "dynamic_species001.txt")).read().splitlines()
    assert len(lines) == STEPS
    sim.close()


@pytest.mark.parametrize("FT", [np.float64, np.float32])
def test_model_budget_matches_downloaded_state(gpu_lib, FT):
    """pi_get_budget on a model handle (either precision): the interior tracer C, N, P and the
    active individuals' C, N, P equal the sums over the downloaded fields and attributes."""
    grid, model, sim, _ = _setup(FT)
    update_b(sim)
    bud = model._native.budget()
    g = grid
    vol = float(g.Δx) * float(g.Δy) * np.asarray(g.dzF)[g.Hz:g.Hz + g.Nz]
    inner = lambda a: np.asarray(a, dtype=np.float64)[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz]
    tot = lambda names: sum(float(np.sum(inner(model.tracers[n].data) * vol)) for n in names)
    d = {k: np.asarray(v, dtype=np.float64) for k, v in model.individuals.phytos.sp1.data.items()}
    ac = np.asarray(model.individuals.phytos.sp1.data["ac"], dtype=bool)
    p = model.phyto.params
    R_NC, R_PC = float(np.ravel(p["R_NC"])[0]), float(np.ravel(p["R_PC"])[0])
    want = [tot(("DIC", "DOC", "POC")), tot(("NH4", "NO3", "DON", "PON")), tot(("PO4", "DOP", "POP")),
            float(np.sum((d["Bm"] + d["Cq"])[ac])), float(np.sum((d["Bm"] * R_NC + d["Nq"])[ac])),
            float(np.sum((d["Bm"] * R_PC + d["Pq"])[ac]))]
    rel = 1e-12 if FT is np.float64 else 1e-6
    for a, b in zip(bud, want):
        assert a == pytest.approx(b, rel=rel)
