"""FP32 form against the FP64 oracle, and the batched FP32 form against single FP32 models.

The FP32 form evaluates the reference formulas in Float32 with cell + offset positions and
fixed-point particle→grid sums, so it is compared with the oracle within stated tolerances:
  - population counts and the set of active slots: identical;
  - cell indices (xi, yi, zi): identical for at least 99.5 % of active individuals (a position
    within FP32 rounding of a cell face may land on the other side);
  - positions: max |Δx| ≤ 1e-3 grid cells;
  - individual quotas (Bm, Cq, Nq, Pq, Chl): max relative error ≤ 1e-4;
  - tracers: max |Δc| ≤ 1e-5 × max|c| per tracer; interior tracer mass Σ c·vol: relative
    error ≤ 1e-5.
Batch members and launch shapes must not change any bit (tolerance 0)."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals._native import CModel, CapacityError, PIError
from PlanktonIndividuals.batch import Member, PlanktonBatch
from helpers import VelCache, compare_states, drive

pytestmark = pytest.mark.gpu

TRACER_MASS_RTOL = 1e-5


def fp32_model(lib, wl):
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP32)
    m.set_state(wl.individuals, wl.tracers)
    return m


def daylight(wl):
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    return wl


def interior(grid, a):
    return a[grid.Hx:grid.Hx + grid.Nx, grid.Hy:grid.Hy + grid.Ny, grid.Hz:grid.Hz + grid.Nz]


def errors_vs_oracle(ref, f32, wl):
    """Per-output errors of the FP32 state against the FP64 oracle (dict)."""
    g = wl.grid
    out = {"count_fp64": [], "count_fp32": [], "ac_mismatch": 0, "cell_mismatch_frac": 0.0,
           "pos_abs": 0.0, "quota_rel": 0.0, "tracer_rel_max": 0.0, "mass_rel": {}}
    n_act = 0
    n_cell_bad = 0
    for s in range(wl.nsp):
        A, B = ref.get_individuals(s), f32.get_individuals(s)
        out["count_fp64"].append(int(A["ac"].sum()))
        out["count_fp32"].append(int(B["ac"].sum()))
        out["ac_mismatch"] += int(np.sum(A["ac"] != B["ac"]))
        both = A["ac"] & B["ac"]
        n_act += int(both.sum())
        same_cell = both & (A["xi"] == B["xi"]) & (A["yi"] == B["yi"]) & (A["zi"] == B["zi"])
        n_cell_bad += int(both.sum() - same_cell.sum())
        for k, N in (("x", g.Nx), ("y", g.Ny), ("z", g.Nz)):
            d = np.abs(A[k][both] - B[k][both])
            d = np.minimum(d, N - d) if k != "z" else d     # periodic wrap
            if d.size:
                out["pos_abs"] = max(out["pos_abs"], float(d.max()))
        for k in ("Bm", "Cq", "Nq", "Pq", "Chl"):
            a, b = A[k][both], B[k][both]
            if a.size:
                rel = np.abs(a - b) / np.maximum(np.abs(a), 1e-30)
                out["quota_rel"] = max(out["quota_rel"], float(rel.max()))
    out["cell_mismatch_frac"] = n_cell_bad / max(n_act, 1)
    vol = float(g.Δx) * float(g.Δy) * np.asarray(g.dzF)[g.Hz:g.Hz + g.Nz]
    for n, name in enumerate(_abi.tracer_names):
        a, b = interior(g, ref.get_tracer(n)), interior(g, f32.get_tracer(n))
        scale = max(float(np.abs(a).max()), 1e-300)
        out["tracer_rel_max"] = max(out["tracer_rel_max"], float(np.abs(a - b).max()) / scale)
        ma = float(np.sum(a * vol[None, None, :]))
        mb = float(np.sum(b * vol[None, None, :]))
        out["mass_rel"][name] = abs(ma - mb) / abs(ma) if ma != 0 else abs(mb)
    return out


def check_errors(e, tracer_rel=1e-5):
    """The FP32 bar: counts and active slots identical, cells identical for >= 99.5 %, positions within
    1e-3 cells, quotas within 1e-4 relative, each tracer within tracer_rel of its largest value
    (1e-5 for runs of tens of steps) and interior tracer masses within TRACER_MASS_RTOL."""
    print({k: v for k, v in e.items() if k != "mass_rel"})
    print("tracer mass relative error:", {k: f"{v:.2e}" for k, v in e["mass_rel"].items()})
    assert e["count_fp32"] == e["count_fp64"]
    assert e["ac_mismatch"] == 0
    assert e["cell_mismatch_frac"] <= 5e-3
    assert e["pos_abs"] <= 1e-3
    assert e["quota_rel"] <= 1e-4
    assert e["tracer_rel_max"] <= tracer_rel
    assert max(e["mass_rel"].values()) <= TRACER_MASS_RTOL


def test_fp32_config1_vs_oracle(gpu_lib):
    wl = daylight(W.config1(n=32, N=1024, steps=40))
    ref, f32 = oracle.from_workload(wl), fp32_model(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 40, vel)
    drive(f32, wl, 40, vel)
    check_errors(errors_vs_oracle(ref, f32, wl))


def test_fp32_divisions_deaths_grazing_vs_oracle(gpu_lib):
    over = {"dvid_P": [1e-3], "dvid_reg": [1.0], "mort_P": [5e-4], "mort_reg": [0.9], "grz_P": [2e-4]}
    wl = daylight(W.config1(n=24, N=1500, steps=60, capacity=6000, phyt_over=over))
    ref, f32 = oracle.from_workload(wl), fp32_model(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 60, vel)
    drive(f32, wl, 60, vel)
    e = errors_vs_oracle(ref, f32, wl)
    check_errors(e)
    assert e["count_fp32"][0] != 1500
    for k in (_abi.PI_DIAG_NUM, _abi.PI_DIAG_GRAZ, _abi.PI_DIAG_MORT, _abi.PI_DIAG_DVID):
        assert np.array_equal(ref.get_diag(k, 0).sum(), f32.get_diag(k, 0).sum())


def test_fp32_config2_small_3d_vs_oracle(gpu_lib):
    over = {"dvid_P": [1e-3, 2e-3], "dvid_reg": [1.0, 1.1], "mort_P": [3e-4, 3e-4], "grz_P": [1e-4, 0.0]}
    wl = daylight(W.config2(nx=16, nz=12, N_per_species=2500, steps=30, nmodes=24, phyt_over=over))
    wl.dT_vel = 10 * wl.dT
    ref, f32 = oracle.from_workload(wl), fp32_model(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 30, vel)
    drive(f32, wl, 30, vel)
    check_errors(errors_vs_oracle(ref, f32, wl))


def _fp32_pair(lib, wl, steps, setup=None):
    ref, f32 = oracle.from_workload(wl), fp32_model(lib, wl)
    if setup:
        setup(ref); setup(f32)
    vel = VelCache(wl)
    drive(ref, wl, steps, vel)
    drive(f32, wl, steps, vel)
    check_errors(errors_vs_oracle(ref, f32, wl))


def test_fp32_landmask_2d_vs_oracle(gpu_lib):
    from test_gpu_parity_edge import OVER, regrid
    from PlanktonIndividuals.grids import RectilinearGrid
    wl = W.config1(n=24, N=1200, steps=30, capacity=4000, phyt_over=OVER)
    lm = np.ones((24, 24, 1), dtype=bool)
    lm[5:9, 3:20, :] = False
    lm[15:17, 10:12, :] = False
    wl = regrid(wl, RectilinearGrid(size=(24, 24, 1), x=(0.0, 24e3), y=(0.0, 24e3), z=(0.0, -10.0),
                                    FT=np.float64, landmask=lm))
    _fp32_pair(gpu_lib, wl, 30)


def test_fp32_landmask_3d_vs_oracle(gpu_lib):
    from test_gpu_parity_edge import OVER, landmask_3d
    wl = landmask_3d(daylight(W.config2(nx=16, nz=10, N_per_species=900, nsp=1, steps=15, nmodes=12,
                                        phyt_over=OVER)))
    _fp32_pair(gpu_lib, wl, 15)


def test_fp32_bounded_xy_vs_oracle(gpu_lib):
    from test_gpu_parity_edge import OVER, regrid
    from PlanktonIndividuals.grids import Bounded, RectilinearGrid
    wl = W.config1(n=20, N=900, steps=25, capacity=3000, phyt_over=OVER)
    wl = regrid(wl, RectilinearGrid(size=(20, 20, 1), x=(0.0, 20e3), y=(0.0, 20e3), z=(0.0, -10.0),
                                    FT=np.float64, topology=(Bounded, Bounded, Bounded)))
    _fp32_pair(gpu_lib, wl, 25)


def test_fp32_bounded_xy_3d_vs_oracle(gpu_lib):
    """Bounded x/y on a 3D grid: every axis has at least H cells, so the halos are filled in one
    pass from their source cells (the 2D grid above keeps the three sequential passes)."""
    from test_gpu_parity_edge import OVER, regrid
    from PlanktonIndividuals.grids import Bounded, RectilinearGrid
    wl = W.config1(n=16, N=900, steps=20, capacity=3000, phyt_over=OVER)
    wl = regrid(wl, RectilinearGrid(size=(16, 16, 4), x=(0.0, 16e3), y=(0.0, 16e3), z=(0.0, -40.0),
                                    FT=np.float64, topology=(Bounded, Bounded, Bounded)))
    _fp32_pair(gpu_lib, wl, 20)


def test_fp32_flux_bcs_vs_oracle(gpu_lib):
    wl = daylight(W.config2(nx=12, nz=6, N_per_species=500, nsp=1, steps=12, nmodes=12))
    g = wl.grid
    rng = np.random.default_rng(0)
    west = np.asfortranarray(rng.uniform(0, 1e-3, (g.Ny, g.Nz)))
    bottom = np.asfortranarray(rng.uniform(0, 1e-5, (g.Nx, g.Ny, 20)))

    def setup(m):
        m.set_flux_bc(_abi.tracer_names.index("NO3"), _abi.FACES["top"], _abi.PI_BC_CONST, [1e-4])
        m.set_flux_bc(_abi.tracer_names.index("DIC"), _abi.FACES["west"], _abi.PI_BC_ARRAY2D, west)
        m.set_flux_bc(_abi.tracer_names.index("DON"), _abi.FACES["bottom"], _abi.PI_BC_ARRAY3D, bottom, 20)
    _fp32_pair(gpu_lib, wl, 12, setup)


def test_fp32_iron_and_sinking_vs_oracle(gpu_lib):
    from test_gpu_parity_edge import OVER, with_iron
    wl = with_iron(daylight(W.config2(nx=12, nz=10, N_per_species=600, nsp=1, steps=15, nmodes=12, phyt_over=OVER)))
    _fp32_pair(gpu_lib, wl, 15)


def test_fp32_diffusion_vs_oracle(gpu_lib):
    from test_gpu_parity_edge import DIFFUSION, OVER
    wl = daylight(W.config2(nx=12, nz=8, N_per_species=700, nsp=1, steps=15, nmodes=12, phyt_over=OVER))
    wl.bgc.update(DIFFUSION)
    _fp32_pair(gpu_lib, wl, 15)


def _members(wls):
    return [Member(wl.grid, wl.bgc, wl.phyt, wl.capacity, wl.seed) for wl in wls]


def _drive_batch(batch, wls, steps, vels):
    for _ in range(steps):
        _, t = batch.get_time()
        for m, wl in enumerate(wls):
            tv, tp, tt = int(np.floor(t / wl.dT_vel)), int(np.floor(t / wl.dT_PAR)), int(np.floor(t / wl.dT_temp))
            batch.set_velocity(m, *vels[m](tv))
            batch.set_PARF(m, wl.parf[:, :, tp])
            batch.set_temp(m, wl.temp[:, :, :, tt])
        batch.step(wls[0].dT, 1)


def _uneven_members():
    over = {"dvid_P": [1e-3, 2e-3], "dvid_reg": [1.0, 1.1], "mort_P": [3e-4, 3e-4], "grz_P": [1e-4, 0.0]}
    a = daylight(W.config2(nx=16, nz=12, N_per_species=2500, steps=20, nmodes=24, seed=11, phyt_over=over))
    b = daylight(W.config2(nx=24, nz=6, N_per_species=700, steps=20, nmodes=16, seed=12, phyt_over=over))
    c = daylight(W.config2(nx=8, nz=4, N_per_species=3000, steps=20, nmodes=8, seed=13, phyt_over=over))
    for wl in (a, b, c):
        wl.dT_vel = 5 * wl.dT
    return [a, b, c]


def test_batch_members_equal_single_fp32_models(gpu_lib):
    wls = _uneven_members()
    batch = PlanktonBatch(_members(wls), nspecies=2)
    for m, wl in enumerate(wls):
        batch.set_state(m, wl.individuals, wl.tracers)
    vels = [VelCache(wl) for wl in wls]
    _drive_batch(batch, wls, 20, vels)
    for m, wl in enumerate(wls):
        single = fp32_model(gpu_lib, wl)
        drive(single, wl, 20, vels[m])
        assert compare_states(single, batch.member(m), wl.nsp) == [], f"member {m}"


def _series(batch, m, wl, nsnap):
    vel = VelCache(wl)
    snaps = [vel(i) for i in range(nsnap)]
    vels = {c: np.stack([sn[q] for sn in snaps], axis=-1) for q, c in enumerate("uvw")}
    batch.set_series(m, vels=vels, ΔT_vel=wl.dT_vel, PARF=wl.parf, ΔT_PAR=wl.dT_PAR, temp=wl.temp,
                     ΔT_temp=wl.dT_temp)


def test_batch_graph_eager_and_autotuned_shapes_identical(gpu_lib):
    wls = _uneven_members()
    for wl in wls:
        wl.parf = np.asfortranarray(np.concatenate([wl.parf] * 3, axis=2))
        wl.temp = np.asfortranarray(np.concatenate([wl.temp] * 3, axis=3))

    def make():
        batch = PlanktonBatch(_members(wls), nspecies=2)
        for m, wl in enumerate(wls):
            batch.set_state(m, wl.individuals, wl.tracers)
            _series(batch, m, wl, 24)
        return batch

    tuned = make()
    report = tuned.autotune(wls[0].dT, steps_per_candidate=1)       # its steps are model steps
    n_tune, _ = tuned.get_time()
    assert report and 0 < n_tune < 100
    tuned.step(wls[0].dT, 10)
    graph = make()
    graph.step(wls[0].dT, n_tune + 10)
    eager = make()
    eager.profile_enable(True)
    eager.step(wls[0].dT, n_tune + 10)
    for b in (tuned, graph, eager):
        assert b.get_time()[0] == n_tune + 10
    for m, wl in enumerate(wls):
        assert compare_states(graph.member(m), eager.member(m), wl.nsp) == [], f"eager member {m}"
        assert compare_states(graph.member(m), tuned.member(m), wl.nsp) == [], f"autotuned member {m}"


def test_fp32_series_equals_step_by_step_forcing(gpu_lib):
    wls = _uneven_members()[:1]
    wl = wls[0]
    vel = VelCache(wl)
    a = PlanktonBatch(_members(wls), nspecies=2)
    a.set_state(0, wl.individuals, wl.tracers)
    _series(a, 0, wl, 5)
    a.step(wl.dT, 20)
    b = PlanktonBatch(_members(wls), nspecies=2)
    b.set_state(0, wl.individuals, wl.tracers)
    _drive_batch(b, wls, 20, [vel])
    assert compare_states(a.member(0), b.member(0), wl.nsp) == []


def test_fp32_capacity_error_message(gpu_lib):
    over = {"dvid_P": [5e-2], "dvid_reg": [0.5]}
    wl = daylight(W.config1(n=8, N=200, steps=50, capacity=210, phyt_over=over))
    f32 = fp32_model(gpu_lib, wl)
    with pytest.raises(CapacityError) as ei:
        drive(f32, wl, 50)
    it, _ = f32.get_time()
    msg = str(ei.value)
    assert msg.startswith("number of individual exceeds the capacity at timestep ")
    assert msg == f"number of individual exceeds the capacity at timestep {it * wl.dT / 86400!r} days"


def test_fp32_budget_matches_downloaded_fields(gpu_lib):
    wls = _uneven_members()[1:2]
    wl = wls[0]
    batch = PlanktonBatch(_members(wls), nspecies=2)
    batch.set_state(0, wl.individuals, wl.tracers)
    _drive_batch(batch, wls, 5, [VelCache(wl)])
    bud = batch.budget(0)
    g = wl.grid
    vol = float(g.Δx) * float(g.Δy) * np.asarray(g.dzF)[g.Hz:g.Hz + g.Nz]
    tot = lambda names: sum(float(np.sum(interior(g, batch.get_tracer(0, _abi.tracer_names.index(n))) * vol)) for n in names)
    assert bud["tracer_C"] == pytest.approx(tot(("DIC", "DOC", "POC")), rel=1e-12)
    assert bud["tracer_N"] == pytest.approx(tot(("NH4", "NO3", "DON", "PON")), rel=1e-12)
    assert bud["tracer_P"] == pytest.approx(tot(("PO4", "DOP", "POP")), rel=1e-12)
    C = 0.0
    for s in range(2):
        d = batch.get_individuals(0, s)
        C += float(np.sum((d["Bm"] + d["Cq"])[d["ac"]]))
    assert bud["ind_C"] == pytest.approx(C, rel=1e-6)


def test_fp32_position_just_below_a_cell_face(gpu_lib):
    """An uploaded position within an FP32 rounding of the next cell face (z = 1 − 2e-9 in a
    one-level box) keeps the cell the Float64 position has, and later steps stay in the grid."""
    wl = W.config5(n_max=1)[0]
    d = wl.individuals[0]
    N = wl.N[0]
    d["z"][:N] = np.minimum(d["z"][:N], 0.5)
    d["z"][0] = 1.0 - 2e-9
    d["x"][1] = 1.0 - 1e-9
    ref, f32 = oracle.from_workload(wl), fp32_model(gpu_lib, wl)
    vel = VelCache(wl)
    drive(ref, wl, 5, vel)
    drive(f32, wl, 5, vel)
    A, B = ref.get_individuals(0), f32.get_individuals(0)
    assert np.array_equal(A["ac"], B["ac"])
    for k in ("xi", "yi", "zi"):
        assert np.array_equal(A[k][A["ac"]], B[k][B["ac"]]), k


def test_storage_order_changes_no_result(gpu_lib):
    """The stored order of individuals (grouped by cell by a periodic counting sort) is invisible:
    runs that never sort, sort before every step, or sort every few steps give identical bits for
    every attribute, tracer, diagnostic and budget, with divisions, deaths and grazing happening
    (draws are keyed by slot number, divisions assigned in slot order)."""
    wls = _uneven_members()
    runs = []
    for interval in (0, 1, 7, 32):
        batch = PlanktonBatch(_members(wls), nspecies=2)
        batch.set_sort_interval(interval)
        for m, wl in enumerate(wls):
            batch.set_state(m, wl.individuals, wl.tracers)
        _drive_batch(batch, wls, 20, [VelCache(wl) for wl in wls])
        runs.append(batch)
    for m, wl in enumerate(wls):
        n0 = sum(int(wl.individuals[s]["ac"].sum()) for s in range(wl.nsp))
        assert sum(runs[0].member(m).count_active(s) for s in range(wl.nsp)) != n0
        for r in runs[1:]:
            assert compare_states(runs[0].member(m), r.member(m), wl.nsp) == [], f"member {m}"
            assert np.array_equal(runs[0].budget(m), r.budget(m))


def test_fused_tracer_kernel_equals_two_kernel_path(gpu_lib):
    """k32_tracer (x, y and z sweeps, sinking, forcing, particle terms and the halo fill in one walk
    down the levels, tracers staged by TMA or, for row pitches that are not a multiple of 16 bytes,
    by cp.async) against the two-kernel path (k32_xy + k32_ztail + halo fill), tolerance 0. The
    second run re-uploads its tracers before every step, which makes that step take the two-kernel
    path. Members: a 3D land mask, Bounded x/y, iron tracers with sinking, a grid whose rows are not
    16-byte multiples, and a grid of two x tiles and two runs of levels."""
    from test_gpu_parity_edge import OVER, landmask_3d, regrid, with_iron
    from PlanktonIndividuals.grids import Bounded, RectilinearGrid
    a = with_iron(daylight(W.config2(nx=13, nz=9, N_per_species=800, nsp=1, steps=12, nmodes=12, seed=21, phyt_over=OVER)))
    b = landmask_3d(daylight(W.config2(nx=16, nz=10, N_per_species=900, nsp=1, steps=12, nmodes=12, seed=22, phyt_over=OVER)))
    c = W.config1(n=20, N=900, steps=12, capacity=3000, phyt_over=OVER)
    c = regrid(c, RectilinearGrid(size=(20, 12, 5), x=(0.0, 20e3), y=(0.0, 12e3), z=(0.0, -50.0),
                                  FT=np.float64, topology=(Bounded, Bounded, Bounded)))
    d = with_iron(daylight(W.config2(nx=36, nz=40, N_per_species=2000, nsp=1, steps=12, nmodes=12, seed=24, phyt_over=OVER)))
    wls = [a, b, c, d]
    assert a.grid.total_size[0] % 4 != 0 and d.grid.total_size[0] % 4 == 0
    vels = [VelCache(wl) for wl in wls]
    fused = PlanktonBatch(_members(wls), nspecies=1)
    plain = PlanktonBatch(_members(wls), nspecies=1)
    fused.set_tracer_kernel(True, 32)
    plain.set_tracer_kernel(False)
    for batch in (fused, plain):
        for m, wl in enumerate(wls):
            batch.set_state(m, wl.individuals, wl.tracers)
    for step in range(12):
        for m in range(len(wls)):
            for n in range(_abi.NTRACERS):
                plain.set_tracer(m, n, plain.get_tracer(m, n))
        _drive_batch(plain, wls, 1, vels)
        _drive_batch(fused, wls, 1, vels)
    for m, wl in enumerate(wls):
        assert compare_states(plain.member(m), fused.member(m), wl.nsp) == [], f"member {m}"


def test_async_float32_setters_equal_sync_path(gpu_lib):
    """The overlapped input path of an FP32 model (pi_set_velocity/PARF/temp_f32 from Float32 host
    arrays, copies on their own stream; pi_time_step_async; pi_count_active_async) against the
    synchronous Float64 path, tolerance 0: a Float32 array is what the device makes of the Float64
    one. The velocity changes every third step, sometimes twice between two steps, to exercise the
    choice of the velocity buffer that the queued steps are not using."""
    import ctypes as ct
    import torch
    wl = daylight(W.config2(nx=16, nz=8, N_per_species=1500, steps=16, nmodes=12, seed=61))
    wl.dT_vel = 3 * wl.dT
    vel = VelCache(wl)
    a, b = fp32_model(gpu_lib, wl), fp32_model(gpu_lib, wl)
    f32 = lambda x: np.asfortranarray(np.asarray(x, dtype=np.float32))
    p = lambda x: ct.c_void_p(x.ctypes.data)
    counts = torch.zeros(16 * wl.nsp, dtype=torch.int64, pin_memory=True)
    keep = []
    for i in range(16):
        t = i * wl.dT
        tv, tp, tt = int(t // wl.dT_vel), int(t // wl.dT_PAR), int(t // wl.dT_temp)
        a.set_velocity(*vel(tv)); a.set_PARF(wl.parf[:, :, tp]); a.set_temp(wl.temp[:, :, :, tt])
        a.time_step(wl.dT)
        if i % 5 == 2:      # a velocity replaced before the step: the second one counts
            junk = tuple(f32(x * 0.5) for x in vel(tv))
            keep.append(junk)
            assert gpu_lib.pi_set_velocity_f32(b.h, *(p(x) for x in junk)) == 0
        u, v, w = (f32(x) for x in vel(tv))
        par, tmp = f32(wl.parf[:, :, tp]), f32(wl.temp[:, :, :, tt])
        keep.append((u, v, w, par, tmp))
        assert gpu_lib.pi_set_velocity_f32(b.h, p(u), p(v), p(w)) == 0
        assert gpu_lib.pi_set_PARF_f32(b.h, p(par)) == 0
        assert gpu_lib.pi_set_temp_f32(b.h, p(tmp)) == 0
        assert gpu_lib.pi_time_step_async(b.h, ct.c_double(wl.dT)) == 0
        for s in range(wl.nsp):
            assert gpu_lib.pi_count_active_async(b.h, s, ct.c_void_p(counts.data_ptr() + 8 * (i * wl.nsp + s))) == 0
    assert gpu_lib.pi_synchronize(b.h) == 0
    assert compare_states(a, b, wl.nsp) == []
    assert [int(c) for c in counts[-wl.nsp:]] == [a.count_active(s) for s in range(wl.nsp)]


def test_launch_options_change_no_result(gpu_lib):
    """Every launch-shape option (register fits, blocks per SM, tile rows, z walk length, PAR warps,
    the x-y kernel on a second graph branch beside the particle kernels) gives the same bits."""
    wls = _uneven_members()
    runs = []
    for opts in ({}, {"xy_beside_particles": 1, "move_fit": 3, "physiology_fit": 2, "xy_rows": 8,
                      "z_levels": 16, "par_warps": 4, "move_blocks_per_sm": 0, "physiology_blocks_per_sm": 2}):
        batch = PlanktonBatch(_members(wls), nspecies=2)
        for k, v in opts.items():
            batch.set_option(k, v)
        for m, wl in enumerate(wls):
            batch.set_state(m, wl.individuals, wl.tracers)
        _drive_batch(batch, wls, 15, [VelCache(wl) for wl in wls])
        runs.append(batch)
    for m, wl in enumerate(wls):
        assert compare_states(runs[0].member(m), runs[1].member(m), wl.nsp) == [], f"member {m}"
    with pytest.raises(PIError):
        runs[0].set_option("xy_rows", 5)
