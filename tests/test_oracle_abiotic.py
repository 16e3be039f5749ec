"""Abiotic particles (src/Individuals/Abiotic/) in the CPU oracle: the parameters and setup of
abiotic_setup/PlanktonModel, the reference's own 2D example with abiotic particles on
(test/example_2D_test.jl), and known answers for each pass — particles_from_bcs!, the
interaction (against a literal transcription of calc_interaction_kernel! and
merge_particle_kernel! run as a single thread would) and particle_release! with its draws."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import _abi, abiotic_params_default, update_abiotic_params, update_bgc_params, update_phyt_params
from PlanktonIndividuals import grids as G
from PlanktonIndividuals import workloads as W
from PlanktonIndividuals._native import CapacityError, PIError
from PlanktonIndividuals.grids import Bounded, Periodic, RectilinearGrid
from PlanktonIndividuals.init import generate_tracers, initialize_abiotic_particle, initialize_plankton
from PlanktonIndividuals.parameters import default_tracer_init
from PlanktonIndividuals.stepping import VelCache, drive

SEED = 9


def test_abiotic_parameters_and_initialisation():
    p = abiotic_params_default(2)
    assert list(p) == list(_abi.ABIOTIC_FIELDS) == [f for f, _ in _abi.pi_abiotic_params._fields_]
    assert p == {"Nsuper": [1.0, 1.0], "Rd": [1.0e-4] * 2, "release_P": [1.0e-6] * 2, "sz_min": [1.0e-3] * 2,
                 "Ktr": [0.0, 0.0]}
    assert update_abiotic_params({"Rd": [2.0, 3.0]}, np.float64, N=2)["Rd"] == [2.0, 3.0]
    with pytest.raises(ValueError, match="abiotic parameter not found"):
        update_abiotic_params({"max_ptc": [1]}, np.float64, N=1)
    grid = RectilinearGrid(size=(8, 6, 4), x=(0, 80), y=(0, 60), z=(0, -8), FT=np.float64)
    d = initialize_abiotic_particle(grid, 300, 500, np.random.default_rng(1))
    a = d["ac"]
    assert a[:300].all() and not a[300:].any()
    assert np.all((d["x"][a] >= 0) & (d["x"][a] < 8) & (d["y"][a] < 6) & (d["z"][a] < 4))
    assert not np.any(d["x"][~a]) and not np.any(d["xi"])         # cell indices as constructed


def _reference_2d_example(with_abiotic=True):
    """test/example_2D_test.jl: RectilinearGrid(size = (16, 16, 1), x = (0,32), y = (0,32),
    z = (0,-32)), PlanktonModel(CPU(), grid; abiotic = abiotic_setup(nothing, [2^10, 2^10], 2,
    Palat([(:sp1, :sa1)], [(:sp1, :sa1)]))), velocities randn·1e-4, ΔT = 60, 10 iterations."""
    grid = RectilinearGrid(size=(16, 16, 1), x=(0, 32), y=(0, 32), z=(0, -32), FT=np.float64)
    rng = np.random.default_rng(SEED)
    C = 8 * 1024
    bgc = update_bgc_params({}, np.float64)
    phyt = update_phyt_params({}, np.float64, N=1)
    m = oracle.OracleModel(grid, bgc, phyt, 1, C, SEED)
    m.set_state([initialize_plankton(grid, phyt, 0, 2 ** 10, C, rng)],
                generate_tracers(grid, default_tracer_init(), rng))
    parts = [initialize_abiotic_particle(grid, 2 ** 10, C, rng) for _ in range(2)]
    if with_abiotic:
        m.set_abiotics(update_abiotic_params(abiotic_params_default(2), np.float64, N=2), 2, [(0, 0)], [(0, 0)])
        for a in range(2):
            m.set_abiotic_particles(a, parts[a])
    vels = [(rng.standard_normal((16, 16, 1)) * 1e-4, rng.standard_normal((16, 16, 1)) * 1e-4,
             rng.standard_normal((16, 16, 2)) * 1e-4) for _ in range(11)]
    return grid, phyt, m, vels


def _total_P(m, grid, phyt):
    vol = G.interior(G.cell_volumes(grid), grid)
    tp = sum(float(np.sum(G.interior(m.get_tracer(_abi.tracer_names.index(n)), grid) * vol)) for n in ("PO4", "DOP", "POP"))
    d = m.get_individuals(0)
    return tp + float(np.sum(d["Pq"] + d["Bm"] * phyt["R_PC"][0]))


def _run_2d(m, vels):
    parf = np.full((16, 16), 300.0)
    for it in range(10):
        _, t = m.get_time()
        m.set_velocity(*vels[int(t // 60.0)])             # ΔT_vel = ΔT: one snapshot per step
        m.set_PARF(parf)
        m.time_step(60.0)


def test_reference_2d_example_with_abiotic_particles():
    """The reference's check, isapprox(TP, TPt; atol = 1e1), with the abiotic particles stepped.
    At the default Rd = 1e-4 m no particle merges, so the phytoplankton and the tracers end
    exactly as in the same run without abiotic particles."""
    grid, phyt, m, vels = _reference_2d_example()
    TP = _total_P(m, grid, phyt)
    a0 = m.get_abiotic_particles(0)
    _run_2d(m, vels)
    TPt = _total_P(m, grid, phyt)
    assert abs(TPt - TP) <= 1e1
    _, _, twin, _ = _reference_2d_example(with_abiotic=False)
    _run_2d(twin, vels)
    for n in range(_abi.NTRACERS):
        assert np.array_equal(m.get_tracer(n), twin.get_tracer(n))
    p, q = m.get_individuals(0), twin.get_individuals(0)
    assert all(np.array_equal(p[k], q[k]) for k in q)
    a1 = m.get_abiotic_particles(0)
    assert m.count_abiotic(0) == m.count_abiotic(1) == 2 ** 10       # no merges, no releases
    assert np.any(a1["x"][a1["ac"]] != a0["x"][a0["ac"]])            # advected and diffused
    assert np.all((a1["xi"][a1["ac"]] >= 3) & (a1["xi"][a1["ac"]] <= 18))
    assert m.get_diag(_abi.PI_DIAG_ABIO_NUM, 0).sum() == 10 * 2 ** 10
    assert not m.get_diag(_abi.PI_DIAG_PTC, 0).any()


def _static_model(grid, C, nsp=1, phyt_over=None):
    """A model whose particles stay where they are for a step: zero velocity and diffusivity, no
    grazing, mortality or division, so each pass can be checked against positions set by hand."""
    over = {"grz_P": [0.0] * nsp, "mort_P": [0.0] * nsp, "dvid_P": [0.0] * nsp}
    over.update(phyt_over or {})
    bgc = update_bgc_params({"κhP": 0.0, "κvP": 0.0}, np.float64)
    phyt = update_phyt_params(over, np.float64, N=nsp)
    m = oracle.OracleModel(grid, bgc, phyt, nsp, C, SEED)
    rng = np.random.default_rng(3)
    m.set_state([initialize_plankton(grid, phyt, s, 0, C, rng) for s in range(nsp)],
                generate_tracers(grid, default_tracer_init(), rng))
    g = grid
    b = [int(t == _abi.PI_BOUNDED) for t in g.topo]
    m.set_velocity(np.zeros((g.Nx + b[0], g.Ny, g.Nz)), np.zeros((g.Nx, g.Ny + b[1], g.Nz)),
                   np.zeros((g.Nx, g.Ny, g.Nz + b[2])))
    m.set_PARF(np.full((g.Nx, g.Ny), 200.0))
    return m, phyt


def _planks(m, phyt, C, x, y, z, ptc=None):
    from PlanktonIndividuals.init import empty_individuals
    d = initialize_plankton(m.grid, phyt, 0, len(x), C, np.random.default_rng(4))
    n = len(x)
    d["ac"][:] = False
    d["ac"][:n] = True
    for k, v in (("x", x), ("y", y), ("z", z)):
        d[k] = np.zeros(C)
        d[k][:n] = v
    d["ptc"] = np.zeros(C) if ptc is None else np.asarray(ptc, dtype=np.float64)
    for k in ("graz", "mort", "dvid"):
        d[k] = np.zeros(C)
    m.set_individuals(0, d)
    return d


def _abiotics(m, sa, C, x, y, z):
    n = len(x)
    d = {"ac": np.zeros(C, dtype=np.uint8)}
    d["ac"][:n] = 1
    for k, v in (("x", x), ("y", y), ("z", z)):
        d[k] = np.zeros(C)
        d[k][:n] = v
    m.set_abiotic_particles(sa, d)
    return d


def _find_inds(v, H):
    return np.trunc(v + 1.0).astype(np.int64) + H


def _literal_interaction(g, pl, ab, Rd, maxc, max_ptc, C):
    """calc_interaction_kernel! then merge_particle_kernel! (particle_interaction.jl:24-66) as
    plain loops over 1-based indices, in the order a single thread runs them."""
    intac = np.zeros((maxc, C), dtype=np.int64)
    for i in range(1, C + 1):
        if not pl["ac"][i - 1]:
            continue
        for k in range(1, C + 1):
            if not ab["ac"][k - 1]:
                continue
            same = all(pl[c][i - 1] == ab[c][k - 1] for c in ("xi", "yi", "zi"))
            if same:
                dx = (pl["x"][i - 1] - ab["x"][k - 1]) * g.Δx
                dy = (pl["y"][i - 1] - ab["y"][k - 1]) * g.Δy
                dz = (pl["z"][i - 1] - ab["z"][k - 1]) * float(np.asarray(g.dzF)[pl["zi"][i - 1] - 1])
                dist = np.sqrt(dx * dx + dy * dy + dz * dz)
            else:
                dist = np.float64(np.float32(1.0e20))
            if dist < Rd:
                intac[(i % maxc), k - 1] = i
    ptc, ac = pl["ptc"].copy(), ab["ac"].astype(bool).copy()
    for k in range(1, C + 1):
        if ac[k - 1]:
            for j in range(1, maxc + 1):
                pid = intac[j - 1, k - 1]
                if pid > 0 and ptc[pid - 1] < max_ptc:
                    ptc[pid - 1] += 1.0
                    ac[k - 1] = False
                    break
    return ptc, ac


@pytest.mark.parametrize("maxc,max_ptc", [(5, 2.0), (25, 25.0), (1, 1.0)])
def test_interaction_matches_the_literal_kernels(maxc, max_ptc):
    """Crowded cells (1 km, Rd = 600 m) so that candidate slots i % max_candidates collide, rows
    fill up and max_ptc caps; particles in neighbouring cells never interact however close."""
    grid = RectilinearGrid(size=(4, 4, 2), x=(0, 4000), y=(0, 4000), z=(0, -20), FT=np.float64)
    C = 96
    rng = np.random.default_rng(maxc)
    m, phyt = _static_model(grid, C)
    m.set_abiotics({"Nsuper": [1.0], "Rd": [600.0], "release_P": [0.0], "sz_min": [1e-3], "Ktr": [0.0]}, 1,
                   intac=[(0, 0)], release=[], max_candidates=maxc, max_ptc=[max_ptc])
    cx = lambda n: rng.choice([0.05, 0.5, 0.95, 1.02, 1.5, 2.5], n) + rng.random(n) * 0.04
    npl, nab = 60, 80
    pl = _planks(m, phyt, C, cx(npl), cx(npl), rng.random(npl) * 2.0)
    ab = _abiotics(m, 0, C, cx(nab), cx(nab), rng.random(nab) * 2.0)
    for d in (pl, ab):
        for c, H, ax in (("xi", grid.Hx, "x"), ("yi", grid.Hy, "y"), ("zi", grid.Hz, "z")):
            d[c] = np.where(d["ac"].astype(bool), _find_inds(d[ax], H), H)
    ptc_exp, ac_exp = _literal_interaction(grid, pl, ab, 600.0, maxc, max_ptc, C)
    m.time_step(60.0)
    got_p, got_a = m.get_individuals(0), m.get_abiotic_particles(0)
    assert np.array_equal(got_p["x"], pl["x"]) and np.array_equal(got_a["x"], ab["x"])      # nothing moved
    assert np.array_equal(got_p["ptc"], ptc_exp)
    assert np.array_equal(got_a["ac"], ac_exp)
    assert 0 < ptc_exp.sum() < nab and ptc_exp.max() <= max_ptc
    d = m.get_diag(_abi.PI_DIAG_PTC, 0)
    cells = [grid_id(grid, *(got_p[c][i] for c in ("xi", "yi", "zi"))) for i in range(npl)]
    ref = np.zeros(d.size)
    np.add.at(ref, cells, ptc_exp[:npl])
    assert np.array_equal(d.ravel(order="F"), ref)


def grid_id(g, i, j, k):
    Gx, Gy = g.Nx + 2 * g.Hx, g.Ny + 2 * g.Hy
    return (i - 1) + Gx * ((j - 1) + Gy * (k - 1))


def test_release_takes_free_slots_in_order_at_the_drawn_offsets():
    """particle_release!: rnd.x < release_P·ΔT·ptc releases one particle into the next free slot
    at the phytoplankton's position plus the release draw in x and the last species' mortality and
    division draws in y and z; ptc drops by one; the particle's cell indices stay stale."""
    grid = RectilinearGrid(size=(4, 4, 2), x=(0, 4000), y=(0, 4000), z=(0, -20), FT=np.float64)
    C, nsp = 64, 2
    m, phyt = _static_model(grid, C, nsp=nsp)
    rP = 0.3 / 60.0
    m.set_abiotics({"Nsuper": [1.0], "Rd": [1e-4], "release_P": [rP], "sz_min": [1e-3], "Ktr": [0.0]}, 1,
                   intac=[], release=[(0, 0)], max_ptc=[np.nan, np.nan])
    rng = np.random.default_rng(8)
    n = 40
    ptc = np.zeros(C)
    ptc[:n] = rng.integers(0, 4, n)
    pl = _planks(m, phyt, C, rng.random(n) * 4, rng.random(n) * 4, rng.random(n) * 2, ptc=ptc)
    occupied = np.zeros(C, dtype=bool)
    occupied[[0, 1, 5, 9]] = True
    ab = {"ac": occupied.astype(np.uint8), "x": np.where(occupied, 1.5, 0.0), "y": np.where(occupied, 1.5, 0.0),
          "z": np.where(occupied, 0.5, 0.0)}
    m.set_abiotic_particles(0, ab)
    m.time_step(60.0)
    it, _ = m.get_time()
    dec = [oracle.draw3(SEED, it, nsp - 1, _abi.PI_DRAW_DECISION, i) for i in range(C)]
    rel = [oracle.draw3(SEED, it, 0, _abi.PI_DRAW_RELEASE, i)[0] for i in range(C)]
    R = [i for i in range(C) if pl["ac"][i] and rel[i] < rP * 60.0 * ptc[i]]
    free = [k for k in range(C) if not occupied[k]]
    a, p = m.get_abiotic_particles(0), m.get_individuals(0)
    assert 5 < len(R) < n
    assert int(a["ac"].sum()) == 4 + len(R)
    for i, d in zip(R, free):
        assert a["ac"][d]
        assert a["x"][d] == pl["x"][i] + rel[i] and a["y"][d] == pl["y"][i] + dec[i][1]
        assert a["z"][d] == pl["z"][i] + dec[i][2]
        assert (a["xi"][d], a["yi"][d], a["zi"][d]) == (grid.Hx, grid.Hy, grid.Hz)
    exp = ptc.copy()
    exp[R] -= 1.0
    assert np.array_equal(p["ptc"], exp)


def test_particles_from_bcs_faces_order_and_positions():
    """particles_from_bcs!: on a one-level grid the top and bottom faces share their cells and the
    later face (bottom) decides; the east face then overwrites its column. New particles fill the
    free slots in column-major cell order at cell − halo − 0.4 (Float32)."""
    grid = RectilinearGrid(size=(5, 3, 1), x=(0, 500), y=(0, 300), z=(0, -10), FT=np.float64,
                           topology=(Bounded, Periodic, Bounded))
    C = 64
    m, phyt = _static_model(grid, C)
    sz, Ns = 1e-3, 2.0
    m.set_abiotics({"Nsuper": [Ns], "Rd": [1e-4], "release_P": [0.0], "sz_min": [sz], "Ktr": [0.0]}, 1,
                   max_ptc=[np.nan])
    _abiotics(m, 0, C, [0.5, 1.5], [0.5, 0.5], [0.2, 0.2])
    top, east = 1.0, 2.0e-8                           # top alone would fill every cell
    bottom = np.asfortranarray(np.random.default_rng(2).random((5, 3)) * 3.0e-9)
    m.set_abiotic_bc(0, _abi.FACES["top"], _abi.PI_BC_CONST, [top])
    m.set_abiotic_bc(0, _abi.FACES["bottom"], _abi.PI_BC_ARRAY2D, bottom)
    m.set_abiotic_bc(0, _abi.FACES["east"], _abi.PI_BC_CONST, [east])
    m.time_step(60.0)
    it, _ = m.get_time()
    Gx, Gy = grid.Nx + 2 * grid.Hx, grid.Ny + 2 * grid.Hy
    flag = {}
    kk = 1 + grid.Hz
    for (i, j) in np.ndindex(5, 3):                   # top, then bottom on the same cells
        q = grid_id(grid, i + 1 + grid.Hx, j + 1 + grid.Hy, kk)
        u = oracle.draw3(SEED, it, 0, _abi.PI_DRAW_ABIO_BC, q)[0]
        flag[q] = u * sz * Ns < bottom[i, j] * 60.0 * (100.0 * 100.0)
    for j in range(3):                                # east: Ax = Δy·ΔzF
        q = grid_id(grid, 5 + grid.Hx, j + 1 + grid.Hy, kk)
        u = oracle.draw3(SEED, it, 0, _abi.PI_DRAW_ABIO_BC, q)[0]
        flag[q] = u * sz * Ns < east * 60.0 * (100.0 * 10.0)
    new = sorted(q for q, f in flag.items() if f)
    a = m.get_abiotic_particles(0)
    assert 2 < len(new) < len(flag) and int(a["ac"].sum()) == 2 + len(new)
    for q, d in zip(new, range(2, 2 + len(new))):
        i, j = q % Gx + 1, (q // Gx) % Gy + 1
        assert a["x"][d] == float(np.float32(i - grid.Hx) - np.float32(0.4))
        assert a["y"][d] == float(np.float32(j - grid.Hy) - np.float32(0.4))
        assert a["z"][d] == float(np.float32(1) - np.float32(0.4))
        assert (a["xi"][d], a["yi"][d]) == (i, j)                       # find_inds! of the step


def test_abiotic_capacity_and_missing_max_ptc_errors():
    grid = RectilinearGrid(size=(4, 4, 1), x=(0, 400), y=(0, 400), z=(0, -10), FT=np.float64)
    C = 8
    m, phyt = _static_model(grid, C)
    m.set_abiotics({"Nsuper": [1.0], "Rd": [1e-4], "release_P": [0.0], "sz_min": [1e-3], "Ktr": [0.0]}, 1,
                   max_ptc=[np.nan])
    m.set_abiotic_bc(0, _abi.FACES["top"], _abi.PI_BC_CONST, [1.0])           # every top cell, 16 > 8 slots
    with pytest.raises(CapacityError, match="number of abiotic particles exceeds the capacity at timestep "
                                            "0.0006944444444444445 days"):
        m.time_step(60.0)
    m2, phyt = _static_model(grid, 16)
    m2.set_abiotics({"Nsuper": [1.0], "Rd": [50.0], "release_P": [0.0], "sz_min": [1e-3], "Ktr": [0.0]}, 1,
                    intac=[(0, 0)], max_ptc=[np.nan])                         # QuotaMode has no max_ptc
    _planks(m2, phyt, 16, [0.5], [0.5], [0.5])
    _abiotics(m2, 0, 16, [0.5], [0.52], [0.5])
    with pytest.raises(PIError, match="no field max_ptc"):
        m2.time_step(60.0)
    with pytest.raises(PIError):
        m2.set_abiotics({k: [1.0] for k in _abi.ABIOTIC_FIELDS}, 1)           # once per model
    m3, _ = _static_model(grid, 16)
    with pytest.raises(PIError):
        m3.set_abiotics({k: [1.0] for k in _abi.ABIOTIC_FIELDS}, 1, intac=[(1, 0)])   # sp2 is not generated


def test_abiotic_workload_steps_with_merges_releases_and_creation():
    wl = W.abiotic(steps=8)
    m = W.configure_abiotics(oracle.from_workload(wl), wl)
    n0 = [m.count_abiotic(a) for a in range(2)]
    drive(m, wl, 8, VelCache(wl))
    p0, p1 = m.get_individuals(0), m.get_individuals(1)
    assert p0["ptc"].sum() > 0 and p1["ptc"].max() == wl.abiotic["max_ptc"][1]
    assert m.count_abiotic(1) > n0[1]                                  # created at the boundaries
    assert m.count_abiotic(0) < n0[0]                                  # merged, some released back
    assert m.get_diag(_abi.PI_DIAG_ABIO_NUM, 1).sum() > 0
