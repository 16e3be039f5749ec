"""The reference's own known-answer tests and invariants, re-run against this project's host logic
and the CPU oracle (test/grid_test.jl, test/field_test.jl, test/example_2D_test.jl,
test/parameter_test.jl)."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import (Bounded, Periodic, RectilinearGrid, bgc_params_default,
                                 phyt_params_default, tracer_names, update_bgc_params,
                                 update_phyt_params)
from PlanktonIndividuals import grids as G
from PlanktonIndividuals import init as I
from PlanktonIndividuals.parameters import default_tracer_init


# ---- test/grid_test.jl --------------------------------------------------------------------

def test_rectilinear_grid():                       # grid_test.jl:5-25
    g = RectilinearGrid(size=(4, 6, 2), x=(0, 12), y=(0, 12), z=(0, -8), halo=(2, 2, 2), FT=np.float64)
    assert (g.Nx, g.Ny, g.Nz) == (4, 6, 2)
    assert g.Δx == 3.0 and g.Δy == 2.0
    assert list(g.dzC) == [4.0] * 6
    assert list(g.dzF) == [4.0] * 6
    assert len(g.xC) == 8 and len(g.yC) == 10 and len(g.zC) == 6
    assert len(g.xF) == 8 and len(g.yF) == 10 and len(g.zF) == 6


def test_vertically_stretched_rectilinear_grid():  # grid_test.jl:27-51
    zfs = [0.0, -1.0, -3.0, -5.0, -10.0]
    g = RectilinearGrid(size=(4, 6, 4), x=(0, 12), y=(0, 12), z=zfs, halo=(2, 2, 2), FT=np.float64)
    assert g.Δx == 3.0 and g.Δy == 2.0
    assert list(g.dzC) == [1.0, 1.0, 1.5, 2.0, 3.5, 5.0, 5.0, 5.0]
    assert list(g.dzF) == [1.0, 1.0, 1.0, 2.0, 2.0, 5.0, 5.0, 5.0]
    assert list(g.zF) == [2.0, 1.0, -0.0, -1.0, -3.0, -5.0, -10.0, -15.0]
    assert list(g.zC) == [1.5, 0.5, -0.5, -2.0, -4.0, -7.5, -12.5, -17.5]


def test_rectilinear_areas_volumes():              # grid_test.jl:53-67
    zfs = [0.0, -1.0, -3.0, -5.0, -10.0]
    g = RectilinearGrid(size=(4, 6, 4), x=(0, 12), y=(0, 12), z=zfs, halo=(2, 2, 2), FT=np.float64)
    assert G.ΔxC(1, 1, 1, g) == g.Δx and G.ΔyC(1, 1, 1, g) == g.Δy and G.ΔzC(1, 1, 1, g) == g.dzC[0]
    assert G.ΔxF(1, 1, 1, g) == g.Δx and G.ΔyF(1, 1, 1, g) == g.Δy and G.ΔzF(1, 1, 1, g) == g.dzF[0]
    assert G.Ax(1, 1, 1, g) == g.Δy * g.dzF[0]
    assert G.Ay(1, 1, 1, g) == g.Δx * g.dzF[0]
    assert G.Az(1, 1, 1, g) == g.Δx * g.Δy
    assert G.volume(1, 1, 1, g) == g.Δx * g.Δy * g.dzF[0]


# ---- test/field_test.jl -------------------------------------------------------------------

def test_fields():                                 # field_test.jl:3-20
    g = RectilinearGrid(size=(4, 6, 2), x=(0, 12), y=(0, 12), z=(0, -8))
    assert tuple(tracer_names) == ("DIC", "NH4", "NO3", "PO4", "DFe", "DOC", "DON", "DOP",
                                   "PFe_inorg", "POC", "PON", "POP", "PFe_bio", "Dust")
    trs = I.generate_tracers(g, default_tracer_init(), np.random.default_rng(0))
    assert trs[0].shape == (8, 10, 6)
    assert trs[0].max() < 23.0 and trs[0].min() > 17.0
    assert np.array_equal(G.interior(trs[0], g).shape, (4, 6, 2))


def test_fill_halos():                             # field_test.jl:21-106
    g = RectilinearGrid(size=(4, 6, 2), x=(0, 12), y=(0, 12), z=(0, -8))
    c = I.generate_tracers(g, default_tracer_init(), np.random.default_rng(1))[0]
    Nx, Ny, Nz, Hx, Hy, Hz = g.Nx, g.Ny, g.Nz, g.Hx, g.Hy, g.Hz
    # periodic, each face separately (0-based slices of the 1-based ranges)
    G._face(c, 0, False, Nx, Hx, 0); assert np.array_equal(c[Nx + Hx:], c[Hx:2 * Hx])
    G._face(c, 0, True, Nx, Hx, 0); assert np.array_equal(c[:Hx], c[Nx:Nx + Hx])
    G._face(c, 1, False, Ny, Hy, 0); assert np.array_equal(c[:, Ny + Hy:], c[:, Hy:2 * Hy])
    G._face(c, 1, True, Ny, Hy, 0); assert np.array_equal(c[:, :Hy], c[:, Ny:Ny + Hy])
    G._face(c, 2, False, Nz, Hz, 0); assert np.array_equal(c[:, :, Nz + Hz:], c[:, :, Hz:2 * Hz])
    G._face(c, 2, True, Nz, Hz, 0); assert np.array_equal(c[:, :, :Hz], c[:, :, Nz:Nz + Hz])
    # bounded
    G._face(c, 0, False, Nx, Hx, 1)
    for i in range(Hx):
        assert np.array_equal(c[Nx + Hx + i], c[Nx + Hx - 1])
    G._face(c, 0, True, Nx, Hx, 1)
    for i in range(Hx):
        assert np.array_equal(c[i], c[Hx])
    G._face(c, 1, False, Ny, Hy, 1)
    for i in range(Hy):
        assert np.array_equal(c[:, Ny + Hy + i], c[:, Ny + Hy - 1])
    G._face(c, 1, True, Ny, Hy, 1)
    for i in range(Hy):
        assert np.array_equal(c[:, i], c[:, Hy])
    G._face(c, 2, False, Nz, Hz, 1)
    for i in range(Hz):
        assert np.array_equal(c[:, :, Nz + Hz + i], c[:, :, Nz + Hz - 1])
    G._face(c, 2, True, Nz, Hz, 1)
    for i in range(Hz):
        assert np.array_equal(c[:, :, i], c[:, :, Hz])
    # velocity rule on the high face
    G._face(c, 0, False, Nx, Hx, 1, "vel")
    for i in range(1, Hx):
        assert np.array_equal(c[Nx + Hx + i], c[Nx + Hx])
    G._face(c, 1, False, Ny, Hy, 1, "vel")
    for i in range(1, Hy):
        assert np.array_equal(c[:, Ny + Hy + i], c[:, Ny + Hy])
    G._face(c, 2, False, Nz, Hz, 1, "vel")
    for i in range(1, Hz):
        assert np.array_equal(c[:, :, Nz + Hz + i], c[:, :, Nz + Hz])
    # Gc rule
    G._face(c, 0, False, Nx, Hx, 1, "Gc"); assert not c[Nx + Hx:].any()
    G._face(c, 1, False, Ny, Hy, 1, "Gc"); assert not c[:, Ny + Hy:].any()
    G._face(c, 2, False, Nz, Hz, 1, "Gc"); assert not c[:, :, Nz + Hz:].any()


def _empty_oracle(grid, nsp=1, C=4, seed=0):
    bgc = update_bgc_params({}, np.float64)
    phyt = update_phyt_params({}, np.float64, N=nsp)
    m = oracle.OracleModel(grid, bgc, phyt, nsp, C, seed)
    m.set_state([I.empty_individuals(C) for _ in range(nsp)],
                [np.zeros(grid.total_size, order="F") for _ in tracer_names])
    return m


def test_boundary_conditions_flux_kat():           # field_test.jl:108-122
    g = RectilinearGrid(size=(4, 4, 4), x=(0, 32), y=(0, 32), z=(0, -32), FT=np.float64)
    m = _empty_oracle(g)
    m.set_flux_bc(0, 0, 2, np.ones((4, 4), order="F"))        # DIC, west, 2D array of ones
    m.set_time(9, 9.0)
    m.set_PARF(np.zeros((4, 4)))
    m.set_temp(np.zeros((4, 4, 4)))
    m.time_step(1.0)
    Gc = m.get_field(17 + 0)
    assert np.all(Gc[2, 2:6, 2:6] == 1 / 8)
    # the tracer took the tendency: zero initial DIC + 1/8 at the west interior column
    dic = m.get_tracer(0)
    assert np.all(dic[2, 2:6, 2:6] == 1 / 8) and not dic[3:6, 2:6, 2:6].any()


# ---- test/parameter_test.jl ---------------------------------------------------------------

def test_parameter_updates():
    p = update_bgc_params({"kw": 0.05}, np.float64)
    assert p["kw"] == 0.05 and p["kc"] == bgc_params_default(np.float64)["kc"]
    with pytest.raises(ValueError, match="PARAM: bgc parameter not found bogus"):
        update_bgc_params({"bogus": 1.0}, np.float64)
    q = update_phyt_params({"PCmax": [5e-5, 6e-5]}, np.float64, N=2)
    assert q["PCmax"] == [5e-5, 6e-5] and q["Nsuper"] == [1, 1]
    with pytest.raises(ValueError, match="PARAM: phyt parameter not found"):
        update_phyt_params({"nope": [1]}, np.float64)
    assert len(phyt_params_default(3)["Cquota"]) == 3


# ---- test/example_2D_test.jl: total-P conservation over 10 steps -----------------------------

def tot_mass(c, g):
    vol = g.Δx * g.Δy * np.asarray(g.dzF)[g.Hz:g.Hz + g.Nz]
    return float(np.sum(G.interior(c, g) * vol[None, None, :]))


def test_example_2D_total_phosphorus_conserved():
    g = RectilinearGrid(size=(16, 16, 1), x=(0, 32), y=(0, 32), z=(0, -32), FT=np.float64)
    rng = np.random.default_rng(2024)
    bgc = update_bgc_params({}, np.float64)
    phyt = update_phyt_params({}, np.float64, N=1)
    C = 8 * 1024
    ind = I.initialize_plankton(g, phyt, 0, 2 ** 10, C, rng)
    trs = I.generate_tracers(g, default_tracer_init(), rng)
    m = oracle.OracleModel(g, bgc, phyt, 1, C, seed=7)
    m.set_state([ind], trs)
    R_PC = phyt["R_PC"][0]

    def TP():
        d = m.get_individuals(0)
        return (tot_mass(m.get_tracer(3), g) + tot_mass(m.get_tracer(7), g) + tot_mass(m.get_tracer(11), g)
                + float(np.sum(d["Pq"] + d["Bm"] * R_PC)))

    tp0 = TP()
    for it in range(10):
        u = rng.standard_normal((16, 16, 1)) * 1e-4
        v = rng.standard_normal((16, 16, 1)) * 1e-4
        w = rng.standard_normal((16, 16, 2)) * 1e-4
        m.set_velocity(u, v, w)
        m.set_PARF(np.full((16, 16), 1000.0))
        m.set_temp(np.full((16, 16, 1), 26.5))
        m.time_step(60.0)
    tp1 = TP()
    assert abs(tp0 - tp1) <= 1e1                     # the reference's own tolerance (atol=1e1)


def test_phosphorus_budget_divergence_free_tight():
    """With a divergence-free flow and no divisions, P moves between individuals, PO4, DOP and POP
    without loss: the budget over active individuals and tracers closes to rounding."""
    from PlanktonIndividuals import workloads as W
    wl = W.config1(n=16, N=600, steps=30, phyt_over={"dvid_P": [0.0], "mort_P": [2e-4], "mort_reg": [0.9]})
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    m = oracle.from_workload(wl)
    g, R_PC = wl.grid, wl.phyt["R_PC"][0]

    def TP():
        d = m.get_individuals(0)
        a = d["ac"]
        return (tot_mass(m.get_tracer(3), g) + tot_mass(m.get_tracer(7), g) + tot_mass(m.get_tracer(11), g)
                + float(np.sum((d["Pq"] + d["Bm"] * R_PC)[a])))

    tp0 = TP()
    u, v, w = wl.velocity(0)
    for it in range(30):
        m.set_velocity(u, v, w)
        m.set_PARF(wl.parf[:, :, int(it * wl.dT // 3600)])
        m.set_temp(wl.temp[:, :, :, 0])
        m.time_step(wl.dT)
    assert m.count_active(0) < 600                 # some individuals died and were remineralised
    assert abs(TP() - tp0) <= 1e-12 * tp0
