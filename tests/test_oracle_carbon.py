"""CarbonMode in the CPU oracle (src/Individuals/Plankton/CarbonMode/), pinned by the reference's
own CarbonMode test (test/example_3D_test.jl: a 16×16×16 grid, random velocities, DON flux boundary
conditions, 10 steps; total carbon DIC + DOC + POC + ΣBm conserved within atol 1e3) and by a tight
carbon budget: photosynthesis and respiration move carbon between DIC and biomass, grazing and
mortality move biomass into DOC and POC, remineralisation moves DOC and POC into DIC, thermal
damage and repair move biomass between its healthy and damaged parts, and division halves it
between two individuals. Without divisions (whose daughters scatter their birth-step respiration
into a halo cell) the budget closes to rounding."""
import numpy as np

import oracle
from PlanktonIndividuals import CarbonMode, tracer_names, workloads as W
from PlanktonIndividuals.grids import RectilinearGrid
from PlanktonIndividuals.init import initialize_plankton_carbon
from PlanktonIndividuals.parameters import default_temperature, update_bgc_params, update_phyt_params
from test_oracle_kats import tot_mass

C_TRACERS = [tracer_names.index(n) for n in ("DIC", "DOC", "POC")]


def _total_carbon(m, g, nsp=1):
    tc = sum(tot_mass(m.get_tracer(n), g) for n in C_TRACERS)
    for s in range(nsp):
        d = m.get_individuals(s)
        tc += float(np.sum(d["Bm"][d["ac"]]))
    return tc


def test_reference_example_3D_carbon_conservation():
    """test/example_3D_test.jl restated: CarbonMode defaults, 16×16×16 grid of 2 m cells,
    velocities randn·1e-4 (11 snapshots, one per step), DON flux boundary conditions, ΔT = 60 s,
    10 steps; |TC − TC₀| ≤ 1e3."""
    rng = np.random.default_rng(3)
    g = RectilinearGrid(size=(16, 16, 16), x=(0.0, 32.0), y=(0.0, 32.0), z=(0.0, -32.0), FT=np.float64)
    bgc = update_bgc_params({}, np.float64)
    phyt = update_phyt_params({}, np.float64, N=1, mode=CarbonMode())
    C = 8 * 1024
    m = oracle.OracleModel(g, bgc, phyt, 1, C, 3, mode="carbon")
    inds = [initialize_plankton_carbon(g, phyt, 0, 1024, C, rng)]
    trs = W.make_tracers(g, rng)
    m.set_state(inds, trs)
    don = tracer_names.index("DON")
    m.set_flux_bc(don, 0, 1, np.array([1.0e-3]))                                    # west
    m.set_flux_bc(don, 1, 2, np.asfortranarray(rng.standard_normal((16, 16)) * 1e-3))  # east
    m.set_flux_bc(don, 2, 3, np.asfortranarray(rng.standard_normal((16, 16, 10)) * 1e-3), 10)
    m.set_flux_bc(don, 3, 3, np.asfortranarray(rng.standard_normal((16, 16, 10)) * 1e-3), 10)
    temp = default_temperature(g, 60.0, 10)
    parf = np.full((16, 16), 500.0)
    tc0 = _total_carbon(m, g)
    for it in range(10):
        u = rng.standard_normal((16, 16, 16)) * 1e-4
        v = rng.standard_normal((16, 16, 16)) * 1e-4
        w = rng.standard_normal((16, 16, 17)) * 1e-4
        m.set_velocity(u, v, w)
        m.set_PARF(parf)
        m.set_temp(temp[:, :, :, 0])
        m.time_step(60.0)
    assert abs(_total_carbon(m, g) - tc0) <= 1e3


def test_carbon_budget_tight_without_divisions():
    """Thermal damage and repair on (T above Topt), grazing and mortality on, no divisions: total
    carbon closes to 1e-12 relative over 40 steps."""
    wl = W.carbon(nx=12, nz=6, N_per_species=800, nsp=2, steps=40, temp=28.6, bd_frac=0.4,
                  phyt_over={"dvid_P": [0.0, 0.0], "mort_P": [5e-4, 5e-4], "grz_P": [2e-4, 0.0]})
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    m = oracle.from_workload(wl)
    g = wl.grid
    tc0 = _total_carbon(m, g, 2)
    bd0 = float(np.sum(m.get_individuals(0)["Bd"]))
    u, v, w = wl.velocity(0)
    for it in range(40):
        m.set_velocity(u, v, w)
        m.set_PARF(wl.parf[:, :, int(it * wl.dT // 3600)])
        m.set_temp(wl.temp[:, :, :, 0])
        m.time_step(wl.dT)
    assert m.count_active(0) < 800                  # grazing and mortality happened
    d = m.get_individuals(1)
    assert float(np.sum(d["Bd"][d["ac"]])) != bd0    # thermal damage and repair moved biomass
    assert abs(_total_carbon(m, g, 2) - tc0) <= 1e-12 * tc0
