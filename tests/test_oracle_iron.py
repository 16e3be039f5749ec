"""IronEnergyMode (src/Individuals/Plankton/IronEnergyMode/) in the CPU oracle: the reference has no
IronEnergyMode test, so the restatement is pinned by the budgets its formulas keep exactly —
phosphorus between PO4, DOP, POP and the individuals' Bm·R_PC + qP; nitrogen (no nitrogen
fixation) between NH4, NO3, DON, PON and Bm·R_NC + qNO3 + qNH4; iron between DFe, PFe_bio,
PFe_inorg and the four Fe quotas — by the parameter list and initialisation rule of the
reference, and by the light-driven iron allocation and dark clock around sunset."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import IronEnergyMode, update_phyt_params, workloads as W
from PlanktonIndividuals import grids as G
from PlanktonIndividuals import _abi
from PlanktonIndividuals.stepping import VelCache, drive

BUDGET = {"P": ("PO4", "DOP", "POP"), "N": ("NH4", "NO3", "DON", "PON"), "Fe": ("DFe", "PFe_bio", "PFe_inorg")}


def _mass(m, g, tracers):
    vol = G.interior(G.cell_volumes(g), g)
    return sum(float(np.sum(G.interior(m.get_tracer(_abi.tracer_names.index(n)), g) * vol)) for n in tracers)


def _inds(m, wl, what):
    out = 0.0
    for s in range(wl.nsp):
        d = m.get_individuals(s)
        a = d["ac"]
        v = {"P": d["Bm"] * wl.phyt["R_PC"][s] + d["qP"], "N": d["Bm"] * wl.phyt["R_NC"][s] + d["qNO3"] + d["qNH4"],
             "Fe": d["qFe"] + d["qFePS"] + d["qFeNF"] + d["qFeNR"]}[what]
        out += float(np.sum(v[a]))
    return out


def test_iron_parameters_and_initialisation():
    p = update_phyt_params({}, np.float64, N=2, mode=IronEnergyMode())
    assert [c for c, _ in _abi.IRON_FIELDS] == [c for c, _ in _abi.pi_iron_params._fields_]
    assert len(_abi.IRON_FIELDS) == 64 and all(key in p for _, key in _abi.IRON_FIELDS) and len(p) == 64
    assert len(_abi.IRON_PROC_NAMES) == 32
    with pytest.raises(ValueError):
        update_phyt_params({"Cqmax": [1.0]}, np.float64, mode=IronEnergyMode())
    wl = W.iron(N_per_species=500, phyt_over={"is_nr": [1.0, 0.0], "is_croc": [0.0, 1.0]})
    for s, (nr, nf) in enumerate(((True, False), (False, True))):
        d = wl.individuals[s]
        a = d["ac"]
        fe = d["qFe"] + d["qFePS"] + d["qFeNR"] + d["qFeNF"]
        assert np.allclose(d["qFePS"][a], 0.4 * fe[a])
        assert np.any(d["qFeNR"][a]) == nr and np.any(d["qFeNF"][a]) == nf
        assert np.all(fe[a] <= 0.1 * p["qFemax"][0] * (d["Bm"][a] + d["CH"][a]) * (1 + 1e-12))
        assert np.allclose(d["Chl"][a], d["Bm"][a] * 0.10)


@pytest.mark.parametrize("what", ["P", "N", "Fe"])
def test_iron_budgets_close_without_divisions(what):
    """Grazing, mortality, uptake, the energy budget, iron allocation, biosynthesis and
    remineralisation move P, N and Fe between the individuals and the tracers without loss over
    40 steps that cross sunset (no nitrogen fixation: is_croc = is_tric = 0 for both species)."""
    over = {"dvid_P": [0.0, 0.0], "mort_P": [5e-4, 3e-4], "grz_P": [1e-4, 5e-5]}
    wl = W.iron(N_per_species=1200, phyt_over=over)
    m = oracle.from_workload(wl)
    b0 = _mass(m, wl.grid, BUDGET[what]) + _inds(m, wl, what)
    drive(m, wl, 40, VelCache(wl))
    assert m.count_active(0) < 1200 and m.count_active(1) < 1200        # losses happened
    b1 = _mass(m, wl.grid, BUDGET[what]) + _inds(m, wl, what)
    assert abs(b1 - b0) <= 1e-12 * b0


def test_iron_sunset_divisions_and_inactive_slots():
    """After sunset par is exactly zero: the dark clock runs, photosystem iron goes back to storage
    (isless(dpar, 0) + isequal(0, par)), the nitrogenase of a Crocosphaera-like species takes iron
    before its clock; divisions copy the pools; inactive slots' iron keeps moving (iron_alloc
    carries no ac) while their age does not."""
    over = {"dvid_P": [2e-4, 2e-4], "dvid_reg": [1.0, 1.0], "grz_P": [1e-4, 1e-4], "is_nr": [1.0, 0.0],
            "is_croc": [0.0, 1.0]}
    wl = W.iron(N_per_species=1000, steps=40, capacity=6000, phyt_over=over)
    m = oracle.from_workload(wl)
    drive(m, wl, 29, VelCache(wl))
    lit = [m.get_individuals(s) for s in range(2)]
    # before sunset only the step's daughters have run the clock (their slots gathered no light)
    assert all(np.mean(d["tdark"][d["ac"]] > 0) < 0.1 for d in lit)
    drive(m, wl, 11, VelCache(wl))
    e = [m.get_individuals(s) for s in range(2)]
    for s in range(2):
        a = e[s]["ac"]
        assert np.all(e[s]["tdark"][a] > 0) and np.sum(e[s]["gen"][a] >= 2.0) > 20
    dead = ~e[0]["ac"] & lit[0]["ac"]
    assert np.any(dead)
    m.time_step(wl.dT)
    f = m.get_individuals(0)
    still = dead & ~f["ac"]
    assert np.any(f["qFePS"][still] != e[0]["qFePS"][still])
    assert np.array_equal(f["age"][still], e[0]["age"][still])
