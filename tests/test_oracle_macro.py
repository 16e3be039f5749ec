"""MacroMolecularMode (src/Individuals/Plankton/MacroMolecularMode/) in the CPU oracle: the
reference has no MacroMolecularMode test, so the restatement is pinned by the budgets the mode's
formulas keep exactly — phosphorus moves between PO4, DOP, POP and the individuals' DNA, RNA and
P reserve, nitrogen between the nutrients, DON, PON and the individuals' protein, nucleic acids,
reserve and chlorophyll — and by the initialisation rule and parameter set of the reference."""
import numpy as np
import pytest

import oracle
from PlanktonIndividuals import MacroMolecularMode, update_phyt_params, workloads as W
from PlanktonIndividuals import grids as G
from PlanktonIndividuals import _abi
from PlanktonIndividuals.stepping import VelCache, drive


def _mass(m, g, tracers):
    vol = G.interior(G.cell_volumes(g), g)
    return sum(float(np.sum(G.interior(m.get_tracer(_abi.tracer_names.index(n)), g) * vol)) for n in tracers)


def _inds(m, wl, what):
    out = 0.0
    for s in range(wl.nsp):
        d = m.get_individuals(s)
        a = d["ac"]
        R = {k: wl.phyt[k][s] for k in ("R_NC_PRO", "R_NC_DNA", "R_NC_RNA", "R_PC_DNA", "R_PC_RNA")}
        if what == "P":
            v = d["DNA"] * R["R_PC_DNA"] + d["RNA"] * R["R_PC_RNA"] + d["PST"]
        else:
            v = (d["PRO"] * R["R_NC_PRO"] + d["DNA"] * R["R_NC_DNA"] + d["RNA"] * R["R_NC_RNA"] + d["NST"]
                 + d["Chl"] / np.float32(893.49) * 4.0)
        out += float(np.sum(v[a]))
    return out


def test_macro_parameters_and_initialisation():
    p = update_phyt_params({}, np.float64, N=2, mode=MacroMolecularMode())
    assert [k for k, _ in _abi.MACRO_FIELDS] == [c for c, _ in _abi.pi_macro_params._fields_]
    assert len(_abi.MACRO_FIELDS) == 47 and all(key in p for _, key in _abi.MACRO_FIELDS)
    with pytest.raises(ValueError):
        update_phyt_params({"Cquota": [1.0]}, np.float64, mode=MacroMolecularMode())
    wl = W.macro(N_per_species=500)
    d = wl.individuals[0]
    a = d["ac"]
    C_DNA = p["C_DNA"][0]
    r = d["DNA"][a] / C_DNA
    assert np.all((r >= 1.0) & (r < 1.3))                        # DNA in C_DNA·(1, 1 + var)
    assert np.allclose(d["Chl"][a], d["DNA"][a] * 3.45 * np.float32(893.49) / 55.0)
    assert np.all(d["PST"][a] <= 1.3 * d["CH"][a] / 106.0)


@pytest.mark.parametrize("what", ["P", "N"])
def test_macro_budget_closes_without_divisions(what):
    """Grazing, mortality, uptake, synthesis, exudation and remineralisation move P (N) between the
    individuals and the tracers without loss: the budget closes to rounding over 30 steps."""
    over = {"dvid_P": [0.0, 0.0], "mort_P": [5e-4, 3e-4], "mort_reg": [0.5, 0.5], "grz_P": [1e-4, 5e-5]}
    wl = W.macro(N_per_species=1200, steps=30, phyt_over=over)
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))     # daylight
    m = oracle.from_workload(wl)
    g = wl.grid
    tr = ("PO4", "DOP", "POP") if what == "P" else ("NH4", "NO3", "DON", "PON")
    b0 = _mass(m, g, tr) + _inds(m, wl, what)
    drive(m, wl, 30, VelCache(wl))
    assert m.count_active(0) < 1200 and m.count_active(1) < 1200   # losses happened
    b1 = _mass(m, g, tr) + _inds(m, wl, what)
    assert abs(b1 - b0) <= 1e-12 * b0


def test_macro_divisions_by_dna_and_inactive_slots_keep_changing():
    """Division when DNA exceeds twice C_DNA·Nsuper (calc_MM_dvid!): dividers and daughters carry
    half of each pool; the synthesis terms of an inactive slot carry no ac, so its stale pools keep
    changing (growth_kernels.jl:136-152) while its age does not."""
    over = {"dvid_P": [3e-3, 3e-3], "mort_P": [1e-3, 1e-3], "grz_P": [0.0, 0.0]}
    wl = W.macro(N_per_species=1000, steps=6, phyt_over=over)
    C_DNA = wl.phyt["C_DNA"][0]
    d = wl.individuals[0]
    d["DNA"][:300] = 2.2 * C_DNA                                    # ready to divide
    d["age"][d["ac"]] = 1.0                                         # old enough to die (calc_MM_mort!)
    m = oracle.from_workload(wl)
    drive(m, wl, 6, VelCache(wl))
    e = m.get_individuals(0)
    assert np.sum(e["gen"][e["ac"]] >= 2.0) > 50                   # dividers and their daughters
    dead = ~e["ac"] & (np.arange(len(e["ac"])) < 1000)
    assert np.any(dead)
    m.time_step(wl.dT)
    f = m.get_individuals(0)
    still = dead & ~f["ac"]
    assert np.any(f["PRO"][still] != e["PRO"][still])
    assert np.array_equal(f["age"][still], e["age"][still])
