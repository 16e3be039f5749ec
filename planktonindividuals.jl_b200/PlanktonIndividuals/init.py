"""Initial conditions on the host: initialize_plankton! and generate_tracers
(src/Individuals/Plankton/QuotaMode/plankton_generation.jl:35-72,
src/Biogeochemistry/tracer_fields.jl:60-101) with a seeded generator instead of the reference's
unseeded one. Arrays are float64 (the C ABI type)."""
import numpy as np

from ._abi import tracer_names
from .grids import fill_halo_tracer


def empty_individuals(C):
    d = {k: np.zeros(C, dtype=np.float64) for k in
         ("x", "y", "z", "Sz", "Bm", "Cq", "Nq", "Pq", "Chl", "gen", "age", "graz", "mort", "dvid")}
    for k in ("xi", "yi", "zi"):
        d[k] = np.zeros(C, dtype=np.int64)
    d["ac"] = np.zeros(C, dtype=bool)
    return d


def species_param(p, key, s):
    v = p[key]
    return float(v[s] if hasattr(v, "__len__") else v)


def initialize_plankton(grid, p, s, N, C, rng):
    """initialize_plankton! for species s (0-based) with N active individuals out of C slots."""
    if N > C:
        raise ValueError("PlanktonModel: number of individuals exceeds max_individuals")
    d = empty_individuals(C)
    ac = np.zeros(C, dtype=bool)
    ac[:N] = True
    mean, var = species_param(p, "mean", s), species_param(p, "var", s)
    Cquota, Nsuper = species_param(p, "Cquota", s), species_param(p, "Nsuper", s)
    cqmax, nqmax, pqmax = (species_param(p, k, s) for k in ("Cqmax", "Nqmax", "Pqmax"))
    R_NC, R_PC, Chl2Cint = (species_param(p, k, s) for k in ("R_NC", "R_PC", "Chl2Cint"))
    Sz = rng.standard_normal(C)
    x, y, z = rng.random(C), rng.random(C), rng.random(C)
    Cq, Nq, Pq = rng.random(C), rng.random(C), rng.random(C)
    d["ac"] = ac
    d["gen"][:N] = 1.0
    d["age"][:N] = 0.0
    d["x"] = (x * grid.Nx) * ac
    d["y"] = (y * grid.Ny) * ac
    d["z"] = (z * grid.Nz) * ac
    d["Sz"] = np.maximum(1.0, Sz * var + mean) * ac
    d["Bm"] = Cquota * d["Sz"] * Nsuper
    d["Cq"] = Cq * cqmax * d["Bm"]
    d["Nq"] = Nq * (nqmax * (d["Bm"] + d["Cq"]) - d["Bm"] * R_NC)
    d["Pq"] = Pq * (pqmax * (d["Bm"] + d["Cq"]) - d["Bm"] * R_PC)
    d["Chl"] = d["Bm"] * Chl2Cint
    mask_individuals(d, grid, N)
    return d


def initialize_plankton_carbon(grid, p, s, N, C, rng):
    """initialize_plankton! of CarbonMode (CarbonMode/plankton_generation.jl:33-56) for species s:
    Sz = max(1, N(mean, var)), Bm = Cquota·Sz·Nsuper, Chl = Bm·Chl2C, Bd = 0."""
    if N > C:
        raise ValueError("PlanktonModel: number of individuals exceeds max_individuals")
    d = empty_individuals(C)
    for k in ("Cq", "Nq", "Pq"):
        del d[k]
    ac = np.zeros(C, dtype=bool)
    ac[:N] = True
    mean, var = species_param(p, "mean", s), species_param(p, "var", s)
    Cquota, Nsuper, Chl2C = (species_param(p, k, s) for k in ("Cquota", "Nsuper", "Chl2C"))
    Sz = rng.standard_normal(C)
    x, y, z = rng.random(C), rng.random(C), rng.random(C)
    d["ac"] = ac
    d["gen"][:N] = 1.0
    d["x"] = (x * grid.Nx) * ac
    d["y"] = (y * grid.Ny) * ac
    d["z"] = (z * grid.Nz) * ac
    d["Sz"] = np.maximum(1.0, Sz * var + mean) * ac
    d["Bm"] = Cquota * d["Sz"] * Nsuper
    d["Chl"] = d["Bm"] * Chl2C
    d["Bd"] = np.zeros(C, dtype=np.float64)
    mask_individuals(d, grid, N)
    return d


def initialize_plankton_iron(grid, p, s, N, C, rng):
    """initialize_plankton! of IronEnergyMode (IronEnergyMode/plankton_generation.jl:53-95) for species
    s: Sz = max(1, N(mean, var)), Bm = Cquota·Sz·Nsuper, CH, qNO3, qNH4, qP, qFe uniform up to a tenth
    of their maxima, the iron split 0.4 / 0.3 / 0.3 between photosystem, nitrate reductase and
    nitrogenase as the species has them, Chl = Bm·Chl2Cint."""
    if N > C:
        raise ValueError("PlanktonModel: number of individuals exceeds max_individuals")
    d = empty_individuals(C)
    for k in ("Cq", "Nq", "Pq"):
        del d[k]
    ac = np.zeros(C, dtype=bool)
    ac[:N] = True
    g = lambda k: species_param(p, k, s)
    CHmax, qNO3max, qNH4max = g("CHmax") * 0.1, g("qNO3max") * 0.1, g("qNH4max") * 0.1
    pqmax, feqmax = g("qPmax") * 0.1, g("qFemax") * 0.1
    Sz = rng.standard_normal(C)
    x, y, z = rng.random(C), rng.random(C), rng.random(C)
    CH, qNO3, qNH4, qP, qFe = (rng.random(C) for _ in range(5))
    d["ac"] = ac
    d["gen"][:N] = 1.0
    d["x"], d["y"], d["z"] = (x * grid.Nx) * ac, (y * grid.Ny) * ac, (z * grid.Nz) * ac
    d["Sz"] = np.maximum(1.0, Sz * g("var") + g("mean")) * ac
    d["Bm"] = g("Cquota") * d["Sz"] * g("Nsuper")
    d["CH"] = CH * CHmax * d["Bm"]
    d["qNO3"] = qNO3 * (qNO3max * (d["Bm"] + d["CH"]))
    d["qNH4"] = qNH4 * (qNH4max * (d["Bm"] + d["CH"]))
    d["qP"] = qP * (pqmax * (d["Bm"] + d["CH"]))
    fe = qFe * (feqmax * (d["Bm"] + d["CH"]))
    d["qFePS"] = fe * 0.4
    d["qFeNR"] = fe * 0.3 * g("is_nr")
    d["qFeNF"] = fe * 0.3 * (g("is_croc") + g("is_tric"))
    d["qFe"] = fe - (d["qFePS"] + d["qFeNR"] + d["qFeNF"])
    d["Chl"] = d["Bm"] * g("Chl2Cint")
    d["exEn"] = np.zeros(C)
    d["tdark"] = np.zeros(C)
    mask_individuals(d, grid, N)
    return d


def initialize_plankton_macro(grid, p, s, N, C, rng):
    """initialize_plankton! of MacroMolecularMode (MacroMolecularMode/plankton_generation.jl:40-79)
    for species s: DNA in C_DNA·Nsuper·(1, 1 + var), RNA, PRO in (1 ± var) times their ratio to
    DNA, CH in (1 ± var)·DNA·CH2DNA, NST = U(1 ± var)·CH·16/106, PST = U(1 ± var)·CH/106,
    Chl = DNA·Chl2DNA·893.49/55."""
    if N > C:
        raise ValueError("PlanktonModel: number of individuals exceeds max_individuals")
    d = empty_individuals(C)
    for k in ("Sz", "Bm", "Cq", "Nq", "Pq"):
        del d[k]
    ac = np.zeros(C, dtype=bool)
    ac[:N] = True
    var, C_DNA, Nsuper = (species_param(p, k, s) for k in ("var", "C_DNA", "Nsuper"))
    RNA2DNA, PRO2DNA, CH2DNA, Chl2DNA = (species_param(p, k, s) for k in ("RNA2DNA", "PRO2DNA", "CH2DNA", "Chl2DNA"))
    DNA, RNA, PRO = rng.random(C), rng.random(C), rng.random(C)
    x, y, z = rng.random(C), rng.random(C), rng.random(C)
    CH, NST, PST = rng.random(C), rng.random(C), rng.random(C)
    d["ac"] = ac
    d["gen"][:N] = 1.0
    DNA = DNA * var + 1.0
    RNA = RNA * var * 2.0 + 1.0 - var
    PRO = PRO * var * 2.0 + 1.0 - var
    CH = CH * var * 2.0 + 1.0 - var
    NST = NST * var * 2.0 + 1.0 - var
    PST = PST * var * 2.0 + 1.0 - var
    d["x"] = (x * grid.Nx) * ac
    d["y"] = (y * grid.Ny) * ac
    d["z"] = (z * grid.Nz) * ac
    d["DNA"] = DNA * C_DNA * Nsuper * ac
    d["RNA"] = RNA * C_DNA * Nsuper * ac * RNA2DNA
    d["PRO"] = PRO * C_DNA * Nsuper * ac * PRO2DNA
    d["CH"] = CH * d["DNA"] * CH2DNA
    d["NST"] = NST * d["CH"] * np.float32(16.0) / np.float32(106.0)
    d["PST"] = PST * d["CH"] / np.float32(106.0)
    d["Chl"] = d["DNA"] * Chl2DNA * np.float32(893.49) / 55.0
    mask_individuals(d, grid, N)
    return d


def mask_individuals(d, grid, N):
    """mask_individuals! (Individuals/utils.jl:89-100)."""
    ac = d["ac"][:N]
    xi = np.trunc((d["x"][:N] + 1) * ac).astype(np.int64) + grid.Hx
    yi = np.trunc((d["y"][:N] + 1) * ac).astype(np.int64) + grid.Hy
    zi = np.trunc((d["z"][:N] + 1) * ac).astype(np.int64) + grid.Hz
    lm = grid.landmask[xi - 1, yi - 1, zi - 1]
    d["ac"][:N] = lm & ac


def initialize_abiotic_particle(grid, N, C, rng):
    """initialize_abiotic_particle! (src/Individuals/Abiotic/particle_generation.jl:24-35): N active
    particles at uniform positions in the domain, masked by land; cell indices zero as constructed."""
    if N > C:
        raise ValueError("PlanktonModel: number of abiotic particles exceeds max_individuals")
    ac = np.zeros(C, dtype=bool)
    ac[:N] = True
    x, y, z = rng.random(C), rng.random(C), rng.random(C)
    d = {"x": (x * grid.Nx) * ac, "y": (y * grid.Ny) * ac, "z": (z * grid.Nz) * ac, "ac": ac}
    for k in ("xi", "yi", "zi"):
        d[k] = np.zeros(C, dtype=np.int64)
    mask_individuals(d, grid, N)
    return d


def generate_tracers(grid, source, rng):
    """generate_tracers for a NamedTuple-style source {initial_condition, rand_noise}: each tracer
    is its value times a draw from lower:1.0e-4:upper, masked by land, halos filled."""
    shape = grid.total_size
    out = []
    ic, noise = source["initial_condition"], source["rand_noise"]
    for name in tracer_names:
        if name not in ic:
            raise ValueError(f"TRAC_INIT: tracer not found {name}")
        if ic[name] < 0.0:
            raise ValueError("TRAC_INIT:  The initial condition should be none-negetive.")
        lower, upper = 1.0 - noise[name], 1.0 + noise[name]
        nsteps = int(round((upper - lower) / 1.0e-4))
        lattice = lower + 1.0e-4 * rng.integers(0, nsteps + 1, size=shape)
        a = np.asfortranarray(float(ic[name]) * lattice)
        a *= grid.landmask
        fill_halo_tracer(a, grid)
        out.append(a)
    return out
