"""ctypes mirror of include/pib200.h (structs, constants and prototypes)."""
import ctypes as ct

PI_OK, PI_ERR_ARG, PI_ERR_SHAPE, PI_ERR_PARAM, PI_ERR_CAPACITY = 0, 1, 2, 3, 4
PI_ERR_CUDA, PI_ERR_TIMEOUT, PI_ERR_NAN, PI_ERR_DOMAIN, PI_ERR_NOMEM, PI_ERR_STATE = 5, 6, 7, 8, 9, 10
PI_FP64, PI_FP32 = 0, 1
PI_PERIODIC, PI_BOUNDED = 0, 1

# Tracer order of the reference, src/Biogeochemistry/Biogeochemistry.jl:20
tracer_names = ("DIC", "NH4", "NO3", "PO4", "DFe", "DOC", "DON", "DOP",
                "PFe_inorg", "POC", "PON", "POP", "PFe_bio", "Dust")
NTRACERS = len(tracer_names)

FACES = {"west": 0, "east": 1, "south": 2, "north": 3, "bottom": 4, "top": 5}
PI_BC_NONE, PI_BC_CONST, PI_BC_ARRAY2D, PI_BC_ARRAY3D = 0, 1, 2, 3
PI_DIAG_PAR, PI_DIAG_NUM, PI_DIAG_GRAZ, PI_DIAG_MORT, PI_DIAG_DVID = 0, 1, 2, 3, 4
PI_DIAG_PTC, PI_DIAG_ABIO_NUM = 5, 6
PI_DIAG_TRACER, PI_DIAG_PROC = 16, 32
# draw purposes of include/pi_numerics.h
PI_DRAW_DIFFUSION, PI_DRAW_DECISION, PI_DRAW_ABIO_DIFFUSION, PI_DRAW_ABIO_BC, PI_DRAW_RELEASE = 0, 1, 2, 3, 4
# QuotaMode processes of diags_spcs! (src/Diagnostics/diagnostics_kernels.jl:22-23), in PI_PROC_* order
PROC_NAMES = ("PS", "BS", "VDOC", "VNH4", "VNO3", "VPO4", "resp", "exu", "Bm", "Cq", "Nq", "Pq", "Chl")

_dp = ct.POINTER(ct.c_double)
_i64p = ct.POINTER(ct.c_int64)
_u8p = ct.POINTER(ct.c_uint8)


class pi_grid_metrics(ct.Structure):
    _fields_ = [("dxC", _dp), ("dyC", _dp), ("dxF", _dp), ("dyF", _dp), ("Az", _dp),
                ("Ax", _dp), ("Ay", _dp), ("Vol", _dp)]


class pi_grid(ct.Structure):
    _fields_ = [("Nx", ct.c_int32), ("Ny", ct.c_int32), ("Nz", ct.c_int32),
                ("Hx", ct.c_int32), ("Hy", ct.c_int32), ("Hz", ct.c_int32),
                ("topo", ct.c_int32 * 3),
                ("dx", ct.c_double), ("dy", ct.c_double),
                ("dzF", _dp), ("dzC", _dp), ("landmask", _u8p),
                ("metrics", ct.POINTER(pi_grid_metrics))]


# bgc_params_default keys (src/Parameters/param_default.jl:44-71) in struct order
BGC_FIELDS = [("kw", "kw"), ("kc", "kc"), ("kDOC", "kDOC"), ("Nit", "Nit"), ("kDON", "kDON"),
              ("kDOP", "kDOP"), ("kPOC", "kPOC"), ("kPON", "kPON"), ("kPOP", "kPOP"),
              ("kappa_h", "κh"), ("kappa_v", "κv"), ("kappa_hP", "κhP"), ("kappa_vP", "κvP"),
              ("shared_graz", "shared_graz"), ("w_sink_org", "w_sink_org"),
              ("w_sink_inorg", "w_sink_inorg"), ("lambda_POC", "lambda_POC"),
              ("lambda_min", "lambda_min"), ("kdiss", "kdiss"), ("lambda_dust", "lambda_dust"),
              ("lambda_Fe", "lambda_Fe"), ("ligand", "ligand"), ("DFeFrac", "DFeFrac")]


class pi_bgc_params(ct.Structure):
    _fields_ = [(c, ct.c_double) for c, _ in BGC_FIELDS]


# QuotaMode param_names (src/Individuals/Plankton/QuotaMode/plankton_generation.jl:16-20)
QUOTA_FIELDS = [("Nsuper", "Nsuper"), ("Cquota", "Cquota"), ("mean", "mean"), ("var", "var"),
                ("Chl2Cint", "Chl2Cint"), ("alpha", "α"), ("Phi", "Φ"), ("Topt", "Topt"),
                ("Tmax", "Tmax"), ("Ea", "Ea"), ("PCmax", "PCmax"), ("VDOCmax", "VDOCmax"),
                ("VNO3max", "VNO3max"), ("VNH4max", "VNH4max"), ("VPO4max", "VPO4max"),
                ("KsatDOC", "KsatDOC"), ("KsatNH4", "KsatNH4"), ("KsatNO3", "KsatNO3"),
                ("KsatPO4", "KsatPO4"), ("Cqmax", "Cqmax"), ("Nqmax", "Nqmax"),
                ("Pqmax", "Pqmax"), ("Chl2N", "Chl2N"), ("R_NC", "R_NC"), ("R_PC", "R_PC"),
                ("k_mtb", "k_mtb"), ("respir", "respir"), ("grz_P", "grz_P"),
                ("dvid_type", "dvid_type"), ("dvid_P", "dvid_P"), ("dvid_reg", "dvid_reg"),
                ("dvid_reg2", "dvid_reg2"), ("mort_P", "mort_P"), ("mort_reg", "mort_reg"),
                ("grazFracC", "grazFracC"), ("grazFracN", "grazFracN"),
                ("grazFracP", "grazFracP"), ("mortFracC", "mortFracC"),
                ("mortFracN", "mortFracN"), ("mortFracP", "mortFracP")]


class pi_quota_params(ct.Structure):
    _fields_ = [(c, ct.c_double) for c, _ in QUOTA_FIELDS]


# CarbonMode param_names (src/Individuals/Plankton/CarbonMode/plankton_generation.jl:13-15)
CARBON_FIELDS = [("Nsuper", "Nsuper"), ("Cquota", "Cquota"), ("mean", "mean"), ("var", "var"),
                 ("alpha", "α"), ("Phi", "Φ"), ("Topt", "Topt"), ("Tmax", "Tmax"), ("Ea", "Ea"),
                 ("PCmax", "PCmax"), ("Chl2C", "Chl2C"), ("respir", "respir"), ("f_T2B", "f_T2B"),
                 ("grz_P", "grz_P"), ("dvid_type", "dvid_type"), ("dvid_P", "dvid_P"),
                 ("dvid_reg", "dvid_reg"), ("dvid_reg2", "dvid_reg2"), ("mort_P", "mort_P"),
                 ("mort_reg", "mort_reg"), ("grazFracC", "grazFracC"), ("mortFracC", "mortFracC"),
                 ("thermal", "thermal"), ("is_bact", "is_bact")]


class pi_carbon_params(ct.Structure):
    _fields_ = [(c, ct.c_double) for c, _ in CARBON_FIELDS]


# CarbonMode processes of diags_spcs! (diagnostics_kernels.jl:16-17), in PI_CPROC_* order
CARBON_PROC_NAMES = ("PS", "BS", "RP", "RS", "TD", "Bm", "Bd", "Chl")

# MacroMolecularMode param_names (src/Individuals/Plankton/MacroMolecularMode/plankton_generation.jl:17-23)
MACRO_FIELDS = [("Nsuper", "Nsuper"), ("C_DNA", "C_DNA"), ("var", "var"), ("PRO2DNA", "PRO2DNA"),
                ("RNA2DNA", "RNA2DNA"), ("CH2DNA", "CH2DNA"), ("Chl2DNA", "Chl2DNA"), ("alpha", "α"),
                ("Phi", "Φ"), ("Topt", "Topt"), ("Tmax", "Tmax"), ("Ea", "Ea"), ("PCmax", "PCmax"),
                ("VDOCmax", "VDOCmax"), ("VNO3max", "VNO3max"), ("VNH4max", "VNH4max"),
                ("VPO4max", "VPO4max"), ("KsatDOC", "KsatDOC"), ("KsatNH4", "KsatNH4"),
                ("KsatNO3", "KsatNO3"), ("KsatPO4", "KsatPO4"), ("CHmax", "CHmax"), ("NSTmax", "NSTmax"),
                ("PSTmax", "PSTmax"), ("Chl2N", "Chl2N"), ("R_NC_PRO", "R_NC_PRO"), ("R_NC_DNA", "R_NC_DNA"),
                ("R_NC_RNA", "R_NC_RNA"), ("R_PC_DNA", "R_PC_DNA"), ("R_PC_RNA", "R_PC_RNA"),
                ("respir", "respir"), ("k_pro", "k_pro"), ("k_sat_pro", "k_sat_pro"), ("k_rna", "k_rna"),
                ("k_sat_rna", "k_sat_rna"), ("k_dna", "k_dna"), ("k_sat_dna", "k_sat_dna"),
                ("dvid_P", "dvid_P"), ("grz_P", "grz_P"), ("mort_P", "mort_P"), ("mort_reg", "mort_reg"),
                ("grazFracC", "grazFracC"), ("grazFracN", "grazFracN"), ("grazFracP", "grazFracP"),
                ("mortFracC", "mortFracC"), ("mortFracN", "mortFracN"), ("mortFracP", "mortFracP")]


class pi_macro_params(ct.Structure):
    _fields_ = [(c, ct.c_double) for c, _ in MACRO_FIELDS]


# MacroMolecularMode processes in PI_MPROC_* order (plank_avail_diags, diagnostics_struct.jl:148-149)
MACRO_PROC_NAMES = ("PS", "VDOC", "VNH4", "VNO3", "VPO4", "resp", "ρChl", "S_PRO", "S_DNA", "S_RNA", "exu",
                    "CH", "NST", "PST", "PRO", "DNA", "RNA", "Chl")
MACRO_POOLS = ("PRO", "DNA", "RNA", "CH", "NST", "PST")

# IronEnergyMode param_names (src/Individuals/Plankton/IronEnergyMode/plankton_generation.jl:27-36)
IRON_FIELDS = [(c, {"alpha": "α"}.get(c, c)) for c in (
    "Nsuper", "Cquota", "SA", "mean", "var", "Chl2Cint", "alpha", "Topt", "Tmax", "Ea", "is_nr", "is_croc", "is_tric",
    "PCmax", "VNO3max", "VNH4max", "VPO4max", "k_cf", "k_rs", "k_nr", "k_nf", "k_mtb", "e_cf", "e_rs", "e_nr", "e_nf",
    "k_Fe_ST2PS", "k_Fe_PS2ST", "k_Fe_ST2NR", "k_Fe_NR2ST", "k_Fe_ST2NF", "k_Fe_NF2ST",
    "KfePS", "KfeNR", "KfeNF", "KsatNH4", "KsatNO3", "KsatPO4", "KSAFe", "CHmax", "qNH4max", "qNO3max", "qPmax", "qFemax",
    "Chl2N", "R_NC", "R_PC", "NF_clock", "grz_P", "dvid_type", "dvid_P", "dvid_reg", "dvid_reg2", "mort_P", "mort_reg",
    "grazFracC", "grazFracN", "grazFracP", "grazFracFe", "mortFracC", "mortFracN", "mortFracP", "mortFracFe", "max_ptc")]


class pi_iron_params(ct.Structure):
    _fields_ = [(c, ct.c_double) for c, _ in IRON_FIELDS]


# IronEnergyMode processes in PI_IPROC_* order (diags_spcs!, diagnostics_kernels.jl:22-23, :ptc aside)
IRON_PROC_NAMES = ("PS", "CF", "ECF", "RS", "ERS", "NR", "ENR", "NF", "ENF", "BS", "VNH4", "VNO3", "VPO4", "VFe",
                   "PS2ST", "ST2PS", "NR2ST", "ST2NR", "NF2ST", "ST2NF", "Bm", "exEn", "CH", "qNO3", "qNH4", "qP",
                   "qFe", "qFePS", "qFeNR", "qFeNF", "Chl", "tdark")
IRON_POOLS = ("CH", "qNO3", "qNH4", "qP", "qFe", "qFePS", "qFeNR", "qFeNF", "exEn", "tdark")


IND_DOUBLE = ("x", "y", "z", "Sz", "Bm", "Cq", "Nq", "Pq", "Chl", "gen", "age", "graz", "mort", "dvid")
IND_INT = ("xi", "yi", "zi")


class pi_individuals(ct.Structure):
    _fields_ = [("x", _dp), ("y", _dp), ("z", _dp),
                ("xi", _i64p), ("yi", _i64p), ("zi", _i64p),
                ("Sz", _dp), ("Bm", _dp), ("Cq", _dp), ("Nq", _dp), ("Pq", _dp),
                ("Chl", _dp), ("gen", _dp), ("age", _dp),
                ("ac", _u8p),
                ("graz", _dp), ("mort", _dp), ("dvid", _dp),
                ("Bd", _dp),
                ("PRO", _dp), ("DNA", _dp), ("RNA", _dp), ("CH", _dp), ("NST", _dp), ("PST", _dp),
                ("ptc", _dp),
                ("qNO3", _dp), ("qNH4", _dp), ("qP", _dp), ("qFe", _dp), ("qFePS", _dp), ("qFeNR", _dp),
                ("qFeNF", _dp), ("exEn", _dp), ("tdark", _dp)]


# construct_abiotic_particle's param_names (src/Individuals/Abiotic/particle_generation.jl:7)
ABIOTIC_FIELDS = ("Nsuper", "Rd", "release_P", "sz_min", "Ktr")


class pi_abiotic_params(ct.Structure):
    _fields_ = [(k, ct.c_double) for k in ABIOTIC_FIELDS]


class pi_abiotic_particles(ct.Structure):
    _fields_ = [("x", _dp), ("y", _dp), ("z", _dp), ("xi", _i64p), ("yi", _i64p), ("zi", _i64p), ("ac", _u8p)]


class pi_member(ct.Structure):
    _fields_ = [("grid", ct.POINTER(pi_grid)), ("bgc", ct.POINTER(pi_bgc_params)),
                ("species", ct.POINTER(pi_quota_params)), ("capacity", ct.c_int64), ("seed", ct.c_uint64)]


def declare(lib, prefix):
    """Attach argtypes/restype for the pi_* (or mirrored) entry points found in `lib`."""
    P = ct.c_void_p
    protos = {
        "create": (ct.c_int32, [ct.POINTER(pi_grid), ct.POINTER(pi_bgc_params),
                                ct.POINTER(pi_quota_params), ct.c_int32, ct.c_int64]),
        "destroy": (ct.c_int32, [P]),
        "set_individuals": (ct.c_int32, [P, ct.c_int32, ct.POINTER(pi_individuals)]),
        "get_individuals": (ct.c_int32, [P, ct.c_int32, ct.POINTER(pi_individuals)]),
        "set_tracer": (ct.c_int32, [P, ct.c_int32, _dp]),
        "get_tracer": (ct.c_int32, [P, ct.c_int32, _dp]),
        "set_velocity": (ct.c_int32, [P, _dp, _dp, _dp]),
        "set_velocity0": (ct.c_int32, [P, _dp, _dp, _dp]),
        "set_PARF": (ct.c_int32, [P, _dp]),
        "set_temp": (ct.c_int32, [P, _dp]),
        "set_flux_bc": (ct.c_int32, [P, ct.c_int32, ct.c_int32, ct.c_int32, _dp, ct.c_int64]),
        "time_step": (ct.c_int32, [P, ct.c_double]),
        "get_time": (ct.c_int32, [P, _i64p, _dp]),
        "set_time": (ct.c_int32, [P, ct.c_int64, ct.c_double]),
        "count_active": (ct.c_int32, [P, ct.c_int32, _i64p]),
        "get_diag": (ct.c_int32, [P, ct.c_int32, ct.c_int32, _dp]),
        "get_budget": (ct.c_int32, [P, _dp]),
        "create_carbon": (ct.c_int32, [ct.POINTER(pi_grid), ct.POINTER(pi_bgc_params),
                                       ct.POINTER(pi_carbon_params), ct.c_int32, ct.c_int64]),
        "create_macro": (ct.c_int32, [ct.POINTER(pi_grid), ct.POINTER(pi_bgc_params),
                                      ct.POINTER(pi_macro_params), ct.c_int32, ct.c_int64]),
        "create_iron": (ct.c_int32, [ct.POINTER(pi_grid), ct.POINTER(pi_bgc_params),
                                     ct.POINTER(pi_iron_params), ct.c_int32, ct.c_int64]),
        "last_error": (ct.c_int32, [P, ct.c_char_p, ct.c_size_t]),
        "set_abiotics": (ct.c_int32, [P, ct.c_int32, ct.POINTER(pi_abiotic_params), ct.c_int32,
                                      ct.POINTER(ct.c_int32), ct.c_int32, ct.POINTER(ct.c_int32), ct.c_int32, _dp]),
        "set_abiotic_particles": (ct.c_int32, [P, ct.c_int32, ct.POINTER(pi_abiotic_particles)]),
        "get_abiotic_particles": (ct.c_int32, [P, ct.c_int32, ct.POINTER(pi_abiotic_particles)]),
        "count_abiotic": (ct.c_int32, [P, ct.c_int32, _i64p]),
        "set_abiotic_bc": (ct.c_int32, [P, ct.c_int32, ct.c_int32, ct.c_int32, _dp, ct.c_int64]),
    }
    for name, (res, args) in protos.items():
        fn = getattr(lib, prefix + name, None)
        if fn is None:
            continue
        if name in ("create", "create_carbon", "create_macro", "create_iron"):
            if prefix == "pi_":
                args = args + [ct.c_int32, ct.c_uint64, ct.POINTER(P)]
            else:
                args = args + [ct.c_uint64, ct.POINTER(P)]
        fn.restype = res
        fn.argtypes = args
    return lib
