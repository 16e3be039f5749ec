"""Parameter sets and default forcing (src/Parameters/param_default.jl,
src/Parameters/param_update.jl). Parameters are plain dicts keyed like the reference's."""
import numpy as np


def default_PARF(grid, ΔT, iterations):
    """Hourly surface PAR of one day repeated over the run (param_default.jl:5-16).
    Shape (Nx, Ny, 24*days)."""
    PAR = [0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.3871666666666666, 87.10258333333333, 475.78150000000016,
           929.2737916666669, 1232.3633333333337, 1638.918916666667, 1823.7921666666664,
           1906.2769583333336, 1776.0280416666667, 1678.5026249999999, 1410.216666666667,
           815.4129583333336, 525.104, 135.993, 2.9493750000000003, 0.0, 0.0, 0.0]
    total_days = int((ΔT * iterations) // 86400 + 1)
    day = np.zeros((grid.Nx, grid.Ny, 24), order="F")
    for i in range(24):
        day[:, :, i] = PAR[i]
    return np.asfortranarray(np.tile(day, (1, 1, total_days)))


def default_temperature(grid, ΔT, iterations):
    """Hourly temperature with a vertical gradient (param_default.jl:22-38).
    Shape (Nx, Ny, Nz, 24*days)."""
    temp = [26.646446609406727, 26.56698729810778, 26.517037086855467, 26.5, 26.517037086855467,
            26.56698729810778, 26.646446609406727, 26.75, 26.87059047744874, 27.0, 27.12940952255126,
            27.25, 27.353553390593273, 27.43301270189222, 27.482962913144533, 27.5,
            27.482962913144533, 27.43301270189222, 27.353553390593273, 27.25, 27.12940952255126,
            27.0, 26.87059047744874, 26.75]
    total_days = int((ΔT * iterations) // 86400 + 1)
    Nz = grid.Nz
    day = np.zeros((grid.Nx, grid.Ny, Nz, 24), order="F")
    for i in range(24):
        day[:, :, Nz - 1, i] = temp[i]
    zC = np.asarray(grid.zC, dtype=np.float64)
    for j in range(Nz - 1, 0, -1):   # j = Nz-1 ... 1 (1-based)
        day[:, :, j - 1, :] = day[:, :, j, :] + 4.0e-4 * zC[j - 1]
    return np.asfortranarray(np.tile(day, (1, 1, 1, total_days)))


def bgc_params_default(FT=np.float32):
    """bgc_params_default(FT) (param_default.jl:44-71)."""
    FT = np.dtype(FT).type
    p = {
        "kw": 0.046, "kc": 0.04,
        "kDOC": 1 / 30 / 86400, "Nit": 1 / 30 / 86400, "kDON": 1 / 30 / 86400,
        "kDOP": 1 / 30 / 86400, "kPOC": 1 / 30 / 86400, "kPON": 1 / 30 / 86400,
        "kPOP": 1 / 30 / 86400,
        "κh": 0.0e-6, "κv": 0.0e-6, "κhP": 0.0e-6, "κvP": 0.0e-6,
        "shared_graz": 1.0,
        "w_sink_org": 2.31e-8, "w_sink_inorg": 2.31e-5,
        "lambda_POC": 5.8e-8, "lambda_min": 3.5e-10, "kdiss": 4.4e-7, "lambda_dust": 1.7e-3,
        "lambda_Fe": 1.7, "ligand": 6.0e-4, "DFeFrac": 0.01,
    }
    return {k: FT(v) for k, v in p.items()}


def phyt_params_default(N=1, mode=None):
    """phyt_params_default(N, QuotaMode()) (param_default.jl:235-284), for CarbonMode()
    param_default.jl:290-320, for MacroMolecularMode() param_default.jl:94-141; one list entry per
    species."""
    from .architectures import CarbonMode, IronEnergyMode, MacroMolecularMode
    if isinstance(mode, IronEnergyMode) or mode is IronEnergyMode:          # param_default.jl:156-228
        params = {
            "Nsuper": [1], "Cquota": [1.8e-11], "SA": [0.18], "mean": [1.2], "var": [0.3], "Chl2Cint": [0.10],
            "α": [4.5e-2], "Topt": [27.0], "Tmax": [30.0], "Ea": [5.3e4], "is_nr": [1.0], "is_croc": [0.0],
            "is_tric": [0.0], "PCmax": [7.8e-8], "VNH4max": [6.9e-6], "VNO3max": [6.9e-6], "VPO4max": [1.2e-6],
            "k_cf": [1.0e-5], "k_rs": [1.5e-6], "k_nr": [2.8e-6], "k_nf": [2.8e-6], "k_mtb": [3.5e-5],
            "e_cf": [9.0], "e_rs": [5.0], "e_nf": [8.0], "e_nr": [10.0], "k_Fe_ST2PS": [2.4e-5],
            "k_Fe_PS2ST": [1.2e-6], "k_Fe_ST2NR": [1.2e-5], "k_Fe_NR2ST": [1.2e-5], "k_Fe_ST2NF": [1.2e-5],
            "k_Fe_NF2ST": [1.2e-5], "KfePS": [3.0e-6], "KfeNR": [2.0e-6], "KfeNF": [5.0e-6], "KsatNH4": [0.005],
            "KsatNO3": [0.010], "KsatPO4": [0.003], "KSAFe": [2.77e-19], "qNO3max": [0.25], "qNH4max": [0.25],
            "qPmax": [0.02], "qFemax": [2.0e-5], "CHmax": [0.4], "Chl2N": [3.0], "R_NC": [16 / 106],
            "R_PC": [1 / 106], "NF_clock": [21600.0], "grz_P": [0.0], "dvid_P": [1e-4], "dvid_type": [1],
            "dvid_reg": [2.5], "dvid_reg2": [12.0], "mort_P": [5e-5], "mort_reg": [0.5], "grazFracC": [0.7],
            "grazFracN": [0.7], "grazFracP": [0.7], "grazFracFe": [0.1], "mortFracC": [0.5], "mortFracN": [0.5],
            "mortFracP": [0.5], "mortFracFe": [0.1], "max_ptc": [25],
        }
        return params if N == 1 else {k: [v[0]] * N for k, v in params.items()}
    if isinstance(mode, MacroMolecularMode) or mode is MacroMolecularMode:
        params = {
            "Nsuper": [1], "C_DNA": [1.8e-13], "var": [0.3], "RNA2DNA": [1.73], "PRO2DNA": [34.83],
            "CH2DNA": [23.3], "Chl2DNA": [3.45], "α": [2.0e-2], "Φ": [4.0e-5], "Topt": [27.0],
            "Tmax": [30.0], "Ea": [5.3e4], "PCmax": [6.2e-5], "VDOCmax": [0.0], "VNH4max": [6.9e-6],
            "VNO3max": [6.9e-6], "VPO4max": [1.2e-6], "KsatNH4": [0.005], "KsatNO3": [0.010],
            "KsatPO4": [0.003], "KsatDOC": [0.0], "NSTmax": [0.12], "PSTmax": [0.70], "CHmax": [0.4],
            "respir": [1.2e-6], "k_pro": [6.0e-5], "k_sat_pro": [4.5e-13], "k_dna": [1.6e-7],
            "k_sat_dna": [1.0e-15], "k_rna": [3.0e-7], "k_sat_rna": [1.0e-12], "Chl2N": [3.0],
            "R_NC_PRO": [1 / 4.5], "R_NC_DNA": [1 / 2.9], "R_PC_DNA": [1 / 11.1], "R_NC_RNA": [1 / 2.8],
            "R_PC_RNA": [1 / 10.7], "dvid_P": [1.0e-5], "grz_P": [0.0], "mort_P": [5e-5],
            "mort_reg": [0.5], "grazFracC": [0.7], "grazFracN": [0.7], "grazFracP": [0.7],
            "mortFracC": [0.5], "mortFracN": [0.5], "mortFracP": [0.5],
        }
        return params if N == 1 else {k: [v[0]] * N for k, v in params.items()}
    if isinstance(mode, CarbonMode) or mode is CarbonMode:
        params = {
            "Nsuper": [1], "Cquota": [1.8e-11], "mean": [1.2], "var": [0.3], "Chl2C": [0.10],
            "α": [2.0e-2], "Φ": [4.0e-5], "Topt": [27.0], "Tmax": [30.0], "Ea": [5.3e4],
            "PCmax": [4.2e-5], "respir": [1.2e-6], "f_T2B": [2.7e-6], "grz_P": [0.0],
            "dvid_P": [5e-5], "dvid_type": [1], "dvid_reg": [1.9], "dvid_reg2": [12.0],
            "mort_P": [5e-5], "mort_reg": [0.5], "grazFracC": [0.7], "mortFracC": [0.5],
            "thermal": [1.0], "is_bact": [0.0],
        }
        return params if N == 1 else {k: [v[0]] * N for k, v in params.items()}
    params = {
        "Nsuper": [1], "Cquota": [1.8e-11], "mean": [1.2], "var": [0.3], "Chl2Cint": [0.10],
        "α": [2.0e-2], "Φ": [4.0e-5], "Topt": [27.0], "Tmax": [30.0], "Ea": [5.3e4],
        "PCmax": [4.2e-5], "VDOCmax": [0.0], "VNH4max": [6.9e-6], "VNO3max": [6.9e-6],
        "VPO4max": [1.2e-6], "KsatNH4": [0.005], "KsatNO3": [0.010], "KsatPO4": [0.003],
        "KsatDOC": [0.0], "Nqmax": [0.25], "Pqmax": [0.02], "Cqmax": [0.4], "k_mtb": [3.5e-5],
        "respir": [1.2e-6], "Chl2N": [3.0], "R_NC": [16 / 106], "R_PC": [1 / 106], "grz_P": [0.0],
        "dvid_P": [1e-4], "dvid_type": [1], "dvid_reg": [2.5], "dvid_reg2": [12.0],
        "mort_P": [5e-5], "mort_reg": [0.5], "grazFracC": [0.7], "grazFracN": [0.7],
        "grazFracP": [0.7], "mortFracC": [0.5], "mortFracN": [0.5], "mortFracP": [0.5],
    }
    if N == 1:
        return params
    return {k: [v[0]] * N for k, v in params.items()}    # generate_n_species_params, :345-352


def update_bgc_params(tmp, FT=np.float32):
    """update_bgc_params (param_update.jl:10-22)."""
    FT = np.dtype(FT).type
    parameters = bgc_params_default(FT)
    for key in tmp:
        if key not in parameters:
            raise ValueError(f"PARAM: bgc parameter not found {key}")
        parameters[key] = FT(tmp[key])
    return parameters


def update_phyt_params(tmp, FT=np.float32, *, N=1, mode=None):
    """update_phyt_params (param_update.jl:34-46)."""
    FT = np.dtype(FT).type
    parameters = phyt_params_default(N, mode)
    for key in tmp:
        if key not in parameters:
            raise ValueError(f"PARAM: phyt parameter not found {key}")
        parameters[key] = [FT(v) for v in np.atleast_1d(tmp[key])]
    return parameters


def abiotic_params_default(N=1):
    """abiotic_params_default(N) (src/Parameters/param_default.jl:329-343)."""
    params = {"Nsuper": [1.0], "Rd": [1.0e-4], "release_P": [1.0e-6], "sz_min": [1.0e-3], "Ktr": [0.0e-5]}
    return {k: v * N for k, v in params.items()}


def update_abiotic_params(tmp, FT=np.float32, *, N=1):
    """update_abiotic_params (src/Parameters/param_update.jl:57-69)."""
    FT = np.dtype(FT).type
    parameters = abiotic_params_default(N)
    for key in tmp:
        if key not in parameters:
            raise ValueError(f"PARAM: abiotic parameter not found {key}")
        parameters[key] = [FT(v) for v in np.atleast_1d(tmp[key])]
    return parameters


def default_tracer_init():
    """default_tracer_init() (tracer_fields.jl:41-45)."""
    init = dict(DIC=20.0, NH4=0.5, NO3=0.8, PO4=0.10, DFe=1.0e-6, DOC=10.0, DON=0.1, DOP=0.05,
                PFe_inorg=0.0, POC=0.0, PON=0.0, POP=0.0, PFe_bio=0.0, Dust=0.0)
    rand_noise = {k: 0.1 for k in init}
    return dict(initial_condition=init, rand_noise=rand_noise)
