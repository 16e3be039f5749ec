/*
 * pib200.h — C ABI of libpib200, the B200 (sm_100a) model time step of PlanktonIndividuals.jl.
 *
 * The reference has no FFI: its public surface is the Julia API (src/PlanktonIndividuals.jl:7-42)
 * RectilinearGrid → PlanktonModel → PlanktonSimulation → update!, with TimeStep! underneath.
 * Each entry point below names the reference function whose job it takes over. A Julia `ccall`
 * shim on the reference side and the Python package `PlanktonIndividuals` in this repository
 * bind exactly these symbols.
 *
 * Conventions
 *  - Arrays cross the boundary as host pointers in Julia column-major order (x fastest), with the
 *    shapes the reference uses: grid fields are (Nx+2Hx, Ny+2Hy, Nz+2Hz) including halos,
 *    individual attributes are `capacity` long (max_individuals, src/Model/models.jl:54).
 *  - Host pointers are borrowed for the duration of the call and copied; calls are synchronous
 *    unless stated. The library owns all device memory of a handle. A handle belongs to one host
 *    thread at a time and runs on its own CUDA stream of the device that was current at
 *    pi_create.
 *  - Every call returns PI_OK or an error code; pi_last_error gives the message. Messages of
 *    validation errors repeat the reference's ArgumentError texts.
 *  - Quantities are Float64 at the boundary. PI_FP64 models compute in Float64 (the plain
 *    drop-in); PI_FP32 models store and compute the bulk of the step in Float32.
 *  - Indices (xi, yi, zi) are the reference's 1-based Julia indices including the halo offset.
 */
#ifndef PIB200_H
#define PIB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t pi_status;

#define PI_OK            0
#define PI_ERR_ARG       1   /* bad argument, NULL pointer, unsupported option            */
#define PI_ERR_SHAPE     2   /* dimension mismatch (src/Simulation/utils.jl:213-304)      */
#define PI_ERR_PARAM     3   /* parameter value rejected (src/Parameters/param_update.jl) */
#define PI_ERR_CAPACITY  4   /* division overflow (QuotaMode/plankton_update.jl:20-22)    */
#define PI_ERR_CUDA      5   /* CUDA runtime error or no usable device                    */
#define PI_ERR_TIMEOUT   6   /* a bounded device-side wait gave up                        */
#define PI_ERR_NAN       7   /* NaN or Inf found by pi_check_finite                       */
#define PI_ERR_DOMAIN    8   /* an individual's cell index left the halo-padded grid      */
#define PI_ERR_NOMEM     9   /* device allocation failed                                  */
#define PI_ERR_STATE    10   /* call not valid in the handle's current state              */

#define PI_FP64 0
#define PI_FP32 1

#define PI_PERIODIC 0
#define PI_BOUNDED  1

/* Tracer order of the reference (src/Biogeochemistry/Biogeochemistry.jl:20). */
enum {
    PI_DIC = 0, PI_NH4, PI_NO3, PI_PO4, PI_DFe, PI_DOC, PI_DON, PI_DOP,
    PI_PFe_inorg, PI_POC, PI_PON, PI_POP, PI_PFe_bio, PI_Dust, PI_NTRACERS
};

/* Flux boundary faces and kinds (src/Biogeochemistry/HaloRegions/apply_bcs.jl:87-98). */
enum { PI_WEST = 0, PI_EAST, PI_SOUTH, PI_NORTH, PI_BOTTOM, PI_TOP };
enum { PI_BC_NONE = 0, PI_BC_CONST, PI_BC_ARRAY2D, PI_BC_ARRAY3D };

/* Diagnostics kept by TimeStep! (src/Diagnostics/diagnostics_struct.jl:23-105): the defaults,
 * and the optional ones of PlanktonDiagnostics(model; tracer, phytoplankton) enabled with
 * pi_set_diags: PI_DIAG_TRACER + tracer index (diags.tracer[name], time_step.jl:168-172) and
 * PI_DIAG_PROC + process index (diags.phytos[sp][process], diags_spcs!,
 * Diagnostics/diagnostics_kernels.jl:14-33) in QuotaMode's order below. */
enum { PI_DIAG_PAR = 0, PI_DIAG_NUM, PI_DIAG_GRAZ, PI_DIAG_MORT, PI_DIAG_DVID,
       PI_DIAG_PTC,        /* diags.phytos[sp].ptc: Σ ptc·ac per cell (time_step.jl:140-149), kept
                              while the model has abiotic species                               */
       PI_DIAG_ABIO_NUM,   /* diags.abiotics[sa].num (time_step.jl:151-158): sp is the abiotic
                              species                                                            */
       PI_DIAG_TRACER = 16, PI_DIAG_PROC = 32 };
enum { PI_PROC_PS = 0, PI_PROC_BS, PI_PROC_VDOC, PI_PROC_VNH4, PI_PROC_VNO3, PI_PROC_VPO4, PI_PROC_resp,
       PI_PROC_exu, PI_PROC_Bm, PI_PROC_Cq, PI_PROC_Nq, PI_PROC_Pq, PI_PROC_Chl, PI_NPROC };
/* The processes of a CarbonMode model (diags_spcs!, diagnostics_kernels.jl:16-17), the same
 * PI_DIAG_PROC + q kinds and proc_mask bits. */
enum { PI_CPROC_PS = 0, PI_CPROC_BS, PI_CPROC_RP, PI_CPROC_RS, PI_CPROC_TD, PI_CPROC_Bm, PI_CPROC_Bd,
       PI_CPROC_Chl, PI_NCPROC };
/* The processes of a MacroMolecularMode model, in the order of plank_avail_diags
 * (Diagnostics/diagnostics_struct.jl:148-149). diags_spcs! (diagnostics_kernels.jl:20-21) lists
 * VNH4 as :VHN4 and has no :exu, so those two fields are kept and stay zero, as there. */
enum { PI_MPROC_PS = 0, PI_MPROC_VDOC, PI_MPROC_VNH4, PI_MPROC_VNO3, PI_MPROC_VPO4, PI_MPROC_resp,
       PI_MPROC_rChl, PI_MPROC_S_PRO, PI_MPROC_S_DNA, PI_MPROC_S_RNA, PI_MPROC_exu, PI_MPROC_CH,
       PI_MPROC_NST, PI_MPROC_PST, PI_MPROC_PRO, PI_MPROC_DNA, PI_MPROC_RNA, PI_MPROC_Chl, PI_NMPROC };
/* The processes of an IronEnergyMode model (diags_spcs!, diagnostics_kernels.jl:22-23, without
 * :ptc, which is PI_DIAG_PTC): 32 fields, all bits of proc_mask. */
enum { PI_IPROC_PS = 0, PI_IPROC_CF, PI_IPROC_ECF, PI_IPROC_RS, PI_IPROC_ERS, PI_IPROC_NR, PI_IPROC_ENR,
       PI_IPROC_NF, PI_IPROC_ENF, PI_IPROC_BS, PI_IPROC_VNH4, PI_IPROC_VNO3, PI_IPROC_VPO4, PI_IPROC_VFe,
       PI_IPROC_PS2ST, PI_IPROC_ST2PS, PI_IPROC_NR2ST, PI_IPROC_ST2NR, PI_IPROC_NF2ST, PI_IPROC_ST2NF,
       PI_IPROC_Bm, PI_IPROC_exEn, PI_IPROC_CH, PI_IPROC_qNO3, PI_IPROC_qNH4, PI_IPROC_qP, PI_IPROC_qFe,
       PI_IPROC_qFePS, PI_IPROC_qFeNR, PI_IPROC_qFeNF, PI_IPROC_Chl, PI_IPROC_tdark, PI_NIPROC };

/* The horizontal metrics of a LatLonGrid (src/Grids/lat_lon_grid.jl:1-45, built by
 * LatLonGrid :57-170 or LoadLatLonGrid :196-316), as the reference stores them: halos included,
 * Julia column-major. ΔxC, ΔyC, ΔxF, ΔyF, Ax, Ay, Az and volume read these arrays
 * (Grids/areas_volumes_spacings.jl:27-38) where a RectilinearGrid uses Δx, Δy and dzF. */
typedef struct {
    const double *dxC, *dyC;    /* (Nx+2Hx)(Ny+2Hy): center-to-center spacings, m          */
    const double *dxF, *dyF;    /* (Nx+2Hx)(Ny+2Hy): face-to-face spacings, m              */
    const double *Az;           /* (Nx+2Hx)(Ny+2Hy): area of a horizontal face, m²          */
    const double *Ax, *Ay;      /* (Nx+2Hx)(Ny+2Hy)(Nz+2Hz): areas of the x and y faces, m² */
    const double *Vol;          /* (Nx+2Hx)(Ny+2Hy)(Nz+2Hz): cell volumes, m³               */
} pi_grid_metrics;

/* RectilinearGrid (src/Grids/rectilinear_grid.jl:1-25) or, with `metrics`, LatLonGrid
 * (src/Grids/lat_lon_grid.jl:1-45). Metrics are passed as the reference stores them after
 * construction (rectilinear_grid.jl:57-122), halos included. */
typedef struct {
    int32_t Nx, Ny, Nz;
    int32_t Hx, Hy, Hz;
    int32_t topo[3];            /* PI_PERIODIC or PI_BOUNDED for x, y, z                   */
    double  dx, dy;             /* Δx, Δy (RectilinearGrid; unused with metrics)           */
    const double*  dzF;         /* Nz+2Hz, g.dzF                                           */
    const double*  dzC;         /* Nz+2Hz, g.dzC                                           */
    const uint8_t* landmask;    /* (Nx+2Hx)(Ny+2Hy)(Nz+2Hz) with halos (Grids/utils.jl:92-129),
                                   NULL = all water                                        */
    const pi_grid_metrics* metrics;   /* NULL: RectilinearGrid. Otherwise the LatLonGrid
                                         arrays (FP64 form only; the FP32 form and
                                         pi_tracer_advection_noalloc return PI_ERR_ARG) */
} pi_grid;

/* Biogeochemical parameters, names and meaning of bgc_params_default
 * (src/Parameters/param_default.jl:44-71). */
typedef struct {
    double kw, kc, kDOC, Nit, kDON, kDOP, kPOC, kPON, kPOP;
    double kappa_h, kappa_v, kappa_hP, kappa_vP;     /* κh, κv, κhP, κvP */
    double shared_graz;
    double w_sink_org, w_sink_inorg;
    double lambda_POC, lambda_min, kdiss, lambda_dust, lambda_Fe, ligand, DFeFrac;
} pi_bgc_params;

/* QuotaMode phytoplankton parameters of one species, in the reference's param_names order
 * (src/Individuals/Plankton/QuotaMode/plankton_generation.jl:16-20). */
typedef struct {
    double Nsuper, Cquota, mean, var, Chl2Cint, alpha, Phi, Topt, Tmax, Ea;
    double PCmax, VDOCmax, VNO3max, VNH4max, VPO4max;
    double KsatDOC, KsatNH4, KsatNO3, KsatPO4, Cqmax, Nqmax, Pqmax;
    double Chl2N, R_NC, R_PC, k_mtb, respir, grz_P, dvid_type, dvid_P, dvid_reg, dvid_reg2;
    double mort_P, mort_reg, grazFracC, grazFracN, grazFracP, mortFracC, mortFracN, mortFracP;
} pi_quota_params;

/* CarbonMode phytoplankton parameters of one species, in the reference's param_names order
 * (src/Individuals/Plankton/CarbonMode/plankton_generation.jl:13-15); thermal = 1 switches on
 * thermal damage and repair, is_bact = 1 makes photosynthesis independent of light. */
typedef struct {
    double Nsuper, Cquota, mean, var, alpha, Phi, Topt, Tmax, Ea, PCmax, Chl2C, respir, f_T2B;
    double grz_P, dvid_type, dvid_P, dvid_reg, dvid_reg2, mort_P, mort_reg, grazFracC, mortFracC;
    double thermal, is_bact;
} pi_carbon_params;

/* MacroMolecularMode phytoplankton parameters of one species, in the reference's param_names
 * order (src/Individuals/Plankton/MacroMolecularMode/plankton_generation.jl:17-23). */
typedef struct {
    double Nsuper, C_DNA, var, PRO2DNA, RNA2DNA, CH2DNA, Chl2DNA, alpha, Phi, Topt, Tmax, Ea;
    double PCmax, VDOCmax, VNO3max, VNH4max, VPO4max, KsatDOC, KsatNH4, KsatNO3, KsatPO4;
    double CHmax, NSTmax, PSTmax, Chl2N, R_NC_PRO, R_NC_DNA, R_NC_RNA, R_PC_DNA, R_PC_RNA, respir;
    double k_pro, k_sat_pro, k_rna, k_sat_rna, k_dna, k_sat_dna;
    double dvid_P, grz_P, mort_P, mort_reg, grazFracC, grazFracN, grazFracP, mortFracC, mortFracN, mortFracP;
} pi_macro_params;

/* IronEnergyMode phytoplankton parameters of one species, in the reference's param_names order
 * (src/Individuals/Plankton/IronEnergyMode/plankton_generation.jl:27-36). */
typedef struct {
    double Nsuper, Cquota, SA, mean, var, Chl2Cint, alpha, Topt, Tmax, Ea, is_nr, is_croc, is_tric;
    double PCmax, VNO3max, VNH4max, VPO4max, k_cf, k_rs, k_nr, k_nf, k_mtb, e_cf, e_rs, e_nr, e_nf;
    double k_Fe_ST2PS, k_Fe_PS2ST, k_Fe_ST2NR, k_Fe_NR2ST, k_Fe_ST2NF, k_Fe_NF2ST;
    double KfePS, KfeNR, KfeNF, KsatNH4, KsatNO3, KsatPO4, KSAFe, CHmax, qNH4max, qNO3max, qPmax, qFemax;
    double Chl2N, R_NC, R_PC, NF_clock, grz_P, dvid_type, dvid_P, dvid_reg, dvid_reg2, mort_P, mort_reg;
    double grazFracC, grazFracN, grazFracP, grazFracFe, mortFracC, mortFracN, mortFracP, mortFracFe, max_ptc;
} pi_iron_params;

/* The persistent per-individual state of one species (QuotaMode struct-of-arrays,
 * plankton_generation.jl:2-13; CarbonMode, CarbonMode/plankton_generation.jl:2-11, keeps Bd, the
 * damaged biomass, and no Cq, Nq, Pq). Every array is `capacity` long. graz/mort/dvid carry the
 * 0/1 decisions drawn at the end of a step and applied at the start of the next. For
 * pi_set_individuals every member the mode uses is required (Bd: CarbonMode only; Cq, Nq, Pq:
 * QuotaMode only); for pi_get_individuals NULL members are skipped. */
typedef struct {
    double  *x, *y, *z;
    int64_t *xi, *yi, *zi;
    double  *Sz, *Bm, *Cq, *Nq, *Pq, *Chl, *gen, *age;
    uint8_t *ac;
    double  *graz, *mort, *dvid;
    double  *Bd;
    double  *PRO, *DNA, *RNA, *CH, *NST, *PST;   /* MacroMolecularMode only (protein, DNA, RNA,
                                                  carbohydrate/lipid, N and P reserves) */
    double  *ptc;                                /* abiotic particles held (every mode); NULL on
                                                  pi_set_individuals sets zeros */
    double  *qNO3, *qNH4, *qP, *qFe, *qFePS, *qFeNR, *qFeNF, *exEn, *tdark;   /* IronEnergyMode
                                                  only, with CH: N, P and Fe (storage, photosystem,
                                                  nitrate reductase, nitrogenase) quotas, excess
                                                  energy and the time since sunset */
} pi_individuals;

typedef struct pi_model pi_model;
typedef struct pi_sim   pi_sim;

/* PlanktonModel(arch, grid; FT, mode = QuotaMode(), max_individuals, bgc_params, phyto)
 * (src/Model/models.jl:51-155) and timestepper(...) (src/Model/timestepper.jl:23-60): allocates
 * the model state and scratch on the current CUDA device. Individuals start inactive and
 * tracers at zero until set. `seed` keys the model's random draws. */
pi_status pi_create(const pi_grid* grid, const pi_bgc_params* bgc,
                    const pi_quota_params* species, int32_t nspecies, int64_t capacity,
                    int32_t precision, uint64_t seed, pi_model** out);

/* PlanktonModel(arch, grid; mode = CarbonMode(), ...): as pi_create with CarbonMode species
 * (src/Individuals/Plankton/CarbonMode/). Built in the FP64 form (precision PI_FP64; PI_FP32 is
 * refused with PI_ERR_ARG). The other calls work as for a QuotaMode model; pi_get_budget reports
 * the individuals' carbon as ΣBm and no individual N or P. */
pi_status pi_create_carbon(const pi_grid* grid, const pi_bgc_params* bgc,
                           const pi_carbon_params* species, int32_t nspecies, int64_t capacity,
                           int32_t precision, uint64_t seed, pi_model** out);

/* PlanktonModel(arch, grid; mode = MacroMolecularMode(), ...): as pi_create with MacroMolecularMode
 * species (src/Individuals/Plankton/MacroMolecularMode/): individuals carry PRO, DNA, RNA, CH, NST,
 * PST, Chl, gen and age (Sz, Bm and the quotas are not used). Built in the FP64 form (precision
 * PI_FP64; PI_FP32 is refused with PI_ERR_ARG). pi_get_budget reports the individuals' carbon,
 * nitrogen and phosphorus from total_C/N/P_biomass (plankton_generation.jl:82-93). */
pi_status pi_create_macro(const pi_grid* grid, const pi_bgc_params* bgc,
                          const pi_macro_params* species, int32_t nspecies, int64_t capacity,
                          int32_t precision, uint64_t seed, pi_model** out);

/* PlanktonModel(arch, grid; mode = IronEnergyMode(), ...): as pi_create with IronEnergyMode species
 * (src/Individuals/Plankton/IronEnergyMode/): individuals carry Sz, Bm, CH, qNO3, qNH4, qP, qFe,
 * qFePS, qFeNR, qFeNF, exEn, Chl, tdark, gen and age; the step also reads DFe and the change of PAR
 * since the previous step, and its consumption and losses reach DFe and PFe_bio. Built in the FP64
 * form (precision PI_FP64; PI_FP32 is refused with PI_ERR_ARG). pi_get_budget reports the
 * individuals' C (Bm + CH), N (Bm·R_NC + qNO3 + qNH4) and P (Bm·R_PC + qP). */
pi_status pi_create_iron(const pi_grid* grid, const pi_bgc_params* bgc,
                         const pi_iron_params* species, int32_t nspecies, int64_t capacity,
                         int32_t precision, uint64_t seed, pi_model** out);

/* Releases every device allocation of the handle. */
pi_status pi_destroy(pi_model* m);

/* Individuals of species `sp` (0-based), as set by initialize_plankton!
 * (plankton_generation.jl:35-72) or read back for output/checkpoint. */
pi_status pi_set_individuals(pi_model* m, int32_t sp, const pi_individuals* in);
pi_status pi_get_individuals(pi_model* m, int32_t sp, pi_individuals* out);

/* Tracer `idx` (PI_DIC..PI_Dust) with halos, as model.tracers[name].data
 * (src/Biogeochemistry/tracer_fields.jl:60-101). */
pi_status pi_set_tracer(pi_model* m, int32_t idx, const double* data);
pi_status pi_get_tracer(pi_model* m, int32_t idx, double* out);

/* vel_copy!(vel₁, u, v, w, grid) (src/Simulation/utils.jl:5-11): interior velocities, sized
 * (Nx[+1], Ny[+1], Nz[+1]) with the +1 on Bounded axes; halos are filled as fill_halo_vel!
 * (src/Biogeochemistry/HaloRegions/halo_regions.jl:64-99). */
pi_status pi_set_velocity(pi_model* m, const double* u, const double* v, const double* w);

/* vel₀ of the timestepper (the previous step's velocity, time_step.jl:174-176), same layout as
 * pi_set_velocity. Only needed to restart from a checkpoint in a fresh handle. */
pi_status pi_set_velocity0(pi_model* m, const double* u, const double* v, const double* w);

/* copyto!(timestepper.PARF, PARF) (src/Simulation/update.jl:23): surface PAR, Nx*Ny. */
pi_status pi_set_PARF(pi_model* m, const double* parf);

/* copy_interior!(timestepper.temp, temp) (src/Simulation/update.jl:26): Nx*Ny*Nz. */
pi_status pi_set_temp(pi_model* m, const double* temp);

/* set_bc!(model; tracer, pos, bc_value) (HaloRegions/boundary_conditions.jl:21-31): flux
 * boundary condition of one tracer face. kind PI_BC_CONST reads values[0]; PI_BC_ARRAY2D reads
 * the face's (n1, n2) array; PI_BC_ARRAY3D reads (n1, n2, nt), indexed by model.iteration. */
pi_status pi_set_flux_bc(pi_model* m, int32_t tracer, int32_t face, int32_t kind,
                         const double* values, int64_t nt);

/* Abiotic particles (src/Individuals/Abiotic/): the parameters of construct_abiotic_particle
 * (particle_generation.jl:1-22) in its param_names order; defaults in abiotic_params_default
 * (src/Parameters/param_default.jl:329-343). */
typedef struct {
    double Nsuper, Rd, release_P, sz_min, Ktr;
} pi_abiotic_params;

/* The state of one abiotic species (particle_generation.jl:2-5), `capacity` long: positions in
 * grid-spacing units, the halo-inclusive cell indices of the last find_inds! and the activity
 * flag. pi_set_abiotic_particles requires x, y, z and ac; NULL xi, yi, zi are taken as find_inds!
 * of the positions (the state initialize_abiotic_particle! leaves, particle_generation.jl:24-35).
 * For pi_get_abiotic_particles NULL members are skipped. */
typedef struct {
    double  *x, *y, *z;
    int64_t *xi, *yi, *zi;
    uint8_t *ac;
} pi_abiotic_particles;

/* PlanktonModel(...; abiotic = abiotic_setup(params, N, Nsa, Palat(intac, release)),
 * max_candidates) (src/Model/models.jl:99-146) for a PI_FP64 model (PI_FP32 is refused with
 * PI_ERR_ARG): `nsa` abiotic species, all inactive until pi_set_abiotic_particles. Palat's pairs
 * are 0-based (phytoplankton species, abiotic species) index pairs, 2·n_intac and 2·n_release
 * int32 values, applied in the order given: intac by particle_interaction! and release by
 * particle_release! (time_step.jl:121-137). max_ptc[sp] is phytoplankton species sp's max_ptc
 * parameter, NaN for a mode whose parameters have none (QuotaMode, CarbonMode and
 * MacroMolecularMode): there the reference's merge kernel fails on the field access, and here
 * the step that would merge a particle into such a species returns PI_ERR_PARAM. Called once,
 * before the first step. */
pi_status pi_set_abiotics(pi_model* m, int32_t nsa, const pi_abiotic_params* params,
                          int32_t n_intac, const int32_t* intac, int32_t n_release, const int32_t* release,
                          int32_t max_candidates, const double* max_ptc);
pi_status pi_set_abiotic_particles(pi_model* m, int32_t sa, const pi_abiotic_particles* in);
pi_status pi_get_abiotic_particles(pi_model* m, int32_t sa, pi_abiotic_particles* out);
/* Active abiotic particles of species sa (calc_active_individuals, models.jl:157-164). */
pi_status pi_count_abiotic(pi_model* m, int32_t sa, int64_t* n);

/* set_bc_particle!(model; sa, pos, bc_value) (HaloRegions/boundary_conditions.jl:33-41): the flux
 * of particles through one face of abiotic species sa that particles_from_bcs! turns into new
 * particles (Abiotic/particle_interaction.jl:138-239), with pi_set_flux_bc's kinds and layout. */
pi_status pi_set_abiotic_bc(pi_model* m, int32_t sa, int32_t face, int32_t kind,
                            const double* values, int64_t nt);

/* TimeStep!(model, ΔT, diags) (src/Model/time_step.jl:12-180), QuotaMode physiology. Advances
 * model.iteration by one and model.t to iteration·ΔT. Returns PI_ERR_CAPACITY with the
 * reference's message when divisions exceed the free slots. */
pi_status pi_time_step(pi_model* m, double dT);

/* The same entry points for a PI_FP32 model fed from Float32 host arrays (the reference's forcing
 * arrays when FT = Float32, its default); same shapes as the Float64 versions. Like those, each
 * call has copied the host arrays when it returns; the copies run on a stream of their own and
 * overlap the steps already queued, and the conversion into the model's fields is queued behind
 * them. PI_ERR_ARG for a PI_FP64 model. */
pi_status pi_set_velocity_f32(pi_model* m, const float* u, const float* v, const float* w);
pi_status pi_set_PARF_f32(pi_model* m, const float* parf);
pi_status pi_set_temp_f32(pi_model* m, const float* temp);

/* TimeStep! queued on the model's stream without waiting for it (the reference's GPU kernels are
 * asynchronous too): the call returns once the step is queued; pi_synchronize waits and reports a
 * capacity overflow or out-of-domain index raised by the queued steps. */
pi_status pi_time_step_async(pi_model* m, double dT);

/* pi_count_active queued on the model's stream: *n is written when the stream reaches the count
 * (after the steps queued before it). *n should be page-locked host memory (cudaHostAlloc) for the
 * call not to wait for the stream. */
pi_status pi_count_active_async(pi_model* m, int32_t sp, int64_t* n);

/* model.iteration and model.t. */
pi_status pi_get_time(pi_model* m, int64_t* iteration, double* t);
pi_status pi_set_time(pi_model* m, int64_t iteration, double t);

/* Number of active individuals of species `sp` (calc_active_individuals, models.jl:157-164). */
pi_status pi_count_active(pi_model* m, int32_t sp, int64_t* n);

/* NaN/Inf check of the model state: every tracer value (halos included) and every attribute of
 * the active individuals. Returns PI_ERR_NAN with a message naming the first tracer cell or
 * individual (1-based, as in the reference) that holds one. No counterpart in the reference, where
 * a user would test the arrays with any(isnan, ...). */
pi_status pi_check_finite(pi_model* m);

/* Diagnostics accumulated by TimeStep! since the last reset: PI_DIAG_PAR (sp ignored) or the
 * per-species PI_DIAG_NUM/GRAZ/MORT/DVID fields, (Nx+2Hx)(Ny+2Hy)(Nz+2Hz) each. */
pi_status pi_get_diag(pi_model* m, int32_t kind, int32_t sp, double* out);
pi_status pi_reset_diags(pi_model* m);

/* PlanktonDiagnostics(model; tracer = (...), phytoplankton = (...)) beyond the defaults: bit n of
 * tracer_mask adds diags.tracer for tracer n, bit q of proc_mask adds process q of every species
 * (PI_PROC_*), read with pi_get_diag(PI_DIAG_TRACER + n / PI_DIAG_PROC + q). Each added field is
 * the sum over steps of the tracer field (halos included) after the tracer update, or of
 * proc·ac at every individual's find_inds! cell after the species' update, as TimeStep! adds
 * them. Enabling (again) starts the added fields at zero; pi_reset_diags clears them too. */
pi_status pi_set_diags(pi_model* m, uint32_t tracer_mask, uint32_t proc_mask);

/* PlanktonSimulation(model; ΔT, iterations, PARF, temp, vels, ΔT_vel, ΔT_PAR, ΔT_temp)
 * (src/Simulation/simulations.jl:98-142) with the shape and time-step validation of
 * src/Simulation/utils.jl:213-304. The forcing series are copied to device memory once:
 * u, v, w are (Nx[+1], Ny[+1], Nz[+1], nvel) (NULL when no velocities are given), PARF is
 * (Nx, Ny, npar), temp is (Nx, Ny, Nz, ntemp). */
pi_status pi_sim_create(pi_model* m, double dT, int64_t iterations,
                        const double* u, const double* v, const double* w, int64_t nvel,
                        double dT_vel,
                        const double* parf, int64_t npar, double dT_PAR,
                        const double* temp, int64_t ntemp, double dT_temp,
                        pi_sim** out);

/* update!(sim; time_offset) (src/Simulation/update.jl:11-48): `iterations` steps, each binding
 * that step's forcing snapshot and calling TimeStep!. Bits 0/1/2 of time_offset select the
 * vels/PARF/temp time offsets. Runs asynchronously on the model's stream unless `sync`. */
pi_status pi_sim_update(pi_sim* s, int32_t time_offset, int32_t sync);

/* Steps first .. first+n-1 (1-based, update!'s loop index i, which the time_offset indexing
 * uses) of update!(sim; time_offset): an update! split into parts, for example to write outputs
 * after every step (write_output!, src/Simulation/update.jl:30). */
pi_status pi_sim_update_steps(pi_sim* s, int64_t first, int64_t n, int32_t time_offset, int32_t sync);

pi_status pi_sim_destroy(pi_sim* s);

/* Blocks until all work queued on the model's stream is done and reports any device-side error
 * (capacity overflow, index out of domain) raised since the last call. */
pi_status pi_synchronize(pi_model* m);

/* The CUDA stream (cudaStream_t) the handle launches on, for callers that record events or order
 * their own work against the model's. */
pi_status pi_get_stream(pi_model* m, void** stream);

/* Per-kernel device timing. While enabled, every kernel launch of a step is bracketed by CUDA
 * events on the model's stream; pi_profile_read synchronises and returns, for up to `max`
 * kernels, the name (NUL-separated in `names`, `names_len` bytes), the number of launches and
 * the summed milliseconds since profiling was enabled. `*n` receives the number of kernels. */
pi_status pi_profile_enable(pi_model* m, int32_t on);
pi_status pi_profile_read(pi_model* m, int32_t max, char* names, size_t names_len,
                          int64_t* launches, double* ms, int32_t* n);

/* DST3FL advection tendency of one tracer field, computed without allocating any device memory.
 * No counterpart in the reference: it serves callers that cannot allocate device memory (a host
 * runtime that owns all device allocations through its own pool, or a loop that must not allocate
 * after start-up). `c`, `u`, `v`, `w` and `Gc` are caller-owned DEVICE pointers to halo-padded
 * fields in the layout of pi_set_tracer, with halos already filled; the grid's dzF, dzC and
 * landmask are host pointers as in pi_create. The call copies dzF, dzC and landmask into device
 * memory on `stream` (a cudaStream_t, NULL for the default stream) and waits for that copy, and
 * so for the work queued on the stream before it, before it returns: the host arrays may be
 * freed or changed once it has returned. The three sweeps are then queued on `stream`; when they
 * have run, Gc's interior holds tracer_temp − tracer after the x, y and z sweeps of
 * tracer_advection! (multi_dim_adv.jl:111-135); Gc's halo is not written.
 * The sweeps' intermediates live in one fixed device array shared by all calls on a device:
 * grids above 524,288 halo-padded cells or 4,096 levels are rejected with PI_ERR_ARG; calls that
 * overlap on the GPU race on that array; the first call on a device looks up its address and
 * should come before any stream capture; the address is kept for the life of the process, so the
 * call must not be used on a device after cudaDeviceReset. pi_noalloc_last_error gives the
 * message of the last call (empty after a call that succeeded). */
pi_status pi_tracer_advection_noalloc(const pi_grid* grid, const double* c, const double* u,
                                      const double* v, const double* w, double dT, double* Gc,
                                      void* stream);
pi_status pi_noalloc_last_error(char* buf, size_t len);

/* Message of the last error of the handle (or of the last failed pi_create when m is NULL). */
pi_status pi_last_error(pi_model* m, char* buf, size_t len);

/* Static description of a status code. */
const char* pi_status_string(pi_status code);

/* Self-test of the bounded device-side waits (no counterpart in the reference): a kernel waits on
 * an mbarrier that nothing arrives on, with the same helper the tracer kernel's staging waits use,
 * and gives up after limit_ns (at most 2 s). *gave_up = 1 and *waited_ns >= limit_ns show that a
 * wait that cannot complete ends with an error status and leaves the context usable. */
pi_status pi_selftest_bounded_wait(int64_t limit_ns, int32_t* gave_up, int64_t* waited_ns);

/* ---------------------------------------------------------------------------------------------
 * Batched FP32 form. A batch holds independent members, each a PlanktonModel of its own (grid,
 * parameters, capacity, individuals, tracers, forcing, seed), that are advanced together: every
 * phase of TimeStep! is one launch over all members, and the step is replayed from a CUDA graph.
 * The reference runs such ensembles as separate models one after another (no batch API); each
 * member here computes what pi_create(..., PI_FP32, ...) followed by the same calls computes for
 * it alone, bit for bit. All members share nspecies and the time step ΔT.
 * --------------------------------------------------------------------------------------------- */
typedef struct pi_batch pi_batch;

typedef struct {
    const pi_grid* grid;
    const pi_bgc_params* bgc;
    const pi_quota_params* species;   /* nspecies entries */
    int64_t capacity;                 /* max_individuals per species */
    uint64_t seed;                    /* key of the member's random draws */
} pi_member;

/* PlanktonModel(...) for every member (src/Model/models.jl:51-155), FP32 form. */
pi_status pi_batch_create(const pi_member* members, int32_t nmembers, int32_t nspecies, pi_batch** out);
pi_status pi_batch_destroy(pi_batch* b);

/* As pi_set_individuals / pi_get_individuals for one member. */
pi_status pi_batch_set_individuals(pi_batch* b, int32_t member, int32_t sp, const pi_individuals* in);
pi_status pi_batch_get_individuals(pi_batch* b, int32_t member, int32_t sp, pi_individuals* out);
/* As pi_set_tracer / pi_get_tracer for one member (halo-padded, Float64 at the boundary). */
pi_status pi_batch_set_tracer(pi_batch* b, int32_t member, int32_t idx, const double* data);
pi_status pi_batch_get_tracer(pi_batch* b, int32_t member, int32_t idx, double* out);
/* As pi_set_velocity / pi_set_velocity0 / pi_set_PARF / pi_set_temp / pi_set_flux_bc, and the
 * Float32-input setters. */
pi_status pi_batch_set_velocity_f32(pi_batch* b, int32_t member, const float* u, const float* v, const float* w);
pi_status pi_batch_set_PARF_f32(pi_batch* b, int32_t member, const float* parf);
pi_status pi_batch_set_temp_f32(pi_batch* b, int32_t member, const float* temp);
pi_status pi_batch_set_velocity(pi_batch* b, int32_t member, const double* u, const double* v, const double* w);
pi_status pi_batch_set_velocity0(pi_batch* b, int32_t member, const double* u, const double* v, const double* w);
pi_status pi_batch_set_PARF(pi_batch* b, int32_t member, const double* parf);
pi_status pi_batch_set_temp(pi_batch* b, int32_t member, const double* temp);
pi_status pi_batch_set_flux_bc(pi_batch* b, int32_t member, int32_t tracer, int32_t face, int32_t kind,
                               const double* values, int64_t nt);

/* PlanktonSimulation's forcing arrays for one member (src/Model/simulations.jl:51-97), kept on the
 * device: u, v, w snapshots (nvel; NULL for none), PARF (npar snapshots of Nx*Ny) and temperature
 * (ntemp snapshots of Nx*Ny*Nz), each with its own interval. Every following step picks its
 * snapshots as update! does (src/Simulation/update.jl:14-26) from model.t, or from the step index
 * within the pi_batch_step call for the bits of `time_offset` set (1 vel, 2 PAR, 4 temp). */
pi_status pi_batch_set_series(pi_batch* b, int32_t member,
                              const double* u, const double* v, const double* w, int64_t nvel, double dT_vel,
                              const double* parf, int64_t npar, double dT_PAR,
                              const double* temp, int64_t ntemp, double dT_temp, int32_t time_offset);
/* update!(sim; time_offset) for the following steps: bits 1 vel, 2 PAR, 4 temp index the series by
 * the step within the pi_batch_step call instead of model.t. */
pi_status pi_batch_set_time_offset(pi_batch* b, int32_t member, int32_t time_offset);
/* Drops a member's series; the snapshots bound for the next step are kept as its own fields. */
pi_status pi_batch_clear_series(pi_batch* b, int32_t member);

/* `nsteps` TimeStep!s of every member (graph replay). With sync = 0 the call returns after
 * queueing; pi_batch_synchronize reports errors. A division overflow in any member stops the
 * whole batch at that step with PI_ERR_CAPACITY and the reference's message. */
pi_status pi_batch_step(pi_batch* b, double dT, int64_t nsteps, int32_t sync);
/* As pi_batch_step, with the step index within the update! call (time_offset indexing) starting
 * at `first` (1-based) instead of 1. */
pi_status pi_batch_step_from(pi_batch* b, double dT, int64_t first, int64_t nsteps, int32_t sync);
pi_status pi_batch_synchronize(pi_batch* b);

/* model.iteration and model.t (shared by all members). */
pi_status pi_batch_get_time(pi_batch* b, int64_t* iteration, double* t);
pi_status pi_batch_set_time(pi_batch* b, int64_t iteration, double t);

/* Active individuals of one member and species (sp = -1: all species; member = -1: all members);
 * the _async form as pi_count_active_async. */
pi_status pi_batch_count_active(pi_batch* b, int32_t member, int32_t sp, int64_t* n);
pi_status pi_batch_count_active_async(pi_batch* b, int32_t member, int32_t sp, int64_t* n);
/* As pi_set_diags, for every member. The FP32 form adds the tracer fields in Float32 (the
 * reference's diagnostics arrays have the model's FT) and the processes as 64-bit fixed-point sums
 * (exact and independent of the order individuals are visited in). */
pi_status pi_batch_set_diags(pi_batch* b, uint32_t tracer_mask, uint32_t proc_mask);
/* As pi_check_finite for one member. */
pi_status pi_batch_check_finite(pi_batch* b, int32_t member);
/* As pi_get_diag / pi_reset_diags. */
pi_status pi_batch_get_diag(pi_batch* b, int32_t member, int32_t kind, int32_t sp, double* out);
pi_status pi_batch_reset_diags(pi_batch* b);

/* FP64 mass budgets of one member (mmol): out[0..2] = Σ volume·tracer over the interior for
 * carbon (DIC+DOC+POC), nitrogen (NH4+NO3+DON+PON) and phosphorus (PO4+DOP+POP); out[3..5] = the
 * active individuals' C (Bm+Cq), N (Bm·R_NC+Nq) and P (Bm·R_PC+Pq). No counterpart in the
 * reference, which has no budget call. */
pi_status pi_batch_budget(pi_batch* b, int32_t member, double out[6]);
/* The same budgets for a model of either precision (a PI_FP32 model is member 0 of its batch). */
pi_status pi_get_budget(pi_model* m, double out[6]);

/* Launch-shape autotuner (no counterpart in the reference): times `steps_per_candidate` real
 * steps of ΔT for each candidate block size, tiles-per-block mode and sweep segment length, and
 * keeps the fastest per kernel. The steps it takes are ordinary steps of the model (results do
 * not depend on launch shapes). `report` (may be NULL) receives one line per choice. */
pi_status pi_batch_autotune(pi_batch* b, double dT, int32_t steps_per_candidate, char* report, size_t report_len);

/* Guard band of the FP32 form's decisions (no counterpart in the reference): a grazing, mortality
 * or division draw within 1e-5 (relative) of its threshold p·ΔT is decided with p recomputed in
 * Float64 from the individual's state. Counts since the batch was created: decisions recomputed
 * and, of those, decisions that the Float32 probability would have taken the other way. */
pi_status pi_batch_guard_stats(pi_batch* b, int64_t* recomputed, int64_t* changed);

/* Tracer update kernels (no counterpart in the reference; pi_batch_autotune chooses): fused = 1
 * runs the single kernel that sweeps x, y and z and finishes the tracer update per column run of
 * `levels` levels (8, 16, 32 or 64), where every member allows it (no tracer diffusion, no flux
 * boundary conditions, at least as many cells as halo points on each axis); fused = 0 runs the x-y
 * kernel, the z kernel and the halo fill. Results are identical either way. */
pi_status pi_batch_set_tracer_kernel(pi_batch* b, int32_t fused, int32_t levels);
/* One launch-shape option (no counterpart in the reference; pi_batch_autotune sets them all):
 * "move_block" 128|256, "move_fit" 2|3|4 (register fit: blocks of 256 per SM),
 * "move_blocks_per_sm" 0|2|4|8 (0: one tile per block), the same three for "physiology_",
 * "xy_rows" 4|8|16|28, "z_levels" 8|16|32|64, "par_warps" 1|2|4|8, "tracer_fused" 0|1,
 * "tracer_fused_levels" 8|16|32|64, "xy_beside_particles" 0|1 (the x-y tracer kernel on a second
 * graph branch beside the particle kernels). Results are identical for every choice. */
pi_status pi_batch_set_option(pi_batch* b, const char* name, int32_t value);
/* Storage order (no counterpart in the reference, which stores individuals in slot order): each
 * (member, species) segment is kept in an order grouped by cell, restored by a counting sort
 * before the first step after pi_batch_set_individuals and then every `steps` steps (default 32;
 * 0 = keep the current order). Setting a positive interval starts a new cycle: the next step
 * sorts first. Slots keep their numbers at the boundary and in every result:
 * draws are keyed by slot number and divisions are assigned in slot order, so the interval changes
 * only the speed, never a result. */
pi_status pi_batch_set_sort_interval(pi_batch* b, int32_t steps);

/* As pi_get_stream / pi_profile_enable / pi_profile_read / pi_last_error. */
pi_status pi_batch_get_stream(pi_batch* b, void** stream);
pi_status pi_batch_profile_enable(pi_batch* b, int32_t on);
pi_status pi_batch_profile_read(pi_batch* b, int32_t max, char* names, size_t names_len,
                                int64_t* launches, double* ms, int32_t* n);
pi_status pi_batch_last_error(pi_batch* b, char* buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* PIB200_H */
