# PIB200 — Julia bindings of libpib200 (the C ABI of include/pib200.h) for PlanktonIndividuals.jl.
#
# Untested here: this image has no Julia. The module mirrors include/pib200.h one to one (struct
# layouts, argument order, status codes); the Python package PlanktonIndividuals in this
# repository binds the same symbols through ctypes and is what the tests exercise.
#
# A GPU architecture of PlanktonIndividuals.jl forwards its model calls here:
#   PlanktonModel(arch, grid; FT, ...)  -> create(grid, bgc, phyt, Nsp, maxN; FT, seed) + set_individuals!/set_tracer!
#   TimeStep!(model, ΔT, diags)         -> time_step!(m, ΔT)
#   PlanktonSimulation(model; ...)      -> simulation(m, ΔT, iterations; PARF, temp, vels, ...)
#   update!(sim; time_offset)           -> update!(s; time_offset)
#   model.individuals / model.tracers / diags -> get_individuals, get_tracer, get_diag
module PIB200

export PiGrid, PiBgc, PiQuota, PiIndividuals, PiMember, PIError
export create, create_carbon, create_macro, create_iron, destroy, set_individuals!, get_individuals, set_tracer!, get_tracer
export set_velocity!, set_PARF!, set_temp!, set_flux_bc!, time_step!, get_time, set_time!
export count_active, get_diag, reset_diags!, check_finite, budget, simulation, update!, synchronize
export set_velocity_f32!, set_PARF_f32!, set_temp_f32!, time_step_async!, count_active_async!, set_diags!
export batch_create, batch_step!, batch_set_sort_interval!
export set_abiotics!, set_abiotic_particles!, get_abiotic_particles, count_abiotic, set_bc_particle!

const lib = get(ENV, "LIBPIB200", joinpath(@__DIR__, "..", "PlanktonIndividuals", "libpib200.so"))

# status codes and constants (include/pib200.h)
const PI_OK = 0
const PI_ERR_CAPACITY = 4
const PI_FP64 = Int32(0)
const PI_FP32 = Int32(1)
const PI_PERIODIC = Int32(0)
const PI_BOUNDED = Int32(1)
const TRACERS = (:DIC, :NH4, :NO3, :PO4, :DFe, :DOC, :DON, :DOP, :PFe_inorg, :POC, :PON, :POP, :PFe_bio, :Dust)
const DIAG_KINDS = Dict(:PAR => Int32(0), :num => Int32(1), :graz => Int32(2), :mort => Int32(3), :dvid => Int32(4),
                        :ptc => Int32(5), :abiotic_num => Int32(6))   # abiotic_num: sp is the abiotic species
# optional diagnostics: PI_DIAG_TRACER + tracer index, PI_DIAG_PROC + process index
const PI_DIAG_TRACER = Int32(16)
const PI_DIAG_PROC = Int32(32)
const PROCS = (:PS, :BS, :VDOC, :VNH4, :VNO3, :VPO4, :resp, :exu, :Bm, :Cq, :Nq, :Pq, :Chl)
const CPROCS = (:PS, :BS, :RP, :RS, :TD, :Bm, :Bd, :Chl)      # CarbonMode processes
# MacroMolecularMode processes (PI_MPROC_* order); VNH4 and exu stay zero as in the reference
const MPROCS = (:PS, :VDOC, :VNH4, :VNO3, :VPO4, :resp, :ρChl, :S_PRO, :S_DNA, :S_RNA, :exu, :CH, :NST, :PST,
                :PRO, :DNA, :RNA, :Chl)
procs(m) = m.mm ? MPROCS : m.carbon ? CPROCS : PROCS

struct PiGrid
    Nx::Int32; Ny::Int32; Nz::Int32
    Hx::Int32; Hy::Int32; Hz::Int32
    topo::NTuple{3,Int32}
    dx::Float64; dy::Float64
    dzF::Ptr{Float64}; dzC::Ptr{Float64}; landmask::Ptr{UInt8}
    metrics::Ptr{Cvoid}          # Ptr{PiGridMetrics} for a LatLonGrid, C_NULL for a RectilinearGrid
end

# pi_grid_metrics: the arrays a LatLonGrid stores (src/Grids/lat_lon_grid.jl:1-45), halos included
struct PiGridMetrics
    dxC::Ptr{Float64}; dyC::Ptr{Float64}; dxF::Ptr{Float64}; dyF::Ptr{Float64}; Az::Ptr{Float64}
    Ax::Ptr{Float64}; Ay::Ptr{Float64}; Vol::Ptr{Float64}
end

# bgc_params_default (src/Parameters/param_default.jl:44-71), field order of pi_bgc_params
const BGC_KEYS = ("kw", "kc", "kDOC", "Nit", "kDON", "kDOP", "kPOC", "kPON", "kPOP", "κh", "κv", "κhP",
                  "κvP", "shared_graz", "w_sink_org", "w_sink_inorg", "lambda_POC", "lambda_min",
                  "kdiss", "lambda_dust", "lambda_Fe", "ligand", "DFeFrac")
struct PiBgc
    v::NTuple{23,Float64}
end
PiBgc(p::AbstractDict) = PiBgc(ntuple(i -> Float64(p[BGC_KEYS[i]]), 23))

# QuotaMode param_names (src/Individuals/Plankton/QuotaMode/plankton_generation.jl:16-20)
const QUOTA_KEYS = ("Nsuper", "Cquota", "mean", "var", "Chl2Cint", "α", "Φ", "Topt", "Tmax", "Ea",
                    "PCmax", "VDOCmax", "VNO3max", "VNH4max", "VPO4max", "KsatDOC", "KsatNH4",
                    "KsatNO3", "KsatPO4", "Cqmax", "Nqmax", "Pqmax", "Chl2N", "R_NC", "R_PC", "k_mtb",
                    "respir", "grz_P", "dvid_type", "dvid_P", "dvid_reg", "dvid_reg2", "mort_P",
                    "mort_reg", "grazFracC", "grazFracN", "grazFracP", "mortFracC", "mortFracN",
                    "mortFracP")
struct PiQuota
    v::NTuple{40,Float64}
end
PiQuota(p::AbstractDict, sp::Integer) = PiQuota(ntuple(i -> Float64(p[QUOTA_KEYS[i]][sp]), 40))

# CarbonMode param_names (src/Individuals/Plankton/CarbonMode/plankton_generation.jl:13-15)
const CARBON_KEYS = ("Nsuper", "Cquota", "mean", "var", "α", "Φ", "Topt", "Tmax", "Ea", "PCmax", "Chl2C",
                     "respir", "f_T2B", "grz_P", "dvid_type", "dvid_P", "dvid_reg", "dvid_reg2", "mort_P",
                     "mort_reg", "grazFracC", "mortFracC", "thermal", "is_bact")
struct PiCarbon
    v::NTuple{24,Float64}
end
PiCarbon(p::AbstractDict, sp::Integer) = PiCarbon(ntuple(i -> Float64(p[CARBON_KEYS[i]][sp]), 24))

# MacroMolecularMode param_names (src/Individuals/Plankton/MacroMolecularMode/plankton_generation.jl:17-23)
const MACRO_KEYS = ("Nsuper", "C_DNA", "var", "PRO2DNA", "RNA2DNA", "CH2DNA", "Chl2DNA", "α", "Φ", "Topt", "Tmax",
                    "Ea", "PCmax", "VDOCmax", "VNO3max", "VNH4max", "VPO4max", "KsatDOC", "KsatNH4", "KsatNO3",
                    "KsatPO4", "CHmax", "NSTmax", "PSTmax", "Chl2N", "R_NC_PRO", "R_NC_DNA", "R_NC_RNA", "R_PC_DNA",
                    "R_PC_RNA", "respir", "k_pro", "k_sat_pro", "k_rna", "k_sat_rna", "k_dna", "k_sat_dna",
                    "dvid_P", "grz_P", "mort_P", "mort_reg", "grazFracC", "grazFracN", "grazFracP", "mortFracC",
                    "mortFracN", "mortFracP")
struct PiMacro
    v::NTuple{47,Float64}
end
PiMacro(p::AbstractDict, sp::Integer) = PiMacro(ntuple(i -> Float64(p[MACRO_KEYS[i]][sp]), 47))

struct PiIndividuals
    x::Ptr{Float64}; y::Ptr{Float64}; z::Ptr{Float64}
    xi::Ptr{Int64}; yi::Ptr{Int64}; zi::Ptr{Int64}
    Sz::Ptr{Float64}; Bm::Ptr{Float64}; Cq::Ptr{Float64}; Nq::Ptr{Float64}; Pq::Ptr{Float64}
    Chl::Ptr{Float64}; gen::Ptr{Float64}; age::Ptr{Float64}
    ac::Ptr{UInt8}
    graz::Ptr{Float64}; mort::Ptr{Float64}; dvid::Ptr{Float64}
    Bd::Ptr{Float64}            # CarbonMode damaged biomass (C_NULL for QuotaMode)
    PRO::Ptr{Float64}; DNA::Ptr{Float64}; RNA::Ptr{Float64}    # MacroMolecularMode pools (C_NULL otherwise)
    CH::Ptr{Float64}; NST::Ptr{Float64}; PST::Ptr{Float64}
    ptc::Ptr{Float64}           # abiotic particles held (every mode); C_NULL uploads zeros
    qNO3::Ptr{Float64}; qNH4::Ptr{Float64}; qP::Ptr{Float64}; qFe::Ptr{Float64}     # IronEnergyMode (C_NULL otherwise)
    qFePS::Ptr{Float64}; qFeNR::Ptr{Float64}; qFeNF::Ptr{Float64}; exEn::Ptr{Float64}; tdark::Ptr{Float64}
end

# construct_abiotic_particle's parameters (Abiotic/particle_generation.jl:7) and one species' state
struct PiAbiotic
    Nsuper::Float64; Rd::Float64; release_P::Float64; sz_min::Float64; Ktr::Float64
end
const ABIOTIC_KEYS = ("Nsuper", "Rd", "release_P", "sz_min", "Ktr")
PiAbiotic(p::AbstractDict, sa::Integer) = PiAbiotic(ntuple(i -> Float64(p[ABIOTIC_KEYS[i]][sa]), 5)...)
struct PiAbioticParticles
    x::Ptr{Float64}; y::Ptr{Float64}; z::Ptr{Float64}
    xi::Ptr{Int64}; yi::Ptr{Int64}; zi::Ptr{Int64}
    ac::Ptr{UInt8}
end

struct PiMember
    grid::Ptr{PiGrid}; bgc::Ptr{PiBgc}; species::Ptr{PiQuota}
    capacity::Int64; seed::UInt64
end

struct PIError <: Exception
    code::Int32
    msg::String
end
Base.showerror(io::IO, e::PIError) = print(io, e.msg)

function lasterror(h::Ptr{Cvoid}, batch::Bool)
    buf = Vector{UInt8}(undef, 1024)
    if batch
        ccall((:pi_batch_last_error, lib), Int32, (Ptr{Cvoid}, Ptr{UInt8}, Csize_t), h, buf, length(buf))
    else
        ccall((:pi_last_error, lib), Int32, (Ptr{Cvoid}, Ptr{UInt8}, Csize_t), h, buf, length(buf))
    end
    unsafe_string(pointer(buf))
end

# Validation errors carry the reference's ArgumentError texts; other failures are a PIError.
function check(st::Integer, h::Ptr{Cvoid}; batch::Bool = false)
    st == PI_OK && return nothing
    msg = lasterror(h, batch)
    st in (1, 2, 3, PI_ERR_CAPACITY) && throw(ArgumentError(msg))
    throw(PIError(Int32(st), msg))
end

# ---- model -------------------------------------------------------------------------------------
mutable struct Model
    h::Ptr{Cvoid}
    G::NTuple{3,Int}
    Nsp::Int
    capacity::Int
    carbon::Bool
    mm::Bool                 # MacroMolecularMode
end

topo_code(T) = occursin("Periodic", string(T)) ? PI_PERIODIC : PI_BOUNDED

function pigrid(g, dzF::Vector{Float64}, dzC::Vector{Float64}, lm::Vector{UInt8}, met::Ptr{Cvoid} = C_NULL)
    PiGrid(g.Nx, g.Ny, g.Nz, g.Hx, g.Hy, g.Hz,
           (topo_code(g.topology[1]), topo_code(g.topology[2]), topo_code(g.topology[3])),
           Float64(g.Δx), Float64(g.Δy), pointer(dzF), pointer(dzC), pointer(lm), met)
end

# The LatLonGrid arrays as Float64 vectors (kept alive by the caller) and their pi_grid_metrics;
# a RectilinearGrid (no dxC field) gives nothing.
function metric_arrays(g)
    hasproperty(g, :dxC) || return (Vector{Float64}[], nothing)
    arrs = [Float64.(vec(collect(getproperty(g, s)))) for s in (:dxC, :dyC, :dxF, :dyF, :Az, :Ax, :Ay, :Vol)]
    (arrs, Ref(PiGridMetrics(map(pointer, arrs)...)))
end

"""PlanktonModel(GPU(), grid; FT, max_individuals, bgc_params, phyto) on the B200: allocates the
model on the current CUDA device (`FT = Float64` → the plain form, `Float32` → the FP32 form)."""
function create(g, bgc::AbstractDict, phyt::AbstractDict, Nsp::Integer, maxN::Integer; FT = Float64, seed::Integer = 0)
    dzF, dzC = Float64.(collect(g.dzF)), Float64.(collect(g.dzC))
    lm = UInt8.(vec(collect(g.landmask)))
    marr, mref = metric_arrays(g)
    pg = Ref(pigrid(g, dzF, dzC, lm, mref === nothing ? C_NULL : Ptr{Cvoid}(Base.unsafe_convert(Ptr{PiGridMetrics}, mref))))
    pb = Ref(PiBgc(bgc))
    ps = [PiQuota(phyt, s) for s in 1:Nsp]
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = GC.@preserve dzF dzC lm marr mref ccall((:pi_create, lib), Int32,
        (Ref{PiGrid}, Ref{PiBgc}, Ptr{PiQuota}, Int32, Int64, Int32, UInt64, Ref{Ptr{Cvoid}}),
        pg, pb, ps, Nsp, maxN, FT === Float32 ? PI_FP32 : PI_FP64, seed, out)
    check(st, C_NULL)
    m = Model(out[], (g.Nx + 2g.Hx, g.Ny + 2g.Hy, g.Nz + 2g.Hz), Nsp, maxN, false, false)
    finalizer(destroy, m)
    m
end

"""PlanktonModel(GPU(), grid; FT = Float64, mode = CarbonMode(), ...): CarbonMode species, built in
the FP64 form only."""
function create_carbon(g, bgc::AbstractDict, phyt::AbstractDict, Nsp::Integer, maxN::Integer; seed::Integer = 0)
    dzF, dzC = Float64.(collect(g.dzF)), Float64.(collect(g.dzC))
    lm = UInt8.(vec(collect(g.landmask)))
    marr, mref = metric_arrays(g)
    pg = Ref(pigrid(g, dzF, dzC, lm, mref === nothing ? C_NULL : Ptr{Cvoid}(Base.unsafe_convert(Ptr{PiGridMetrics}, mref))))
    pb = Ref(PiBgc(bgc))
    ps = [PiCarbon(phyt, s) for s in 1:Nsp]
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = GC.@preserve dzF dzC lm marr mref ccall((:pi_create_carbon, lib), Int32,
        (Ref{PiGrid}, Ref{PiBgc}, Ptr{PiCarbon}, Int32, Int64, Int32, UInt64, Ref{Ptr{Cvoid}}),
        pg, pb, ps, Nsp, maxN, PI_FP64, seed, out)
    check(st, C_NULL)
    m = Model(out[], (g.Nx + 2g.Hx, g.Ny + 2g.Hy, g.Nz + 2g.Hz), Nsp, maxN, true, false)
    finalizer(destroy, m)
    m
end

# IronEnergyMode parameters in param_names order (IronEnergyMode/plankton_generation.jl:27-36)
const IRON_KEYS = ("Nsuper", "Cquota", "SA", "mean", "var", "Chl2Cint", "α", "Topt", "Tmax", "Ea", "is_nr", "is_croc",
    "is_tric", "PCmax", "VNO3max", "VNH4max", "VPO4max", "k_cf", "k_rs", "k_nr", "k_nf", "k_mtb", "e_cf", "e_rs",
    "e_nr", "e_nf", "k_Fe_ST2PS", "k_Fe_PS2ST", "k_Fe_ST2NR", "k_Fe_NR2ST", "k_Fe_ST2NF", "k_Fe_NF2ST", "KfePS",
    "KfeNR", "KfeNF", "KsatNH4", "KsatNO3", "KsatPO4", "KSAFe", "CHmax", "qNH4max", "qNO3max", "qPmax", "qFemax",
    "Chl2N", "R_NC", "R_PC", "NF_clock", "grz_P", "dvid_type", "dvid_P", "dvid_reg", "dvid_reg2", "mort_P",
    "mort_reg", "grazFracC", "grazFracN", "grazFracP", "grazFracFe", "mortFracC", "mortFracN", "mortFracP",
    "mortFracFe", "max_ptc")
struct PiIron
    v::NTuple{64,Float64}
end
PiIron(p::AbstractDict, sp::Integer) = PiIron(ntuple(i -> Float64(p[IRON_KEYS[i]][sp]), 64))

"""PlanktonModel(GPU(), grid; FT = Float64, mode = IronEnergyMode(), ...): IronEnergyMode species, built
in the FP64 form only. Its individual columns (CH, qNO3, qNH4, qP, qFe, qFePS, qFeNR, qFeNF, exEn,
tdark) are the PiIndividuals members of those names."""
function create_iron(g, bgc::AbstractDict, phyt::AbstractDict, Nsp::Integer, maxN::Integer; seed::Integer = 0)
    dzF, dzC = Float64.(collect(g.dzF)), Float64.(collect(g.dzC))
    lm = UInt8.(vec(collect(g.landmask)))
    marr, mref = metric_arrays(g)
    pg = Ref(pigrid(g, dzF, dzC, lm, mref === nothing ? C_NULL : Ptr{Cvoid}(Base.unsafe_convert(Ptr{PiGridMetrics}, mref))))
    pb = Ref(PiBgc(bgc))
    ps = [PiIron(phyt, s) for s in 1:Nsp]
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = GC.@preserve dzF dzC lm marr mref ccall((:pi_create_iron, lib), Int32,
        (Ref{PiGrid}, Ref{PiBgc}, Ptr{PiIron}, Int32, Int64, Int32, UInt64, Ref{Ptr{Cvoid}}),
        pg, pb, ps, Nsp, maxN, PI_FP64, seed, out)
    check(st, C_NULL)
    m = Model(out[], (g.Nx + 2g.Hx, g.Ny + 2g.Hy, g.Nz + 2g.Hz), Nsp, maxN, false, false)
    finalizer(destroy, m)
    m
end

"""PlanktonModel(GPU(), grid; FT = Float64, mode = MacroMolecularMode(), ...): MacroMolecularMode
species (individuals carry PRO, DNA, RNA, CH, NST, PST, Chl), built in the FP64 form only."""
function create_macro(g, bgc::AbstractDict, phyt::AbstractDict, Nsp::Integer, maxN::Integer; seed::Integer = 0)
    dzF, dzC = Float64.(collect(g.dzF)), Float64.(collect(g.dzC))
    lm = UInt8.(vec(collect(g.landmask)))
    marr, mref = metric_arrays(g)
    pg = Ref(pigrid(g, dzF, dzC, lm, mref === nothing ? C_NULL : Ptr{Cvoid}(Base.unsafe_convert(Ptr{PiGridMetrics}, mref))))
    pb = Ref(PiBgc(bgc))
    ps = [PiMacro(phyt, s) for s in 1:Nsp]
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = GC.@preserve dzF dzC lm marr mref ccall((:pi_create_macro, lib), Int32,
        (Ref{PiGrid}, Ref{PiBgc}, Ptr{PiMacro}, Int32, Int64, Int32, UInt64, Ref{Ptr{Cvoid}}),
        pg, pb, ps, Nsp, maxN, PI_FP64, seed, out)
    check(st, C_NULL)
    m = Model(out[], (g.Nx + 2g.Hx, g.Ny + 2g.Hy, g.Nz + 2g.Hz), Nsp, maxN, false, true)
    finalizer(destroy, m)
    m
end

function destroy(m::Model)
    m.h != C_NULL && ccall((:pi_destroy, lib), Int32, (Ptr{Cvoid},), m.h)
    m.h = C_NULL
    nothing
end

"""Upload species `sp` (1-based) from a StructArray-like table with the mode's columns
(QuotaMode: Sz, Bm, Cq, Nq, Pq; CarbonMode: Sz, Bm, Bd; MacroMolecularMode: PRO, DNA, RNA, CH, NST, PST)."""
function set_individuals!(m::Model, sp::Integer, d)
    C = m.capacity
    z() = zeros(Float64, C)
    szbm = m.mm ? (z(), z()) : (Float64.(d.Sz), Float64.(d.Bm))
    quota = (m.carbon || m.mm) ? (z(), z(), z()) : (Float64.(d.Cq), Float64.(d.Nq), Float64.(d.Pq))
    bd = m.carbon ? Float64.(d.Bd) : Float64[]
    pools = m.mm ? map(k -> Float64.(getproperty(d, k)), (:PRO, :DNA, :RNA, :CH, :NST, :PST)) : ()
    cols = (Float64.(d.x), Float64.(d.y), Float64.(d.z), Int64.(d.xi), Int64.(d.yi), Int64.(d.zi),
            szbm..., quota..., Float64.(d.Chl), Float64.(d.gen), Float64.(d.age),
            UInt8.(d.ac), Float64.(d.graz), Float64.(d.mort), Float64.(d.dvid))
    ptc = hasproperty(d, :ptc) ? Float64.(d.ptc) : Float64[]
    GC.@preserve cols bd pools ptc begin
        pp = m.mm ? map(pointer, pools) : ntuple(_ -> Ptr{Float64}(C_NULL), 6)
        pi = Ref(PiIndividuals(map(pointer, cols)..., m.carbon ? pointer(bd) : Ptr{Float64}(C_NULL), pp...,
                               isempty(ptc) ? Ptr{Float64}(C_NULL) : pointer(ptc), ntuple(_ -> Ptr{Float64}(C_NULL), 9)...))
        check(ccall((:pi_set_individuals, lib), Int32, (Ptr{Cvoid}, Int32, Ref{PiIndividuals}), m.h, sp - 1, pi), m.h)
    end
end

"""Download species `sp` (1-based) as a NamedTuple of the QuotaMode columns."""
function get_individuals(m::Model, sp::Integer)
    C = m.capacity
    f = ntuple(_ -> zeros(Float64, C), 3); i = ntuple(_ -> zeros(Int64, C), 3)
    q = ntuple(_ -> zeros(Float64, C), 8); ac = zeros(UInt8, C); dec = ntuple(_ -> zeros(Float64, C), 3)
    bd = zeros(Float64, C)
    pools = ntuple(_ -> zeros(Float64, C), 6)
    ptc = zeros(Float64, C)      # stays zero for a Float32 model, which keeps no abiotic particles
    GC.@preserve f i q ac dec bd pools ptc begin
        pi = Ref(PiIndividuals(pointer(f[1]), pointer(f[2]), pointer(f[3]), pointer(i[1]), pointer(i[2]), pointer(i[3]),
                               map(pointer, q)..., pointer(ac), map(pointer, dec)..., pointer(bd), map(pointer, pools)...,
                               pointer(ptc), ntuple(_ -> Ptr{Float64}(C_NULL), 9)...))
        check(ccall((:pi_get_individuals, lib), Int32, (Ptr{Cvoid}, Int32, Ref{PiIndividuals}), m.h, sp - 1, pi), m.h)
    end
    m.mm && return (x = f[1], y = f[2], z = f[3], xi = i[1], yi = i[2], zi = i[3], PRO = pools[1], DNA = pools[2],
                       RNA = pools[3], CH = pools[4], NST = pools[5], PST = pools[6], Chl = q[6], gen = q[7], age = q[8],
                       ac = ac .== 1, graz = dec[1], mort = dec[2], dvid = dec[3], ptc = ptc)
    m.carbon ? (x = f[1], y = f[2], z = f[3], xi = i[1], yi = i[2], zi = i[3], Sz = q[1], Bm = q[2], Bd = bd,
                Chl = q[6], gen = q[7], age = q[8], ac = ac .== 1, graz = dec[1], mort = dec[2], dvid = dec[3], ptc = ptc) :
               (x = f[1], y = f[2], z = f[3], xi = i[1], yi = i[2], zi = i[3], Sz = q[1], Bm = q[2], Cq = q[3], Nq = q[4],
                Pq = q[5], Chl = q[6], gen = q[7], age = q[8], ac = ac .== 1, graz = dec[1], mort = dec[2], dvid = dec[3],
                ptc = ptc)
end

tracer_index(name::Symbol) = Int32(findfirst(==(name), TRACERS) - 1)

set_tracer!(m::Model, name::Symbol, a::Array{Float64,3}) =
    check(ccall((:pi_set_tracer, lib), Int32, (Ptr{Cvoid}, Int32, Ptr{Float64}), m.h, tracer_index(name), a), m.h)

function get_tracer(m::Model, name::Symbol)
    a = zeros(Float64, m.G)
    check(ccall((:pi_get_tracer, lib), Int32, (Ptr{Cvoid}, Int32, Ptr{Float64}), m.h, tracer_index(name), a), m.h)
    a
end

# vel_copy!(vel₁, u, v, w, grid), copyto!(PARF), copy_interior!(temp) (Simulation/update.jl:18-26)
set_velocity!(m::Model, u, v, w) =
    check(ccall((:pi_set_velocity, lib), Int32, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                m.h, Float64.(u), Float64.(v), Float64.(w)), m.h)
set_PARF!(m::Model, parf) = check(ccall((:pi_set_PARF, lib), Int32, (Ptr{Cvoid}, Ptr{Float64}), m.h, Float64.(parf)), m.h)
set_temp!(m::Model, temp) = check(ccall((:pi_set_temp, lib), Int32, (Ptr{Cvoid}, Ptr{Float64}), m.h, Float64.(temp)), m.h)

# The same uploads from Float32 arrays (the reference's arrays when FT = Float32), for a model
# created with FT = Float32: the copies are queued on the model's copy stream and overlap the step
# queued before them; the arrays may be reused when the call returns.
set_velocity_f32!(m::Model, u::Array{Float32}, v::Array{Float32}, w::Array{Float32}) =
    check(ccall((:pi_set_velocity_f32, lib), Int32, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}), m.h, u, v, w), m.h)
set_PARF_f32!(m::Model, parf::Array{Float32}) =
    check(ccall((:pi_set_PARF_f32, lib), Int32, (Ptr{Cvoid}, Ptr{Float32}), m.h, parf), m.h)
set_temp_f32!(m::Model, temp::Array{Float32}) =
    check(ccall((:pi_set_temp_f32, lib), Int32, (Ptr{Cvoid}, Ptr{Float32}), m.h, temp), m.h)

# set_bc!(model; tracer, pos, bc_value) (HaloRegions/boundary_conditions.jl:21-31)
const FACES = Dict(:west => 0, :east => 1, :south => 2, :north => 3, :bottom => 4, :top => 5)
function set_flux_bc!(m::Model, tracer::Symbol, pos::Symbol, value)
    kind, vals, nt = value isa Number ? (1, [Float64(value)], 0) :
                     ndims(value) == 2 ? (2, vec(Float64.(value)), 0) : (3, vec(Float64.(value)), size(value, 3))
    check(ccall((:pi_set_flux_bc, lib), Int32, (Ptr{Cvoid}, Int32, Int32, Int32, Ptr{Float64}, Int64),
                m.h, tracer_index(tracer), FACES[pos], kind, vals, nt), m.h)
end

# abiotic = abiotic_setup(params, N, Nsa, Palat(intac, release)) and max_candidates of PlanktonModel
# (models.jl:99-146), FP64 models: pairs are (phytoplankton, abiotic) species indices (1-based);
# max_ptc per phytoplankton species, NaN for modes without that parameter (a merge then fails).
function set_abiotics!(m::Model, params::AbstractDict, Nsa::Integer; intac = (), release = (),
                       max_candidates::Integer = 25, max_ptc = fill(NaN, m.Nsp))
    ps = [PiAbiotic(params, a) for a in 1:Nsa]
    ia = Int32[v - 1 for p in intac for v in p]; ra = Int32[v - 1 for p in release for v in p]
    mp = Float64.(collect(max_ptc))
    check(ccall((:pi_set_abiotics, lib), Int32,
                (Ptr{Cvoid}, Int32, Ptr{PiAbiotic}, Int32, Ptr{Int32}, Int32, Ptr{Int32}, Int32, Ptr{Float64}),
                m.h, Nsa, ps, length(intac), ia, length(release), ra, max_candidates, mp), m.h)
end

"""Upload abiotic species `sa` (1-based): x, y, z, ac and optionally xi, yi, zi."""
function set_abiotic_particles!(m::Model, sa::Integer, d)
    cols = (Float64.(d.x), Float64.(d.y), Float64.(d.z))
    cells = hasproperty(d, :xi) ? (Int64.(d.xi), Int64.(d.yi), Int64.(d.zi)) : ()
    ac = UInt8.(d.ac)
    GC.@preserve cols cells ac begin
        cp = isempty(cells) ? ntuple(_ -> Ptr{Int64}(C_NULL), 3) : map(pointer, cells)
        pa = Ref(PiAbioticParticles(map(pointer, cols)..., cp..., pointer(ac)))
        check(ccall((:pi_set_abiotic_particles, lib), Int32, (Ptr{Cvoid}, Int32, Ref{PiAbioticParticles}), m.h, sa - 1, pa), m.h)
    end
end

"""model.individuals.abiotics[sa].data (1-based sa) as a NamedTuple."""
function get_abiotic_particles(m::Model, sa::Integer)
    C = m.capacity
    f = ntuple(_ -> zeros(Float64, C), 3); i = ntuple(_ -> zeros(Int64, C), 3); ac = zeros(UInt8, C)
    GC.@preserve f i ac begin
        pa = Ref(PiAbioticParticles(map(pointer, f)..., map(pointer, i)..., pointer(ac)))
        check(ccall((:pi_get_abiotic_particles, lib), Int32, (Ptr{Cvoid}, Int32, Ref{PiAbioticParticles}), m.h, sa - 1, pa), m.h)
    end
    (x = f[1], y = f[2], z = f[3], xi = i[1], yi = i[2], zi = i[3], ac = ac .== 1)
end

function count_abiotic(m::Model, sa::Integer)
    n = Ref{Int64}(0)
    check(ccall((:pi_count_abiotic, lib), Int32, (Ptr{Cvoid}, Int32, Ref{Int64}), m.h, sa - 1, n), m.h)
    n[]
end

# set_bc_particle!(model; sa, pos, bc_value) (HaloRegions/boundary_conditions.jl:33-41)
function set_bc_particle!(m::Model, sa::Integer, pos::Symbol, value)
    kind, vals, nt = value isa Number ? (1, [Float64(value)], 0) :
                     ndims(value) == 2 ? (2, vec(Float64.(value)), 0) : (3, vec(Float64.(value)), size(value, 3))
    check(ccall((:pi_set_abiotic_bc, lib), Int32, (Ptr{Cvoid}, Int32, Int32, Int32, Ptr{Float64}, Int64),
                m.h, sa - 1, FACES[pos], kind, vals, nt), m.h)
end

# TimeStep!(model, ΔT, diags) (src/Model/time_step.jl:12-180)
time_step!(m::Model, ΔT) = check(ccall((:pi_time_step, lib), Int32, (Ptr{Cvoid}, Float64), m.h, ΔT), m.h)
# queues the step and returns; errors of the step are reported by the next synchronize
time_step_async!(m::Model, ΔT) = check(ccall((:pi_time_step_async, lib), Int32, (Ptr{Cvoid}, Float64), m.h, ΔT), m.h)
# queues the count of species sp into n (which must stay valid until synchronize)
count_active_async!(m::Model, sp::Integer, n::Base.RefValue{Int64}) =
    check(ccall((:pi_count_active_async, lib), Int32, (Ptr{Cvoid}, Int32, Ptr{Int64}), m.h, sp - 1, n), m.h)

function get_time(m::Model)
    it = Ref{Int64}(0); t = Ref{Float64}(0)
    check(ccall((:pi_get_time, lib), Int32, (Ptr{Cvoid}, Ref{Int64}, Ref{Float64}), m.h, it, t), m.h)
    (iteration = it[], t = t[])
end
set_time!(m::Model, it, t) = check(ccall((:pi_set_time, lib), Int32, (Ptr{Cvoid}, Int64, Float64), m.h, it, t), m.h)

function count_active(m::Model, sp::Integer)
    n = Ref{Int64}(0)
    check(ccall((:pi_count_active, lib), Int32, (Ptr{Cvoid}, Int32, Ref{Int64}), m.h, sp - 1, n), m.h)
    n[]
end

"""diags.tracer.PAR / diags.tracer[name] (kind = :PAR or a tracer name) or
diags.phytos[sp].num/graz/mort/dvid/<process>, halo-padded. Tracers and processes must have been
enabled with set_diags!."""
function get_diag(m::Model, kind::Symbol, sp::Integer = 1)
    k = haskey(DIAG_KINDS, kind) ? DIAG_KINDS[kind] :
        kind in TRACERS ? PI_DIAG_TRACER + tracer_index(kind) :
        kind in procs(m) ? PI_DIAG_PROC + Int32(findfirst(==(kind), procs(m)) - 1) :
        throw(ArgumentError("$kind is not one of the diagnostics"))
    a = zeros(Float64, m.G)
    check(ccall((:pi_get_diag, lib), Int32, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}), m.h, k, sp - 1, a), m.h)
    a
end

"""PlanktonDiagnostics(model; tracer = (...), phytoplankton = (...)): adds the named tracer fields
and QuotaMode processes to the diagnostics the step accumulates."""
function set_diags!(m::Model; tracer = (), phytoplankton = ())
    tm = UInt32(0); pm = UInt32(0)
    for n in tracer
        n === :PAR && continue
        tm |= UInt32(1) << tracer_index(n)
    end
    for p in phytoplankton
        p in keys(DIAG_KINDS) && continue
        q = findfirst(==(p), procs(m))
        q === nothing && throw(ArgumentError("$p is not one of the diagnostics"))
        pm |= UInt32(1) << (q - 1)
    end
    check(ccall((:pi_set_diags, lib), Int32, (Ptr{Cvoid}, UInt32, UInt32), m.h, tm, pm), m.h)
end
reset_diags!(m::Model) = check(ccall((:pi_reset_diags, lib), Int32, (Ptr{Cvoid},), m.h), m.h)
check_finite(m::Model) = check(ccall((:pi_check_finite, lib), Int32, (Ptr{Cvoid},), m.h), m.h)

"""Mass budgets (mmol): interior tracer C, N, P, then the active individuals' C, N, P."""
function budget(m::Model)
    out = zeros(Float64, 6)
    check(ccall((:pi_get_budget, lib), Int32, (Ptr{Cvoid}, Ptr{Float64}), m.h, out), m.h)
    return out
end
synchronize(m::Model) = check(ccall((:pi_synchronize, lib), Int32, (Ptr{Cvoid},), m.h), m.h)

# ---- simulation ---------------------------------------------------------------------------------
mutable struct Simulation
    h::Ptr{Cvoid}
    model::Model
end

"""PlanktonSimulation(model; ΔT, iterations, PARF, temp, vels, ΔT_vel, ΔT_PAR, ΔT_temp): the
forcing series are copied to device memory once; vels = (u = …, v = …, w = …) with a 4th
(snapshot) dimension, or nothing."""
function simulation(m::Model, ΔT, iterations; PARF, temp, vels = nothing, ΔT_vel = ΔT, ΔT_PAR = 3600.0, ΔT_temp = 3600.0)
    parf, tp = Float64.(PARF), Float64.(temp)
    has = vels !== nothing
    u, v, w = has ? (Float64.(vels.u), Float64.(vels.v), Float64.(vels.w)) : (Float64[], Float64[], Float64[])
    nvel = has ? size(u, 4) : 0
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = GC.@preserve parf tp u v w ccall((:pi_sim_create, lib), Int32,
        (Ptr{Cvoid}, Float64, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int64, Float64,
         Ptr{Float64}, Int64, Float64, Ptr{Float64}, Int64, Float64, Ref{Ptr{Cvoid}}),
        m.h, ΔT, iterations, has ? pointer(u) : C_NULL, has ? pointer(v) : C_NULL, has ? pointer(w) : C_NULL,
        nvel, ΔT_vel, parf, size(parf, 3), ΔT_PAR, tp, size(tp, 4), ΔT_temp, out)
    check(st, m.h)
    s = Simulation(out[], m)
    finalizer(s) do s
        s.h != C_NULL && ccall((:pi_sim_destroy, lib), Int32, (Ptr{Cvoid},), s.h)
        s.h = C_NULL
    end
    s
end

"""update!(sim; time_offset = (vels = false, PARF = false, temp = false)) (src/Simulation/update.jl:11-48)."""
function update!(s::Simulation; time_offset = (vels = false, PARF = false, temp = false), sync::Bool = true)
    mask = Int32(time_offset.vels) | (Int32(time_offset.PARF) << 1) | (Int32(time_offset.temp) << 2)
    check(ccall((:pi_sim_update, lib), Int32, (Ptr{Cvoid}, Int32, Int32), s.h, mask, sync), s.model.h)
end

# ---- batched FP32 form (ensembles) ----------------------------------------------------------------
"""One batch of independent FP32 models advanced together; `members` are PiMember records whose
pointers the caller keeps alive for the call."""
function batch_create(members::Vector{PiMember}, Nsp::Integer)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = ccall((:pi_batch_create, lib), Int32, (Ptr{PiMember}, Int32, Int32, Ref{Ptr{Cvoid}}), members, length(members), Nsp, out)
    check(st, C_NULL; batch = true)
    out[]
end
batch_step!(b::Ptr{Cvoid}, ΔT, n) =
    check(ccall((:pi_batch_step, lib), Int32, (Ptr{Cvoid}, Float64, Int64, Int32), b, ΔT, n, 1), b; batch = true)
batch_set_sort_interval!(b::Ptr{Cvoid}, n) =
    check(ccall((:pi_batch_set_sort_interval, lib), Int32, (Ptr{Cvoid}, Int32), b, n), b; batch = true)

end # module
