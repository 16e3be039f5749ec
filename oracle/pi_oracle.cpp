/*
 * pi_oracle.cpp — CPU oracle for the model time step of PlanktonIndividuals.jl (QuotaMode,
 * CarbonMode, MacroMolecularMode and IronEnergyMode physiology; abiotic particles).
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product library links or calls this file; it is what
 * the tests, smoke() and the CPU-baseline leg of bench.py compare the CUDA path against.
 *
 * This is a plain Float64 restatement of the reference's TimeStep! written pass by pass in the
 * order of the Julia kernels, each pass citing the file:line it follows (paths relative to the
 * reference repository root). Summation of scatters is in ascending slot order, species in
 * order — the order a single-threaded KernelAbstractions CPU run of the reference takes.
 *
 * Parity status: the reference (Julia 1.12, KernelAbstractions) cannot run in this environment,
 * so step outputs are "parity unpinned" against the reference itself. What pins the restatement:
 * the reference's own known-answer tests for the grid metrics, halo rules and flux boundary
 * condition (test/grid_test.jl:5-67, test/field_test.jl:21-122), the 14-tracer order
 * (test/field_test.jl:8), and its total-P conservation invariant (test/example_2D_test.jl:19-47),
 * all re-run against this code by tests/test_oracle_kats.py. Random draws come from the shared
 * counter-based generator in include/pi_numerics.h instead of the reference's unseeded
 * MersenneTwister (src/Architectures.jl:33); exp and integer powers come from the same header.
 *
 * Out-of-domain indices (which the reference would read out of bounds under @inbounds) are
 * clamped into the halo-padded grid and reported as PI_ERR_DOMAIN, the same rule as the CUDA path.
 *
 * The elementwise passes are OpenMP-parallel; scatters, scans and column sweeps are sequential,
 * so the result does not depend on the thread count.
 */
#include "../include/pib200.h"
#include "../include/pi_numerics.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::vector<double> dvec;

/* Float32 literals of the reference that appear inside Float64 arithmetic. */
const double F_1em30 = (double)1.0e-30f;   /* 1.0f-30  */
const double F_RGAS  = (double)8.3145f;    /* 8.3145f0 */
const double F_T0    = (double)273.15f;    /* 273.15f0 */
const double F_4em2  = (double)4.0e-2f;    /* 4.0f-2   */
const double F_1em4  = (double)1.0e-4f;    /* 1.0f-4   */
const double F_1em2  = (double)1.0e-2f;    /* 1.0f-2   */
const double F_1em1  = (double)1.0e-1f;    /* 1.0f-1   */
const double F_2em3  = (double)2.0e-3f;    /* 2.0f-3   */
const double F_1em3  = (double)1.0e-3f;    /* 1.0f-3   */
const double F_1em5  = (double)1.0e-5f;    /* 1.0f-5   */
const double F_1em6  = (double)1.0e-6f;    /* 1.0f-6   */
const double F_0p99  = (double)0.99f;      /* 0.99f0   */
const double F_THMAX = (double)1.0e20f;    /* θmax = 1.0f20, DST3FL.jl:2 */
const double F_1em20 = (double)1.0e-20f;   /* 1.0f-20  */
const double F_5em2  = (double)0.05f;      /* 0.05f0   */
const double F_CHL   = (double)893.49f;    /* 893.49f0 (mg Chl per mmol, MacroMolecularMode) */

const uint32_t ERR_DOMAIN = 1u, ERR_CAPACITY = 2u;

struct Grid {
    int Nx, Ny, Nz, Hx, Hy, Hz, Gx, Gy, Gz;
    int tx, ty, tz;
    double dx, dy;
    dvec dzF, dzC;               /* 1-based access through f(k) below */
    std::vector<uint8_t> lm;     /* landmask with halos */
    size_t G;
    inline size_t id(long i, long j, long k) const {   /* 1-based Julia indices */
        return (size_t)(i - 1) + (size_t)Gx * ((size_t)(j - 1) + (size_t)Gy * (size_t)(k - 1));
    }
    inline double dzF1(long k) const { return dzF[k - 1]; }
    inline double dzC1(long k) const { return dzC[k - 1]; }
    /* LatLonGrid (lat_lon_grid.jl:1-45): the stored arrays; empty for a RectilinearGrid */
    bool ll = false;
    dvec mdxC, mdyC, mdxF, mdyF, mAz, mAx, mAy, mVol;
    inline size_t id2(long i, long j) const { return (size_t)(i - 1) + (size_t)Gx * (size_t)(j - 1); }
    /* Grids/areas_volumes_spacings.jl:9-38, 1-based halo-inclusive indices */
    inline double dxC(long i, long j) const { return ll ? mdxC[id2(i, j)] : dx; }
    inline double dyC(long i, long j) const { return ll ? mdyC[id2(i, j)] : dy; }
    inline double dxF(long i, long j) const { return ll ? mdxF[id2(i, j)] : dx; }
    inline double dyF(long i, long j) const { return ll ? mdyF[id2(i, j)] : dy; }
    inline double vol(long i, long j, long k) const { return ll ? mVol[id(i, j, k)] : dx * dy * dzF1(k); }  /* Δx*Δy*dzF[k] */
    inline double Axk(long i, long j, long k) const { return ll ? mAx[id(i, j, k)] : dy * dzF1(k); }      /* Δy*dzF[k] */
    inline double Ayk(long i, long j, long k) const { return ll ? mAy[id(i, j, k)] : dx * dzF1(k); }      /* Δx*dzF[k] */
    inline double Az(long i, long j) const { return ll ? mAz[id2(i, j)] : dx * dy; }                      /* Δx*Δy */
    inline int L(long i, long j, long k) const { return lm[id(i, j, k)]; }
};

struct Species {
    pi_quota_params p;
    dvec x, y, z;
    std::vector<int64_t> xi, yi, zi, idx;
    dvec Sz, Bm, Cq, Nq, Pq, Chl, gen, age;
    std::vector<uint8_t> ac;
    dvec PS, VDOC, VNH4, VNO3, VPO4, rChl, resp, BS, exu, graz, mort, dvid;
    /* diagnostics (diags.phytos[sp]): defaults and the optional QuotaMode processes */
    dvec d_num, d_graz, d_mort, d_dvid;
    std::vector<dvec> d_proc;            /* PI_NPROC fields when enabled */
    /* CarbonMode species (CarbonMode/plankton_generation.jl:2-11): damaged biomass and the rates
     * of repair, respiration and thermal damage (PS and BS are shared with QuotaMode) */
    int carbon = 0;
    pi_carbon_params cp{};
    dvec Bd, RP, RS, TD;
    /* MacroMolecularMode species (MacroMolecularMode/plankton_generation.jl:2-15): protein, DNA,
     * RNA, carbohydrate/lipid, N and P reserves, and the synthesis rates */
    int macro = 0;
    pi_macro_params mp{};
    dvec PRO, DNA, RNA, CH, NST, PST, S_PRO, S_DNA, S_RNA;
    /* abiotic particles held (ptc, every mode's plankton_generation.jl) and their diagnostic */
    dvec ptc, d_ptc;
    /* IronEnergyMode species (IronEnergyMode/plankton_generation.jl:2-22; CH and RS are shared with
     * the fields above): N, P and Fe quotas, excess energy, time since sunset, and the rates */
    int iron = 0;
    pi_iron_params ipp{};
    dvec qNO3, qNH4, qP, qFe, qFePS, qFeNR, qFeNF, exEn, tdark;
    dvec CF, ECF, NF, ENF, VFe, PS2ST, ST2PS, NR2ST, ST2NR, NF2ST, ST2NF, ERS, NR, ENR;
};

struct FluxBC { int kind = PI_BC_NONE; dvec v; int64_t nt = 0; };

/* One abiotic species, construct_abiotic_particle (Abiotic/particle_generation.jl:1-22): the
 * positions, the find_inds! cells and the activity flag of `capacity` slots, its parameters, the
 * particle flux boundary conditions (abiotic_particle.bc) and diags.abiotics[sa].num. */
struct Abiotic {
    pi_abiotic_params p{};
    dvec x, y, z;
    std::vector<int64_t> xi, yi, zi;
    std::vector<uint8_t> ac;
    FluxBC bc[6];
    dvec d_num;
};

}  // namespace

struct orc_model {
    Grid g;
    pi_bgc_params bgc;
    int nsp;
    int64_t C;
    uint64_t seed;
    std::vector<Species> sp;
    std::vector<dvec> tr, Gcs, tt, plk;      /* 14 fields each */
    dvec u0, v0, w0, u1, v1, w1, uh, vh, wh; /* vel₀, vel₁, vel½ */
    dvec PARF, temp, flux_sink, par, par0, Chl, pop;
    /* C-length scratch: rnd, velos, trs (timestepper.jl:40-55) */
    dvec rx, ry, rz;
    dvec vx, vy, vz, vu1, vv1, vw1, vu2, vv2, vw2;
    dvec tNH4, tNO3, tPO4, tDOC, tDFe, tpar, tT, tpop, tdpar, tidc;
    std::vector<int64_t> tidc_int;
    dvec d_PAR;
    uint32_t tr_mask = 0, proc_mask = 0;  /* optional diagnostics (PlanktonDiagnostics keywords) */
    std::vector<dvec> d_tr;               /* 14 fields when any tracer is enabled */
    FluxBC bc[PI_NTRACERS][6];
    /* abiotic particles (abiotic_setup): species, Palat pairs (phytoplankton, abiotic), the
     * candidate table intac (max_candidates × capacity, timestepper.jl:52) and max_ptc per
     * phytoplankton species (NaN: the mode has no such parameter) */
    std::vector<Abiotic> ab;
    std::vector<std::pair<int, int>> pal_intac, pal_release;
    int maxc = 25;
    dvec max_ptc;
    std::vector<int64_t> intac;
    int64_t iteration;
    double t;
    uint32_t err_flags;
    std::string err;
};

namespace {

/* Clamp a 1-based index into [lo, hi], recording an out-of-domain access. */
inline long clampi(orc_model* m, long v, long lo, long hi) {
    if (v < lo) { __atomic_or_fetch(&m->err_flags, ERR_DOMAIN, __ATOMIC_RELAXED); return lo; }
    if (v > hi) { __atomic_or_fetch(&m->err_flags, ERR_DOMAIN, __ATOMIC_RELAXED); return hi; }
    return v;
}

/* ---------------------------------------------------------------------------------------- */
/* Halo rules, src/Biogeochemistry/HaloRegions/halo_regions.jl:2-62. Each fill reads its whole */
/* source range before writing, as Julia's broadcast unaliases overlapping views.              */
/* ---------------------------------------------------------------------------------------- */

/* axis 0/1/2 = x/y/z; face 0 = low (west/south/top), 1 = high (east/north/bottom). */
/* mode: 0 tracer rule, 1 velocity rule for the high face (fill_halo_*_vel!), 2 Gc rule for the
 * high face (fill_halo_*_Gc!). */
void fill_face(const Grid& g, dvec& c, int axis, int face, int mode) {
    int N = axis == 0 ? g.Nx : axis == 1 ? g.Ny : g.Nz;
    int H = axis == 0 ? g.Hx : axis == 1 ? g.Hy : g.Hz;
    int topo = axis == 0 ? g.tx : axis == 1 ? g.ty : g.tz;
    int n1 = axis == 0 ? g.Gy : g.Gx;              /* the two other axes, full range */
    int n2 = axis == 2 ? g.Gy : g.Gz;
    auto at = [&](long a, long b1, long b2) -> double& {   /* a along axis, 1-based */
        if (axis == 0) return c[g.id(a, b1, b2)];
        if (axis == 1) return c[g.id(b1, a, b2)];
        return c[g.id(b1, b2, a)];
    };
    std::vector<long> dst, src;
    bool zero = false;
    if (face == 0) {
        for (int h = 1; h <= H; ++h) dst.push_back(h);
        if (topo == PI_PERIODIC) for (int h = 1; h <= H; ++h) src.push_back(N + h);      /* c[1:H] = c[N+1:N+H] */
        else for (int h = 1; h <= H; ++h) src.push_back(H + 1);                          /* c[1:H] = c[H+1]    */
    } else {
        if (mode == 1 && topo == PI_BOUNDED) {
            for (int h = N + H + 2; h <= N + 2 * H; ++h) { dst.push_back(h); src.push_back(N + H + 1); }
        } else if (mode == 2 && topo == PI_BOUNDED) {
            for (int h = N + H + 1; h <= N + 2 * H; ++h) dst.push_back(h);
            zero = true;
        } else if (topo == PI_PERIODIC) {
            for (int h = 1; h <= H; ++h) { dst.push_back(N + H + h); src.push_back(H + h); }  /* c[N+H+1:N+2H] = c[1+H:2H] */
        } else {
            for (int h = 1; h <= H; ++h) { dst.push_back(N + H + h); src.push_back(N + H); }  /* c[N+H+1:N+2H] = c[N+H] */
        }
    }
    std::vector<double> tmp(dst.size());
    for (int b2 = 1; b2 <= n2; ++b2)
        for (int b1 = 1; b1 <= n1; ++b1) {
            if (!zero) for (size_t q = 0; q < dst.size(); ++q) tmp[q] = at(src[q], b1, b2);
            for (size_t q = 0; q < dst.size(); ++q) at(dst[q], b1, b2) = zero ? 0.0 : tmp[q];
        }
}

void fill_halo_tracer(const Grid& g, dvec& c) {          /* halo_regions.jl:37-47 */
    fill_face(g, c, 0, 0, 0); fill_face(g, c, 0, 1, 0);
    fill_face(g, c, 1, 0, 0); fill_face(g, c, 1, 1, 0);
    fill_face(g, c, 2, 0, 0); fill_face(g, c, 2, 1, 0);
}
void fill_halo_Gc(const Grid& g, dvec& c) {              /* halo_regions.jl:49-56 */
    fill_face(g, c, 0, 1, 2); fill_face(g, c, 1, 1, 2); fill_face(g, c, 2, 1, 2);
}
void fill_halo_u(const Grid& g, dvec& c) {               /* halo_regions.jl:64-72 */
    fill_face(g, c, 0, 1, 1); fill_face(g, c, 0, 0, 0);
    fill_face(g, c, 1, 0, 0); fill_face(g, c, 1, 1, 0);
    fill_face(g, c, 2, 0, 0); fill_face(g, c, 2, 1, 0);
}
void fill_halo_v(const Grid& g, dvec& c) {               /* halo_regions.jl:74-82 */
    fill_face(g, c, 1, 1, 1); fill_face(g, c, 0, 0, 0); fill_face(g, c, 0, 1, 0);
    fill_face(g, c, 1, 0, 0); fill_face(g, c, 2, 0, 0); fill_face(g, c, 2, 1, 0);
}
void fill_halo_w(const Grid& g, dvec& c) {               /* halo_regions.jl:84-92 */
    fill_face(g, c, 2, 1, 1); fill_face(g, c, 0, 0, 0); fill_face(g, c, 0, 1, 0);
    fill_face(g, c, 1, 0, 0); fill_face(g, c, 1, 1, 0); fill_face(g, c, 2, 0, 0);
}

/* ---------------------------------------------------------------------------------------- */
/* Particle advection, src/Individuals/Advection/ (all files)                                         */
/* ---------------------------------------------------------------------------------------- */

/* particle_boundary_condition, particle_advection_kernels.jl:2-11 */
inline double bc_pos(double x, double xr, int topo) {
    const double xl = 0.0;
    if (topo == PI_PERIODIC) {
        if (x > xr) return xl + (x - xr);
        if (x < xl) return xr - (xl - x);
        return x;
    }
    if (x > xr) return xr - (x - xr) * 1.0;
    if (x < xl) return xl + (xl - x) * 1.0;
    return x;
}

/* normalized trilinear interpolation, interpolation.jl:12-83. comp 0/1/2 = u/v/w. The face
 * coordinate along the component's own axis uses +1, the others +0.5. */
double itpl(orc_model* m, const dvec& f, int comp, double x, double y, double z, int ac) {
    const Grid& g = m->g;
    double fx = jl_mulb(comp == 0 ? x + 1.0 : x + 0.5, ac);
    double fy = jl_mulb(comp == 1 ? y + 1.0 : y + 0.5, ac);
    double fz = jl_mulb(comp == 2 ? z + 1.0 : z + 0.5, ac);
    double xd = jl_mod1(fx); long xi = (long)jl_trunc(fx);
    double yd = jl_mod1(fy); long yi = (long)jl_trunc(fy);
    double zd = jl_mod1(fz); long zi = (long)jl_trunc(fz);
    long i = clampi(m, xi + g.Hx, 1, g.Gx - 1);
    long j = clampi(m, yi + g.Hy, 1, g.Gy - 1);
    long k = clampi(m, zi + g.Hz, 1, g.Gz - 1);
    double w000 = (1.0 - xd) * (1.0 - yd) * (1.0 - zd);
    double w001 = (1.0 - xd) * (1.0 - yd) * zd;
    double w010 = (1.0 - xd) * yd * (1.0 - zd);
    double w011 = (1.0 - xd) * yd * zd;
    double w100 = xd * (1.0 - yd) * (1.0 - zd);
    double w101 = xd * (1.0 - yd) * zd;
    double w110 = xd * yd * (1.0 - zd);
    double w111 = xd * yd * zd;
    /* each corner is divided by ΔxC, ΔyC or ΔzC at that corner (interpolation.jl:23-50) */
    auto D = [&](long a, long b, long c) -> double {
        return comp == 0 ? g.dxC(i + a, j + b) : comp == 1 ? g.dyC(i + a, j + b) : g.dzC1(k + c);
    };
    return w000 * f[g.id(i, j, k)] / D(0, 0, 0)
         + w001 * f[g.id(i, j, k + 1)] / D(0, 0, 1)
         + w010 * f[g.id(i, j + 1, k)] / D(0, 1, 0)
         + w011 * f[g.id(i, j + 1, k + 1)] / D(0, 1, 1)
         + w100 * f[g.id(i + 1, j, k)] / D(1, 0, 0)
         + w101 * f[g.id(i + 1, j, k + 1)] / D(1, 0, 1)
         + w110 * f[g.id(i + 1, j + 1, k)] / D(1, 1, 0)
         + w111 * f[g.id(i + 1, j + 1, k + 1)] / D(1, 1, 1);
}

/* vel_interpolate_kernel!, particle_advection_kernels.jl:26-31 */
template <class P>
void vel_interpolate(orc_model* m, P& s, const dvec& X, const dvec& Y, const dvec& Z,
                     const dvec& U, const dvec& V, const dvec& W) {
    int64_t C = m->C;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        m->vu1[i] = jl_mulb(itpl(m, U, 0, X[i], Y[i], Z[i], ac), ac);
        m->vv1[i] = jl_mulb(itpl(m, V, 1, X[i], Y[i], Z[i], ac), ac);
        m->vw1[i] = jl_mulb(itpl(m, W, 2, X[i], Y[i], Z[i], ac), ac);
    }
}

/* calc_coord_kernel!, particle_advection_kernels.jl:40-45 */
template <class P>
void calc_coord(orc_model* m, P& s, dvec& oX, dvec& oY, dvec& oZ,
                const dvec& U, const dvec& V, const dvec& W, double dT, double weight) {
    int64_t C = m->C;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        double x = s.x[i], y = s.y[i], z = s.z[i];
        oX[i] = x + jl_mulb(weight * U[i] * dT, ac);
        oY[i] = y + jl_mulb(weight * V[i] * dT, ac);
        oZ[i] = z - jl_mulb(weight * W[i] * dT, ac);
    }
}

/* particle_boundaries_kernel!, particle_advection_kernels.jl:13-17 */
template <class P>
void particle_boundaries(orc_model* m, P& s, dvec& X, dvec& Y, dvec& Z) {
    const Grid& g = m->g;
    int64_t C = m->C;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        X[i] = jl_mulb(bc_pos(X[i], (double)g.Nx, g.tx), ac);
        Y[i] = jl_mulb(bc_pos(Y[i], (double)g.Ny, g.ty), ac);
        Z[i] = jl_mulb(bc_pos(Z[i], (double)g.Nz, g.tz), ac);
    }
}

/* particle_advection!, particle_advection.jl:2-56 (RK4) */
template <class P>
void particle_advection(orc_model* m, P& s, double dT) {
    int64_t C = m->C;
    vel_interpolate(m, s, s.x, s.y, s.z, m->u0, m->v0, m->w0);
    for (int64_t i = 0; i < C; ++i) { m->vu2[i] = m->vu1[i]; m->vv2[i] = m->vv1[i]; m->vw2[i] = m->vw1[i]; }
    calc_coord(m, s, m->vx, m->vy, m->vz, m->vu1, m->vv1, m->vw1, dT, 0.5);
    particle_boundaries(m, s, m->vx, m->vy, m->vz);
    /* stage 2 */
    vel_interpolate(m, s, m->vx, m->vy, m->vz, m->uh, m->vh, m->wh);
    for (int64_t i = 0; i < C; ++i) {
        m->vu2[i] = m->vu2[i] + m->vu1[i] * 2.0; m->vv2[i] = m->vv2[i] + m->vv1[i] * 2.0;
        m->vw2[i] = m->vw2[i] + m->vw1[i] * 2.0;
    }
    calc_coord(m, s, m->vx, m->vy, m->vz, m->vu1, m->vv1, m->vw1, dT, 0.5);
    particle_boundaries(m, s, m->vx, m->vy, m->vz);
    /* stage 3 */
    vel_interpolate(m, s, m->vx, m->vy, m->vz, m->uh, m->vh, m->wh);
    for (int64_t i = 0; i < C; ++i) {
        m->vu2[i] = m->vu2[i] + m->vu1[i] * 2.0; m->vv2[i] = m->vv2[i] + m->vv1[i] * 2.0;
        m->vw2[i] = m->vw2[i] + m->vw1[i] * 2.0;
    }
    calc_coord(m, s, m->vx, m->vy, m->vz, m->vu1, m->vv1, m->vw1, dT, 1.0);
    particle_boundaries(m, s, m->vx, m->vy, m->vz);
    /* stage 4 */
    vel_interpolate(m, s, m->vx, m->vy, m->vz, m->u1, m->v1, m->w1);
    for (int64_t i = 0; i < C; ++i) {
        m->vu2[i] = m->vu2[i] + m->vu1[i]; m->vv2[i] = m->vv2[i] + m->vv1[i];
        m->vw2[i] = m->vw2[i] + m->vw1[i];
    }
    for (int64_t i = 0; i < C; ++i) {
        m->vu2[i] = m->vu2[i] / 6.0; m->vv2[i] = m->vv2[i] / 6.0; m->vw2[i] = m->vw2[i] / 6.0;
    }
    calc_coord(m, s, s.x, s.y, s.z, m->vu2, m->vv2, m->vw2, dT, 1.0);
    particle_boundaries(m, s, s.x, s.y, s.z);
}

/* particle_diffusion!, particle_diffusion.jl:16-33 */
template <class P>
void particle_diffusion(orc_model* m, P& s, int spi, double dT, uint32_t purpose = PI_DRAW_DIFFUSION) {
    const Grid& g = m->g;
    int64_t C = m->C;
    double kx = m->bgc.kappa_hP, ky = m->bgc.kappa_hP, kz = m->bgc.kappa_vP;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i)
        pi_draw3(m->seed, (uint32_t)m->iteration, (uint32_t)spi, purpose, (uint32_t)i,
                 &m->rx[i], &m->ry[i], &m->rz[i]);
    for (int64_t i = 0; i < C; ++i) {
        m->rx[i] = (m->rx[i] - 0.5) * 2.0; m->ry[i] = (m->ry[i] - 0.5) * 2.0; m->rz[i] = (m->rz[i] - 0.5) * 2.0;
    }
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {   /* calc_diffusion_kernel!, :2-8; ΔzC at zi+Hz of the stored zi */
        long kk = clampi(m, (long)s.zi[i] + g.Hz, 1, g.Gz);
        /* ΔxC/ΔyC at (xi+Hx, yi+Hy) of the stored indices; the reference reads past the array
           there when x = Nx exactly, which is held at the last column here */
        long ii = std::min<long>(std::max<long>((long)s.xi[i] + g.Hx, 1), g.Gx);
        long jj = std::min<long>(std::max<long>((long)s.yi[i] + g.Hy, 1), g.Gy);
        m->rx[i] = m->rx[i] * sqrt(kx * dT) / g.dxC(ii, jj);
        m->ry[i] = m->ry[i] * sqrt(ky * dT) / g.dyC(ii, jj);
        m->rz[i] = m->rz[i] * sqrt(kz * dT) / g.dzC1(kk);
    }
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        s.x[i] = s.x[i] + jl_mulb(m->rx[i], ac);
        s.y[i] = s.y[i] + jl_mulb(m->ry[i], ac);
        s.z[i] = s.z[i] + jl_mulb(m->rz[i], ac);
    }
    particle_boundaries(m, s, s.x, s.y, s.z);
}

/* ---------------------------------------------------------------------------------------- */
/* Particle-grid coupling, src/Individuals/utils.jl                                            */
/* ---------------------------------------------------------------------------------------- */

template <class P>
void find_inds(orc_model* m, P& s) {     /* utils.jl:2-7 */
    const Grid& g = m->g;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m->C; ++i) {
        int ac = s.ac[i];
        s.xi[i] = clampi(m, (long)jl_trunc(jl_mulb(s.x[i] + 1.0, ac)) + g.Hx, 1, g.Gx);
        s.yi[i] = clampi(m, (long)jl_trunc(jl_mulb(s.y[i] + 1.0, ac)) + g.Hy, 1, g.Gy);
        s.zi[i] = clampi(m, (long)jl_trunc(jl_mulb(s.z[i] + 1.0, ac)) + g.Hz, 1, g.Gz);
    }
}

template <class P>
inline size_t cell_of(orc_model* m, const P& s, int64_t i) {
    const Grid& g = m->g;
    long a = clampi(m, (long)s.xi[i], 1, g.Gx);
    long b = clampi(m, (long)s.yi[i], 1, g.Gy);
    long c = clampi(m, (long)s.zi[i], 1, g.Gz);
    return g.id(a, b, c);
}

void acc_chl(orc_model* m, Species& s) {       /* utils.jl:33-36 */
    for (int64_t i = 0; i < m->C; ++i) m->Chl[cell_of(m, s, i)] += jl_mulb(s.Chl[i], s.ac[i]);
}
void acc_counts(orc_model* m, Species& s) {    /* utils.jl:44-47 */
    for (int64_t i = 0; i < m->C; ++i) m->pop[cell_of(m, s, i)] += (double)s.ac[i];
}

void calc_par(orc_model* m, int ki) {          /* utils.jl:55-63 */
    const Grid& g = m->g;
    #pragma omp parallel for schedule(static)
    for (int j = 1; j <= g.Ny; ++j)
        for (int i = 1; i <= g.Nx; ++i) {
            long ii = i + g.Hx, jj = j + g.Hy, kk = ki + g.Hz;
            size_t c = g.id(ii, jj, kk);
            size_t f = (size_t)(i - 1) + (size_t)g.Nx * (size_t)(j - 1);
            double atten = (m->Chl[c] / g.vol(ii, jj, kk) * m->bgc.kc + m->bgc.kw) * g.dzF1(kk);
            m->par[c] = m->PARF[f] * (1.0 - pi_exp(-atten)) / atten;
            m->PARF[f] = m->PARF[f] * pi_exp(-atten);
        }
}

void find_NPT(orc_model* m, Species& s) {      /* utils.jl:14-25 */
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m->C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        m->tNH4[i] = jl_mulb(jl_max(0.0, m->tr[PI_NH4][c]), ac);
        m->tNO3[i] = jl_mulb(jl_max(0.0, m->tr[PI_NO3][c]), ac);
        m->tPO4[i] = jl_mulb(jl_max(0.0, m->tr[PI_PO4][c]), ac);
        m->tDOC[i] = jl_mulb(jl_max(0.0, m->tr[PI_DOC][c]), ac);
        m->tDFe[i] = jl_mulb(jl_max(0.0, m->tr[PI_DFe][c]), ac);
        m->tpar[i] = jl_mulb(m->par[c], ac);
        m->tdpar[i] = jl_mulb(m->par[c] - m->par0[c], ac);
        m->tT[i] = jl_mulb(m->temp[c], ac);
        m->tpop[i] = jl_mulb(m->pop[c], ac);
    }
}

/* ---------------------------------------------------------------------------------------- */
/* QuotaMode physiology, src/Individuals/Plankton/QuotaMode/ (all files)                             */
/* ---------------------------------------------------------------------------------------- */

/* shape functions, Individuals/utils.jl:109-121 */
inline double shape_func_dec(double x, double xmax, double k, int pw) {
    double fx = jl_max(0.0, jl_min(1.0, 1.0 - x / xmax));
    return pi_pow_int(fx, pw) / (k + pi_pow_int(fx, pw));
}
inline double shape_func_inc(double x, double xmax, double k, int pw) {
    double fx = jl_max(0.0, jl_min(1.0, 1.0 - x / xmax));
    double reg = pi_pow_int(fx, pw) / (k + pi_pow_int(fx, pw));
    return 1.0 - reg;
}

inline double tempFunc_PS(double T, const pi_quota_params& p) {   /* growth_kernels.jl:2-9 */
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double regT = shape_func_dec(x, xmax, F_4em2, 4);
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * regT;
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
inline double tempFunc(double T, const pi_quota_params& p) {      /* growth_kernels.jl:12-17 */
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0)));
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}

void plankton_growth(orc_model* m, Species& s, int spi, double dT, double t) {
    const pi_quota_params& p = s.p;
    int64_t C = m->C;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        double par = m->tpar[i], T = m->tT[i], pop = m->tpop[i];
        double NH4 = m->tNH4[i], NO3 = m->tNO3[i], PO4 = m->tPO4[i], DOC = m->tDOC[i];
        /* calc_inorganic_uptake_kernel!, growth_kernels.jl:48-56 with calc_PS :20-25 and
         * calc_NP_uptake :28-39 */
        {
            double aI = par * p.alpha * p.Phi;
            double PCm = p.PCmax * tempFunc_PS(T, p);
            double PS = PCm * (1.0 - pi_exp(-aI / jl_max(F_1em30, PCm) * s.Chl[i] / jl_max(F_1em30, s.Bm[i]))) * s.Bm[i];
            s.PS[i] = jl_mulb(PS, ac);
            double Bm = s.Bm[i], Cq = s.Cq[i], Nq = s.Nq[i], Pq = s.Pq[i];
            double Qn = (Nq + Bm * p.R_NC) / jl_max(F_1em30, Bm + Cq);
            double Qp = (Pq + Bm * p.R_PC) / jl_max(F_1em30, Bm + Cq);
            double regQN = shape_func_dec(Qn, p.Nqmax, F_1em4, 4);
            double regQP = shape_func_dec(Qp, p.Pqmax, F_1em4, 4);
            double VNH4 = jl_mulb(p.VNH4max * regQN * NH4 / jl_max(F_1em30, NH4 + p.KsatNH4) * tempFunc(T, p) * Bm, ac);
            double VNO3 = jl_mulb(p.VNO3max * regQN * NO3 / jl_max(F_1em30, NO3 + p.KsatNO3) * tempFunc(T, p) * Bm, ac);
            double VPO4 = jl_mulb(p.VPO4max * regQP * PO4 / jl_max(F_1em30, PO4 + p.KsatPO4) * tempFunc(T, p) * Bm, ac);
            s.VNH4[i] = jl_min(VNH4, NH4 / dT / jl_max(1.0, pop));
            s.VNO3[i] = jl_min(VNO3, NO3 / dT / jl_max(1.0, pop));
            s.VPO4[i] = jl_min(VPO4, PO4 / dT / jl_max(1.0, pop));
        }
        /* update_quotas_1_kernel!, :64-69 */
        s.Cq[i] += s.PS[i] * dT;
        s.Pq[i] += s.VPO4[i] * dT;
        s.Nq[i] += (s.VNH4[i] + s.VNO3[i]) * dT;
        /* calc_organic_uptake_kernel!, :78-84 with calc_DOC_uptake :41-46 */
        {
            double Cq = s.Cq[i], Bm = s.Bm[i];
            double Qc = Cq / jl_max(F_1em30, Bm + Cq);
            double regQ = shape_func_dec(Qc, p.Cqmax, F_1em4, 4);
            double VN = p.VDOCmax * regQ * DOC / jl_max(F_1em30, DOC + p.KsatDOC) * tempFunc(T, p) * Bm;
            double VDOC = jl_mulb(jl_min(VN, DOC / dT / jl_max(1.0, pop)), ac);
            s.VDOC[i] = jl_mulb(VDOC, jl_isless(F_1em2, s.PS[i] / (VDOC + s.PS[i])));
        }
        /* calc_ρChl_kernel!, :92-97 */
        s.rChl[i] = jl_mulb(jl_mulb(s.PS[i] / jl_max(F_1em30, s.Bm[i]) * p.Chl2N /
                                    jl_max(F_1em30, par * p.alpha * p.Phi * s.Chl[i] / s.Bm[i]),
                                    jl_isless(F_1em1, par)), ac);
        /* calc_respir_kernel!, :105-108 */
        s.resp[i] = jl_mulb(p.respir * s.Bm[i] * tempFunc(T, p), ac);
        /* update_quotas_2_kernel!, :117-124 */
        s.Cq[i] = s.Cq[i] + (s.VDOC[i] - s.resp[i]) * dT;
        s.Bm[i] = s.Bm[i] - jl_max(0.0, (0.0 - s.Cq[i]));
        s.Nq[i] = s.Nq[i] + jl_max(0.0, (0.0 - s.Cq[i])) * p.R_NC;
        s.Pq[i] = s.Pq[i] + jl_max(0.0, (0.0 - s.Cq[i])) * p.R_PC;
        s.Cq[i] = s.Cq[i] + jl_max(0.0, (0.0 - s.Cq[i]));
        /* calc_BS_kernel!, :132-138 */
        {
            double mn = jl_min(jl_min(s.Cq[i], s.Nq[i] / p.R_NC), s.Pq[i] / p.R_PC);
            s.BS[i] = jl_mulb(mn * p.k_mtb, ac);
            double mn2 = jl_min(jl_min(s.Cq[i], s.Nq[i] / p.R_NC), s.Pq[i] / p.R_PC);
            s.exu[i] = jl_mulb(jl_max(0.0, s.Cq[i] - mn2) * p.k_mtb, ac);
        }
        /* update_biomass_kernel!, :146-154 */
        s.Bm[i] += dT * s.BS[i];
        s.Cq[i] -= dT * (s.BS[i] + s.exu[i]);
        s.Nq[i] -= dT * s.BS[i] * p.R_NC;
        s.Pq[i] -= dT * s.BS[i] * p.R_PC;
        s.Chl[i] += dT * s.BS[i] * p.R_NC * s.rChl[i];
        s.age[i] += jl_mulb(dT / 3600.0, ac);
        /* update_cellsize_kernel!, :163-166 */
        s.Sz[i] = s.Bm[i] / (p.Cquota * p.Nsuper);
        /* calc_graz_quadratic_kernel!, division_death_probability.jl:49-52 */
        s.graz[i] = jl_mulb(pop * p.grz_P, ac);
        /* calc_mort_kernel!, :60-63 */
        s.mort[i] = jl_mulb(p.mort_P * shape_func_dec(s.Sz[i], p.mort_reg, F_1em5, 4), ac);
        /* calc_dvid_kernel!, :26-30 with calc_division :7-12 */
        {
            double dv;
            int ty = (int)p.dvid_type;
            if (ty == 1) dv = p.dvid_P * shape_func_inc(s.Sz[i], p.dvid_reg, F_2em3, 2);
            else if (ty == 2) dv = p.dvid_P * shape_func_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg, F_1em5, 4);
            else dv = p.dvid_P * shape_func_inc(s.Sz[i], p.dvid_reg, F_1em3, 4)
                      * shape_func_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg2, F_1em5, 4);
            s.dvid[i] = jl_mulb(dv, ac);
        }
    }
    /* get_probability!, division_death_probability.jl:95-107 */
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        double r0, r1, r2;
        pi_draw3(m->seed, (uint32_t)m->iteration, (uint32_t)spi, PI_DRAW_DECISION, (uint32_t)i, &r0, &r1, &r2);
        m->rx[i] = r0; m->ry[i] = r1; m->rz[i] = r2;
    }
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        s.graz[i] = (double)(jl_isless(m->rx[i], s.graz[i] * dT) && ac);
        s.mort[i] = (double)(jl_isless(m->ry[i], s.mort[i] * dT) && ac);
        s.dvid[i] = (double)(jl_isless(m->rz[i], s.dvid[i] * dT) && ac);
    }
}

/* calc_loss_kernel!, QuotaMode/consume_loss.jl:17-26, then inactivate!, utils.jl:103-105 */
void calc_loss(orc_model* m, Species& s, const dvec& loss, double fC, double fN, double fP) {
    const pi_quota_params& p = s.p;
    for (int64_t i = 0; i < m->C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        double Bm = s.Bm[i], Cq = s.Cq[i], Nq = s.Nq[i], Pq = s.Pq[i], l = loss[i];
        m->plk[PI_DOC][c] += jl_mulb((Bm + Cq) * fC, ac) * l;
        m->plk[PI_DON][c] += jl_mulb((Bm * p.R_NC + Nq) * fN, ac) * l;
        m->plk[PI_DOP][c] += jl_mulb((Bm * p.R_PC + Pq) * fP, ac) * l;
        m->plk[PI_POC][c] += jl_mulb((Bm + Cq) * (1.0 - fC), ac) * l;
        m->plk[PI_PON][c] += jl_mulb((Bm * p.R_NC + Nq) * (1.0 - fN), ac) * l;
        m->plk[PI_POP][c] += jl_mulb((Bm * p.R_PC + Pq) * (1.0 - fP), ac) * l;
    }
    for (int64_t i = 0; i < m->C; ++i) s.ac[i] = (uint8_t)(s.ac[i] && jl_isless(loss[i], 1.0));
}

/* diags_proc_kernel!, Diagnostics/diagnostics_kernels.jl:4-7 */
void diags_proc(orc_model* m, Species& s, dvec& d, const dvec* proc) {
    for (int64_t i = 0; i < m->C; ++i) {
        size_t c = cell_of(m, s, i);
        d[c] += proc ? jl_mulb((*proc)[i], s.ac[i]) : (double)(s.ac[i] && s.ac[i]);
    }
}

/* The capacity error of plankton_update! (plankton_update.jl:21): Julia prints the Float64 day
 * with the shortest digits that round-trip. */
std::string capacity_message(double t) {
    char num[64];
    double d = t / 86400.0;
    for (int p = 1; p <= 17; ++p) { snprintf(num, sizeof num, "%.*g", p, d); if (strtod(num, nullptr) == d) break; }
    std::string ns(num);
    if (ns.find('e') != std::string::npos) {
        std::string mant = ns.substr(0, ns.find('e')), ex = ns.substr(ns.find('e') + 1);
        if (mant.find('.') == std::string::npos) mant += ".0";
        ns = mant + "e" + std::to_string(atoi(ex.c_str()));
    } else if (ns.find('.') == std::string::npos) {
        ns += ".0";
    }
    return "number of individual exceeds the capacity at timestep " + ns + " days";
}

bool plankton_update_carbon(orc_model* m, Species& s, int spi, double dT, double t);
bool plankton_update_macro(orc_model* m, Species& s, int spi, double dT, double t);
bool plankton_update_iron(orc_model* m, Species& s, int spi, double dT, double t);

/* plankton_update!, QuotaMode/plankton_update.jl:1-34 */
bool plankton_update(orc_model* m, Species& s, int spi, double dT, double t) {
    if (s.iron) return plankton_update_iron(m, s, spi, dT, t);
    if (s.carbon) return plankton_update_carbon(m, s, spi, dT, t);
    if (s.macro) return plankton_update_macro(m, s, spi, dT, t);
    const pi_quota_params& p = s.p;
    int64_t C = m->C;
    diags_proc(m, s, s.d_graz, &s.graz);
    calc_loss(m, s, s.graz, p.grazFracC, p.grazFracN, p.grazFracP);          /* grazing!   */
    diags_proc(m, s, s.d_mort, &s.mort);
    calc_loss(m, s, s.mort, p.mortFracC, p.mortFracN, p.mortFracP);          /* mortality! */
    for (int64_t i = 0; i < C; ++i) s.dvid[i] = jl_mulb(s.dvid[i], s.ac[i]);
    diags_proc(m, s, s.d_dvid, &s.dvid);
    double dvidnum = 0.0;
    std::vector<int64_t> free_slots;
    for (int64_t i = 0; i < C; ++i) {
        dvidnum += s.dvid[i] * (double)s.ac[i];
        if (!s.ac[i]) free_slots.push_back(i + 1);                          /* 1-based */
    }
    if (dvidnum > (double)free_slots.size()) {
        m->err = capacity_message(t);
        m->err_flags |= ERR_CAPACITY;
        return false;
    }
    /* divide!, QuotaMode/division_death.jl:69-77 */
    double acc = 0.0;
    for (int64_t i = 0; i < C; ++i) { acc += s.dvid[i]; m->tidc[i] = acc; m->tidc_int[i] = (int64_t)acc; }
    for (int64_t i = 0; i < C; ++i)                                           /* get_tind!   */
        if (s.dvid[i] == 1.0) s.idx[i] = free_slots[(size_t)m->tidc_int[i] - 1];
    for (int64_t i = 0; i < C; ++i)                                           /* copy :28-45 */
        if (s.dvid[i] == 1.0 && s.idx[i] != 0) {
            int64_t d = s.idx[i] - 1;
            s.x[d] = s.x[i]; s.y[d] = s.y[i]; s.z[d] = s.z[i];
            s.Sz[d] = s.Sz[i]; s.Bm[d] = s.Bm[i]; s.Cq[d] = s.Cq[i]; s.Nq[d] = s.Nq[i]; s.Pq[d] = s.Pq[i];
            s.Chl[d] = s.Chl[i]; s.gen[d] = s.gen[i]; s.ac[d] = s.ac[i]; s.dvid[d] = s.dvid[i];
        }
    for (int64_t i = 0; i < C; ++i) {                                         /* divide_to_half :53-63 */
        double f = (2.0 - s.dvid[i]) / 2.0;
        s.Sz[i] *= f; s.Bm[i] *= f; s.Cq[i] *= f; s.Nq[i] *= f; s.Pq[i] *= f; s.Chl[i] *= f;
        s.gen[i] += s.dvid[i];
        s.age[i] *= (1.0 - s.dvid[i]);
    }
    for (int64_t i = 0; i < C; ++i) s.idx[i] = 0;
    plankton_growth(m, s, spi, dT, t);
    /* calc_consume_kernel!, consume_loss.jl:2-9 */
    for (int64_t i = 0; i < C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        m->plk[PI_DIC][c] += jl_mulb((s.resp[i] - s.PS[i]) * dT, ac);
        m->plk[PI_DOC][c] += jl_mulb((s.exu[i] - s.VDOC[i]) * dT, ac);
        m->plk[PI_NH4][c] += jl_mulb(-s.VNH4[i] * dT, ac);
        m->plk[PI_NO3][c] += jl_mulb(-s.VNO3[i] * dT, ac);
        m->plk[PI_PO4][c] += jl_mulb(-s.VPO4[i] * dT, ac);
    }
    /* diags_spcs! (Diagnostics/diagnostics_kernels.jl:14-33), QuotaMode processes */
    if (m->proc_mask) {
        const dvec* procs[PI_NPROC] = { &s.PS, &s.BS, &s.VDOC, &s.VNH4, &s.VNO3, &s.VPO4, &s.resp, &s.exu,
                                        &s.Bm, &s.Cq, &s.Nq, &s.Pq, &s.Chl };
        for (int q = 0; q < PI_NPROC; ++q)
            if (m->proc_mask & (1u << q)) diags_proc(m, s, s.d_proc[q], procs[q]);
    }
    diags_proc(m, s, s.d_num, nullptr);
    return true;
}

/* ---------------------------------------------------------------------------------------- */
/* CarbonMode physiology, src/Individuals/Plankton/CarbonMode/ (all files)                   */
/* ---------------------------------------------------------------------------------------- */

inline double c_tempFunc_PS(double T, const pi_carbon_params& p) {   /* CarbonMode/growth_kernels.jl:2-9 */
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double regT = shape_func_dec(x, xmax, F_1em1, 4);
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * regT;
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
inline double c_tempFunc(double T, const pi_carbon_params& p) {      /* :12-17 */
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0)));
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
inline double c_gamma(double Bm, double Bd, const pi_carbon_params& p) {   /* gamma_alloc, :22-26 */
    double g = jl_mulb(Bd / jl_max(F_1em30, Bm), jl_isless(0.0, Bd));
    return jl_mulb(jl_min(1.0, g), p.thermal == 1.0);
}

/* plankton_growth!, CarbonMode/plankton_growth.jl:2-29, with the kernels of growth_kernels.jl */
void plankton_growth_carbon(orc_model* m, Species& s, int spi, double dT, double t) {
    const pi_carbon_params& p = s.cp;
    int64_t C = m->C;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        double par = m->tpar[i], T = m->tT[i], pop = m->tpop[i];
        double Bm = s.Bm[i], Bd = s.Bd[i], Chl = s.Chl[i];
        /* calc_PS! (calc_photosynthesis, :29-36) */
        double aI = par * p.alpha * p.Phi;
        double PCm = p.PCmax * (c_tempFunc(T, p) * p.thermal + c_tempFunc_PS(T, p) * (1.0 - p.thermal));
        double light = 1.0 - pi_exp(-aI / jl_max(F_1em30, PCm) * Chl / jl_max(F_1em30, Bm));
        double PS = PCm * jl_max(0.0, Bm - Bd) * (light * (1.0 - p.is_bact) + p.is_bact);
        s.PS[i] = jl_mulb(PS, ac);
        /* calc_BS!, calc_repair! (:55-64) */
        s.BS[i] = s.PS[i] * (1.0 - c_gamma(Bm, Bd, p));
        s.RP[i] = s.PS[i] * c_gamma(Bm, Bd, p);
        /* calc_thermal_damage! (:69-75) */
        double TD = jl_mulb(jl_mulb(jl_mulb((T - p.Topt) * p.f_T2B * (Bm - Bd), jl_isless(p.Topt, T)),
                                    jl_isless(Bd, Bm)), p.thermal == 1.0);
        s.TD[i] = jl_max(0.0, jl_min(TD, (Bm - Bd) / dT));
        /* calc_respir! (:82-85) */
        s.RS[i] = jl_mulb(p.respir * Bm * c_tempFunc(T, p), ac);
        /* update_quotas! (:92-97) */
        s.Bm[i] += (s.BS[i] - s.RS[i]) * dT;
        s.Bd[i] += (s.TD[i] - s.RP[i]) * dT;
        s.age[i] += jl_mulb(dT / 3600.0, ac);
        /* update_cellsize! (:104-108) */
        s.Sz[i] = s.Bm[i] / (p.Cquota * p.Nsuper);
        s.Chl[i] = s.Bm[i] * p.Chl2C;
        /* calc_graz_quadratic!, calc_dvid!, calc_thermal_mort! or calc_mort!
         * (division_death_probability.jl:26-30, 49-52, 60-77) */
        s.graz[i] = jl_mulb(pop * p.grz_P, ac);
        double dv;
        int ty = (int)p.dvid_type;
        if (ty == 1) dv = p.dvid_P * shape_func_inc(s.Sz[i], p.dvid_reg, F_2em3, 2);
        else if (ty == 2) dv = p.dvid_P * shape_func_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg, F_1em5, 4);
        else dv = p.dvid_P * shape_func_inc(s.Sz[i], p.dvid_reg, F_1em3, 4)
                  * shape_func_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg2, F_1em5, 4);
        s.dvid[i] = jl_mulb(dv, ac);
        if (p.thermal == 1.0)
            s.mort[i] = jl_mulb(p.mort_P * shape_func_inc(s.Bd[i] / jl_max(F_1em30, s.Bm[i]), F_0p99, F_1em6, 4), ac);
        else
            s.mort[i] = jl_mulb(p.mort_P * shape_func_dec(s.Sz[i], p.mort_reg, F_1em5, 4), ac);
    }
    /* get_probability!, division_death_probability.jl:95-107 */
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        double r0, r1, r2;
        pi_draw3(m->seed, (uint32_t)m->iteration, (uint32_t)spi, PI_DRAW_DECISION, (uint32_t)i, &r0, &r1, &r2);
        m->rx[i] = r0; m->ry[i] = r1; m->rz[i] = r2;
    }
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        s.graz[i] = (double)(jl_isless(m->rx[i], s.graz[i] * dT) && ac);
        s.mort[i] = (double)(jl_isless(m->ry[i], s.mort[i] * dT) && ac);
        s.dvid[i] = (double)(jl_isless(m->rz[i], s.dvid[i] * dT) && ac);
    }
}

/* calc_loss_kernel!, CarbonMode/consume_loss.jl:12-16, then inactivate! */
void calc_loss_carbon(orc_model* m, Species& s, const dvec& loss, double fC) {
    for (int64_t i = 0; i < m->C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        double Bm = s.Bm[i], l = loss[i];
        m->plk[PI_DOC][c] += jl_mulb(Bm * fC, ac) * l;
        m->plk[PI_POC][c] += jl_mulb(Bm * (1.0 - fC), ac) * l;
    }
    for (int64_t i = 0; i < m->C; ++i) s.ac[i] = (uint8_t)(s.ac[i] && jl_isless(loss[i], 1.0));
}

std::string capacity_message(double t);

/* plankton_update!, CarbonMode/plankton_update.jl:1-32 */
bool plankton_update_carbon(orc_model* m, Species& s, int spi, double dT, double t) {
    const pi_carbon_params& p = s.cp;
    int64_t C = m->C;
    diags_proc(m, s, s.d_graz, &s.graz);
    calc_loss_carbon(m, s, s.graz, p.grazFracC);                          /* grazing!   */
    diags_proc(m, s, s.d_mort, &s.mort);
    calc_loss_carbon(m, s, s.mort, p.mortFracC);                          /* mortality! */
    for (int64_t i = 0; i < C; ++i) s.dvid[i] = jl_mulb(s.dvid[i], s.ac[i]);
    diags_proc(m, s, s.d_dvid, &s.dvid);
    double dvidnum = 0.0;
    std::vector<int64_t> free_slots;
    for (int64_t i = 0; i < C; ++i) {
        dvidnum += s.dvid[i] * (double)s.ac[i];
        if (!s.ac[i]) free_slots.push_back(i + 1);
    }
    if (dvidnum > (double)free_slots.size()) {
        m->err = capacity_message(t);
        m->err_flags |= ERR_CAPACITY;
        return false;
    }
    /* divide!, CarbonMode/division_death.jl:62-69: copy_daughter_individuals! (:28-45) copies
     * x, y, z, Sz, Bm, Chl, gen, ac and dvid (not Bd, not age); divide_to_half! (:49-57) halves
     * Sz, Bm, Bd and Chl of every divider and daughter */
    double acc = 0.0;
    for (int64_t i = 0; i < C; ++i) { acc += s.dvid[i]; m->tidc[i] = acc; m->tidc_int[i] = (int64_t)acc; }
    for (int64_t i = 0; i < C; ++i)
        if (s.dvid[i] == 1.0) s.idx[i] = free_slots[(size_t)m->tidc_int[i] - 1];
    for (int64_t i = 0; i < C; ++i)
        if (s.dvid[i] == 1.0 && s.idx[i] != 0) {
            int64_t d = s.idx[i] - 1;
            s.x[d] = s.x[i]; s.y[d] = s.y[i]; s.z[d] = s.z[i];
            s.Sz[d] = s.Sz[i]; s.Bm[d] = s.Bm[i]; s.Chl[d] = s.Chl[i]; s.gen[d] = s.gen[i];
            s.ac[d] = s.ac[i]; s.dvid[d] = s.dvid[i];
        }
    for (int64_t i = 0; i < C; ++i) {
        double f = (2.0 - s.dvid[i]) / 2.0;
        s.Sz[i] *= f; s.Bm[i] *= f; s.Bd[i] *= f; s.Chl[i] *= f;
        s.gen[i] += s.dvid[i];
        s.age[i] *= (1.0 - s.dvid[i]);
    }
    for (int64_t i = 0; i < C; ++i) s.idx[i] = 0;
    plankton_growth_carbon(m, s, spi, dT, t);
    /* calc_consume_kernel!, CarbonMode/consume_loss.jl:2-5 */
    for (int64_t i = 0; i < C; ++i) {
        size_t c = cell_of(m, s, i);
        m->plk[PI_DIC][c] += jl_mulb((s.RS[i] - s.PS[i]) * dT, s.ac[i]);
    }
    /* diags_spcs! (Diagnostics/diagnostics_kernels.jl:14-33), CarbonMode processes */
    if (m->proc_mask) {
        const dvec* procs[PI_NCPROC] = { &s.PS, &s.BS, &s.RP, &s.RS, &s.TD, &s.Bm, &s.Bd, &s.Chl };
        for (int q = 0; q < PI_NCPROC; ++q)
            if (m->proc_mask & (1u << q)) diags_proc(m, s, s.d_proc[q], procs[q]);
    }
    diags_proc(m, s, s.d_num, nullptr);
    return true;
}

/* ---------------------------------------------------------------------------------------- */
/* MacroMolecularMode physiology, src/Individuals/Plankton/MacroMolecularMode/ (all files)      */
/* ---------------------------------------------------------------------------------------- */

inline double m_tempFunc_PS(double T, const pi_macro_params& p) {   /* MacroMolecularMode/growth_kernels.jl:2-9 */
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double regT = shape_func_dec(x, xmax, F_4em2, 4);
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * regT;
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
inline double m_tempFunc(double T, const pi_macro_params& p) {      /* :12-17 */
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0)));
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
/* total_C/N/P_biomass, MacroMolecularMode/plankton_generation.jl:82-93 */
inline double m_totC(double PRO, double DNA, double RNA, double CH, double Chl) {
    return PRO + DNA + RNA + CH + Chl / F_CHL * 55.0;
}
inline double m_totN(double PRO, double DNA, double RNA, double NST, double Chl, const pi_macro_params& p) {
    return PRO * p.R_NC_PRO + DNA * p.R_NC_DNA + RNA * p.R_NC_RNA + NST + Chl / F_CHL * 4.0;
}
inline double m_totP(double DNA, double RNA, double PST, const pi_macro_params& p) {
    return DNA * p.R_PC_DNA + RNA * p.R_PC_RNA + PST;
}

/* plankton_growth!, MacroMolecularMode/plankton_growth.jl:2-28, with the kernels of
 * growth_kernels.jl:1-200 and division_death_probability.jl:37-40, 49-52, 84-87. Every slot is
 * updated: the synthesis and exudation terms carry no ac, so the state of an inactive slot keeps
 * changing as in the reference (its temperature, light and nutrients are zero unless it was
 * active when they were gathered). */
void plankton_growth_macro(orc_model* m, Species& s, int spi, double dT) {
    const pi_macro_params& p = s.mp;
    int64_t C = m->C;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        double NH4 = m->tNH4[i], NO3 = m->tNO3[i], PO4 = m->tPO4[i], DOC = m->tDOC[i];
        double par = m->tpar[i], T = m->tT[i], pop = m->tpop[i];
        double PRO = s.PRO[i], DNA = s.DNA[i], RNA = s.RNA[i], CH = s.CH[i], NST = s.NST[i], PST = s.PST[i];
        double Chl = s.Chl[i];
        /* calc_inorganic_uptake_kernel! (:45-54): calc_PS (:20-25), calc_NP_uptake (:28-42) */
        double aI = par * p.alpha * p.Phi;
        double PCm = p.PCmax * m_tempFunc_PS(T, p);
        double PS = PCm * (1.0 - pi_exp(-aI / jl_max(F_1em30, PCm) * Chl / jl_max(F_1em30, PRO))) * PRO;
        PS = jl_mulb(PS, ac);
        double N_tot = m_totN(PRO, DNA, RNA, NST, Chl, p), P_tot = m_totP(DNA, RNA, PST, p);
        double R_NST = NST / jl_max(F_1em30, N_tot), R_PST = PST / jl_max(F_1em30, P_tot);
        double regQN = shape_func_dec(R_NST, p.NSTmax, F_1em4, 4), regQP = shape_func_dec(R_PST, p.PSTmax, F_1em4, 4);
        double VNH4 = jl_mulb(p.VNH4max * regQN * NH4 / jl_max(F_1em30, NH4 + p.KsatNH4) * m_tempFunc(T, p) * PRO, ac);
        double VNO3 = jl_mulb(p.VNO3max * regQN * NO3 / jl_max(F_1em30, NO3 + p.KsatNO3) * m_tempFunc(T, p) * PRO, ac);
        double VPO4 = jl_mulb(p.VPO4max * regQP * PO4 / jl_max(F_1em30, PO4 + p.KsatPO4) * m_tempFunc(T, p) * PRO, ac);
        VNH4 = jl_min(VNH4, NH4 / dT / jl_max(1.0, pop));
        VNO3 = jl_min(VNO3, NO3 / dT / jl_max(1.0, pop));
        VPO4 = jl_min(VPO4, PO4 / dT / jl_max(1.0, pop));
        /* update_quotas_1_kernel! (:63-67) */
        CH += PS * dT; PST += VPO4 * dT; NST += (VNH4 + VNO3) * dT;
        /* calc_organic_uptake_kernel! (:82-90): calc_DOC_uptake (:73-80) */
        double R_CH = CH / jl_max(F_1em30, m_totC(PRO, DNA, RNA, CH, Chl));
        double regQ = shape_func_dec(R_CH, p.CHmax, F_1em4, 4);
        double VN = p.VDOCmax * regQ * DOC / jl_max(F_1em30, DOC + p.KsatDOC) * m_tempFunc(T, p) * PRO;
        double VDOC = jl_mulb(jl_min(VN, DOC / dT / jl_max(1.0, pop)), ac);
        VDOC = jl_mulb(VDOC, jl_isless(F_5em2, PS / (VDOC + PS)));
        /* calc_ρChl_kernel! (:98-103) */
        double rChl = jl_mulb(jl_mulb(PS / jl_max(F_1em30, PRO) / jl_max(F_1em30, par * p.alpha * p.Phi * Chl / jl_max(F_1em30, PRO)),
                                      jl_isless(F_1em1, par)), ac);
        /* calc_respir_kernel! (:111-114) */
        double resp = jl_mulb(p.respir * PRO * m_tempFunc(T, p), ac);
        /* update_quotas_2_kernel! (:124-130) */
        CH = CH + (VDOC - resp) * dT;
        PRO = PRO - jl_max(0.0, 0.0 - CH);
        NST = NST + jl_max(0.0, 0.0 - CH) * p.R_NC_PRO;
        CH = CH + jl_max(0.0, 0.0 - CH);
        /* calc_BS_kernel! (:136-152) */
        double tf = m_tempFunc(T, p);
        double limit_PRO = jl_min(CH / (CH + p.k_sat_pro * p.Nsuper), NST / (NST + p.k_sat_pro * p.Nsuper * p.R_NC_PRO));
        double limit_DNA = jl_min(jl_min(CH / (CH + p.k_sat_dna * p.Nsuper), NST / (NST + p.k_sat_dna * p.Nsuper * p.R_NC_DNA)),
                                  PST / (PST + p.k_sat_dna * p.Nsuper * p.R_PC_DNA));
        double limit_RNA = jl_min(jl_min(CH / (CH + p.k_sat_rna * p.Nsuper), NST / (NST + p.k_sat_rna * p.Nsuper * p.R_NC_RNA)),
                                  PST / (PST + p.k_sat_rna * p.Nsuper * p.R_PC_RNA));
        double S_PRO = p.k_pro * RNA * limit_PRO * tf;
        double S_DNA = jl_mulb(p.k_dna * PRO * limit_DNA * tf, jl_isless(DNA / (p.C_DNA * p.Nsuper), 2.0));
        double S_RNA = p.k_rna * PRO * limit_RNA * tf;
        /* update_biomass_kernel! (:159-171) */
        PRO += dT * S_PRO;
        DNA += dT * S_DNA;
        RNA += dT * S_RNA;
        CH -= dT * (S_PRO + S_DNA + S_RNA + S_PRO * rChl);
        NST -= dT * (S_PRO * p.R_NC_PRO + S_DNA * p.R_NC_DNA + S_RNA * p.R_NC_RNA + S_PRO * rChl * 4.0 / 55.0);
        PST -= dT * (S_DNA * p.R_PC_DNA + S_RNA * p.R_PC_RNA);
        Chl += dT * S_PRO * rChl * F_CHL / 55.0;
        s.age[i] += jl_mulb(dT / 3600.0, ac);
        /* calc_exudation_kernel! (:179-183), update_CH_kernel! (:190-193) */
        double exu = jl_max(0.0, CH - p.CHmax * m_totC(PRO, DNA, RNA, CH, Chl));
        CH -= exu;
        s.PS[i] = PS; s.VNH4[i] = VNH4; s.VNO3[i] = VNO3; s.VPO4[i] = VPO4; s.VDOC[i] = VDOC;
        s.rChl[i] = rChl; s.resp[i] = resp; s.S_PRO[i] = S_PRO; s.S_DNA[i] = S_DNA; s.S_RNA[i] = S_RNA;
        s.exu[i] = exu;
        s.PRO[i] = PRO; s.DNA[i] = DNA; s.RNA[i] = RNA; s.CH[i] = CH; s.NST[i] = NST; s.PST[i] = PST; s.Chl[i] = Chl;
        /* calc_graz_quadratic!, calc_MM_mort!, calc_MM_dvid! (division_death_probability.jl:37-40,
         * 49-52, 84-87) */
        s.graz[i] = jl_mulb(pop * p.grz_P, ac);
        s.mort[i] = jl_mulb(p.mort_P * shape_func_inc(s.age[i], p.mort_reg, F_1em4, 4), ac);
        s.dvid[i] = jl_mulb(p.dvid_P, jl_isless(2.0, DNA / (p.C_DNA * p.Nsuper)));
    }
    /* get_probability!, division_death_probability.jl:95-107 */
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        double r0, r1, r2;
        pi_draw3(m->seed, (uint32_t)m->iteration, (uint32_t)spi, PI_DRAW_DECISION, (uint32_t)i, &r0, &r1, &r2);
        m->rx[i] = r0; m->ry[i] = r1; m->rz[i] = r2;
    }
    for (int64_t i = 0; i < C; ++i) {
        int ac = s.ac[i];
        s.graz[i] = (double)(jl_isless(m->rx[i], s.graz[i] * dT) && ac);
        s.mort[i] = (double)(jl_isless(m->ry[i], s.mort[i] * dT) && ac);
        s.dvid[i] = (double)(jl_isless(m->rz[i], s.dvid[i] * dT) && ac);
    }
}

/* calc_loss_kernel!, MacroMolecularMode/consume_loss.jl:14-24, then inactivate! */
void calc_loss_macro(orc_model* m, Species& s, const dvec& loss, double fC, double fN, double fP) {
    const pi_macro_params& p = s.mp;
    for (int64_t i = 0; i < m->C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        double l = loss[i];
        double tC = m_totC(s.PRO[i], s.DNA[i], s.RNA[i], s.CH[i], s.Chl[i]);
        double tN = m_totN(s.PRO[i], s.DNA[i], s.RNA[i], s.NST[i], s.Chl[i], p);
        double tP = m_totP(s.DNA[i], s.RNA[i], s.PST[i], p);
        m->plk[PI_DOC][c] += jl_mulb(tC * fC, ac) * l;
        m->plk[PI_DON][c] += jl_mulb(tN * fN, ac) * l;
        m->plk[PI_DOP][c] += jl_mulb(tP * fP, ac) * l;
        m->plk[PI_POC][c] += jl_mulb(tC * (1.0 - fC), ac) * l;
        m->plk[PI_PON][c] += jl_mulb(tN * (1.0 - fN), ac) * l;
        m->plk[PI_POP][c] += jl_mulb(tP * (1.0 - fP), ac) * l;
    }
    for (int64_t i = 0; i < m->C; ++i) s.ac[i] = (uint8_t)(s.ac[i] && jl_isless(loss[i], 1.0));
}

/* plankton_update!, MacroMolecularMode/plankton_update.jl:1-33 */
bool plankton_update_macro(orc_model* m, Species& s, int spi, double dT, double t) {
    const pi_macro_params& p = s.mp;
    int64_t C = m->C;
    diags_proc(m, s, s.d_graz, &s.graz);
    calc_loss_macro(m, s, s.graz, p.grazFracC, p.grazFracN, p.grazFracP);   /* grazing!   */
    diags_proc(m, s, s.d_mort, &s.mort);
    calc_loss_macro(m, s, s.mort, p.mortFracC, p.mortFracN, p.mortFracP);   /* mortality! */
    for (int64_t i = 0; i < C; ++i) s.dvid[i] = jl_mulb(s.dvid[i], s.ac[i]);
    diags_proc(m, s, s.d_dvid, &s.dvid);
    double dvidnum = 0.0;
    std::vector<int64_t> free_slots;
    for (int64_t i = 0; i < C; ++i) {
        dvidnum += s.dvid[i] * (double)s.ac[i];
        if (!s.ac[i]) free_slots.push_back(i + 1);
    }
    if (dvidnum > (double)free_slots.size()) {
        m->err = capacity_message(t);
        m->err_flags |= ERR_CAPACITY;
        return false;
    }
    /* divide!, MacroMolecularMode/division_death.jl:70-78: copy_daughter_individuals! (:28-46)
     * copies x, y, z, PRO, DNA, RNA, CH, NST, PST, Chl, gen, ac and dvid (not age);
     * divide_to_half! (:51-62) halves the seven biomass pools of every divider and daughter */
    double acc = 0.0;
    for (int64_t i = 0; i < C; ++i) { acc += s.dvid[i]; m->tidc[i] = acc; m->tidc_int[i] = (int64_t)acc; }
    for (int64_t i = 0; i < C; ++i)
        if (s.dvid[i] == 1.0) s.idx[i] = free_slots[(size_t)m->tidc_int[i] - 1];
    for (int64_t i = 0; i < C; ++i)
        if (s.dvid[i] == 1.0 && s.idx[i] != 0) {
            int64_t d = s.idx[i] - 1;
            s.x[d] = s.x[i]; s.y[d] = s.y[i]; s.z[d] = s.z[i];
            s.PRO[d] = s.PRO[i]; s.DNA[d] = s.DNA[i]; s.RNA[d] = s.RNA[i]; s.CH[d] = s.CH[i];
            s.NST[d] = s.NST[i]; s.PST[d] = s.PST[i]; s.Chl[d] = s.Chl[i]; s.gen[d] = s.gen[i];
            s.ac[d] = s.ac[i]; s.dvid[d] = s.dvid[i];
        }
    for (int64_t i = 0; i < C; ++i) {
        double f = (2.0 - s.dvid[i]) / 2.0;
        s.PRO[i] *= f; s.DNA[i] *= f; s.RNA[i] *= f; s.CH[i] *= f; s.NST[i] *= f; s.PST[i] *= f; s.Chl[i] *= f;
        s.gen[i] += s.dvid[i];
        s.age[i] *= (1.0 - s.dvid[i]);
    }
    for (int64_t i = 0; i < C; ++i) s.idx[i] = 0;
    plankton_growth_macro(m, s, spi, dT);
    /* calc_consume_kernel!, MacroMolecularMode/consume_loss.jl:2-9 */
    for (int64_t i = 0; i < C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        m->plk[PI_DIC][c] += jl_mulb((s.resp[i] - s.PS[i]) * dT, ac);
        m->plk[PI_DOC][c] += jl_mulb((s.exu[i] - s.VDOC[i]) * dT, ac);
        m->plk[PI_NH4][c] += jl_mulb(-s.VNH4[i] * dT, ac);
        m->plk[PI_NO3][c] += jl_mulb(-s.VNO3[i] * dT, ac);
        m->plk[PI_PO4][c] += jl_mulb(-s.VPO4[i] * dT, ac);
    }
    /* diags_spcs! (Diagnostics/diagnostics_kernels.jl:20-21): VNH4 (listed there as :VHN4) and
     * exu are not accumulated */
    if (m->proc_mask) {
        const dvec* procs[PI_NMPROC] = { &s.PS, &s.VDOC, nullptr, &s.VNO3, &s.VPO4, &s.resp, &s.rChl, &s.S_PRO,
                                         &s.S_DNA, &s.S_RNA, nullptr, &s.CH, &s.NST, &s.PST, &s.PRO, &s.DNA,
                                         &s.RNA, &s.Chl };
        for (int q = 0; q < PI_NMPROC; ++q)
            if ((m->proc_mask & (1u << q)) && procs[q]) diags_proc(m, s, s.d_proc[q], procs[q]);
    }
    diags_proc(m, s, s.d_num, nullptr);
    return true;
}

/* ---------------------------------------------------------------------------------------- */
/* Tracer update, src/Biogeochemistry/ (all files)                                                       */
/* ---------------------------------------------------------------------------------------- */

/* Difference operators with landmask, Advection/operaters.jl:1-14 */
/* ---------------------------------------------------------------------------------------- */
/* IronEnergyMode physiology, src/Individuals/Plankton/IronEnergyMode/ (all files)           */
/* ---------------------------------------------------------------------------------------- */

inline double i_tempFunc_CF(double T, const pi_iron_params& p) {   /* growth_kernels.jl:2-9 */
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double regT = shape_func_dec(x, xmax, F_4em2, 4);
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * regT;
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
inline double i_tempFunc(double T, const pi_iron_params& p) {      /* :12-17 */
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0)));
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
/* the Fe quota sum, qFe + qFePS + qFeNF + qFeNR in the reference's order (:46, consume_loss.jl:28) */
inline double i_feq(double qFe, double qFePS, double qFeNR, double qFeNF) { return qFe + qFePS + qFeNF + qFeNR; }

/* plankton_growth! (plankton_growth.jl:2-26), one pass per kernel in the reference's order */
void plankton_growth_iron(orc_model* m, Species& s, int spi, double dT, double t) {
    const pi_iron_params& p = s.ipp;
    const int64_t C = m->C;
    const double nfx = p.is_croc + p.is_tric;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
        const int ac = s.ac[i];
        const double NH4 = m->tNH4[i], NO3 = m->tNO3[i], PO4 = m->tPO4[i], DFe = m->tDFe[i];
        const double par = m->tpar[i], dpar = m->tdpar[i], T = m->tT[i], pop = m->tpop[i];
        const double Bm = s.Bm[i], Sz = s.Sz[i];
        double CH = s.CH[i], qNH4 = s.qNH4[i], qNO3 = s.qNO3[i], qP = s.qP[i], qFe = s.qFe[i];
        const double qFePS = s.qFePS[i], qFeNR = s.qFeNR[i], qFeNF = s.qFeNF[i], Chl = s.Chl[i];
        /* calc_trs_uptake_kernel! (growth_kernels.jl:56-66) with calc_NH4/NO3/P/Fe_uptake (:20-53) */
        double reg = shape_func_dec(qNH4 / jl_max(F_1em30, Bm + CH), p.qNH4max, F_1em4, 2);
        double VNH4 = jl_mulb(p.VNH4max * reg * NH4 / jl_max(F_1em30, NH4 + p.KsatNH4) * i_tempFunc(T, p) * Bm, ac);
        VNH4 = jl_min(VNH4, NH4 / dT / jl_max(1.0, pop)) * p.is_nr;
        reg = shape_func_dec(qNO3 / jl_max(F_1em30, Bm + CH), p.qNO3max, F_1em4, 2);
        double VNO3 = jl_mulb(p.VNO3max * reg * NO3 / jl_max(F_1em30, NO3 + p.KsatNO3) * i_tempFunc(T, p) * Bm, ac);
        VNO3 = jl_min(VNO3, NO3 / dT / jl_max(1.0, pop)) * p.is_nr;
        reg = shape_func_dec((qP + Bm * p.R_PC) / jl_max(F_1em30, Bm + CH), p.qPmax, F_1em4, 2);
        double VPO4 = jl_mulb(p.VPO4max * reg * PO4 / jl_max(F_1em30, PO4 + p.KsatPO4) * i_tempFunc(T, p) * Bm, ac);
        VPO4 = jl_min(VPO4, PO4 / dT / jl_max(1.0, pop));
        reg = shape_func_dec(i_feq(qFe, qFePS, qFeNR, qFeNF) / jl_max(F_1em30, Bm + CH), p.qFemax, F_1em4, 2);
        const double SA = p.SA * pi_pow(Sz, (double)(2.0f / 3.0f));
        double VFe = jl_mulb(p.KSAFe * SA * DFe * reg * p.Nsuper * i_tempFunc(T, p), ac);
        VFe = jl_min(VFe, DFe / dT / jl_max(1.0, pop));
        /* update_state_1_kernel! (:73-79) */
        qP += VPO4 * dT; qNO3 += VNO3 * dT; qNH4 += VNH4 * dT; qFe += VFe * dT;
        /* calc_PS (:87-93) */
        const double aI = par * p.alpha * Chl / jl_max(F_1em30, Bm);
        const double Qfe_ps = qFePS / jl_max(F_1em30, Bm + CH);
        const double PS = p.PCmax * (1.0 - pi_exp(-aI)) * Bm * (Qfe_ps / jl_max(F_1em30, Qfe_ps + p.KfePS));
        /* calc_respir (:106-111) */
        double RS = jl_mulb(CH * p.k_rs * i_tempFunc(T, p), ac);
        RS = jl_min(RS, CH / dT);
        double ERS = jl_mulb(RS * p.e_rs, ac);
        /* calc_CF (:125-131) */
        reg = shape_func_dec(CH / jl_max(F_1em30, Bm + CH), p.CHmax, F_1em4, 2);
        double CF = jl_mulb(p.k_cf * reg * i_tempFunc_CF(T, p) * Bm, ac);
        double ECF = jl_mulb(CF * p.e_cf, ac);
        /* calc_NR (:145-155) */
        reg = shape_func_dec(qNH4 / jl_max(F_1em30, Bm + CH), p.qNH4max, F_1em4, 2);
        const double Qfe_NR = qFeNR / jl_max(F_1em30, Bm + CH);
        double NR = jl_mulb(p.k_nr * reg * qNO3 * (Qfe_NR / jl_max(F_1em30, Qfe_NR + p.KfeNR)) * i_tempFunc(T, p), ac);
        NR = jl_min(NR, qNO3 / dT);
        double ENR = jl_mulb(NR * p.e_nr, ac);
        NR = NR * p.is_nr; ENR = ENR * p.is_nr;
        /* calc_NF (:167-176) */
        const double Qfe_NF = qFeNF / jl_max(F_1em30, Bm + CH);
        double NF = jl_mulb(p.k_nf * reg * (Qfe_NF / jl_max(F_1em30, Qfe_NF + p.KfeNF)) * i_tempFunc(T, p) * Bm, ac);
        double ENF = jl_mulb(NF * p.e_nf, ac);
        NF = NF * nfx; ENF = ENF * nfx;
        /* energy_alloc (:190-197) and energy_allocation_kernel! (:198-206) */
        const double ECFt = jl_min(PS, ECF);
        const double ENFt = jl_min(ENF, PS + ERS - ECFt) * nfx;
        const double ENRt = jl_min(ENR, PS + ERS - ECFt) * p.is_nr;
        const double ERSt = jl_min(ERS, jl_max(0.0, ECFt + ENFt + ENRt - PS));
        const double exEn = jl_max(0.0, PS - ECFt - ENFt - ENRt);
        ERS = ERSt; ECF = ECFt; ENF = ENFt; ENR = ENRt;
        RS = ERS / p.e_rs; CF = ECF / p.e_cf; NF = ENF / p.e_nf; NR = ENR / p.e_nr;
        /* update_state_2_kernel! (:213-219) */
        CH += (CF - RS) * dT;
        qNO3 += -NR * dT;
        qNH4 += NR * dT;
        qNH4 += NF * dT;
        /* calc_ρChl_kernel! (:227-231) and calc_BS_kernel! (:239-243) */
        const double rChl = jl_mulb(jl_mulb(p.Chl2N / jl_max(F_1em30, par * p.alpha * Chl / Bm), jl_isless(F_1em1, par)), ac);
        const double BS = jl_mulb(jl_min(jl_min(CH, qNH4 / p.R_NC), qP / p.R_PC) * p.k_mtb, ac);
        /* iron_alloc (:251-283): Bool·Bool is a Bool, Bool + Bool an Int */
        const int pos_dpar = jl_isless(0.0, dpar), neg_dpar = jl_isless(dpar, 0.0), dark = jl_isequal(0.0, par);
        const int light = jl_isless(0.0, par), early = jl_isless(s.tdark[i], p.NF_clock), late = jl_isless(p.NF_clock, s.tdark[i]);
        double ST2PS = jl_mulb(p.k_Fe_ST2PS * qFe, pos_dpar);
        double PS2ST = p.k_Fe_PS2ST * qFePS * (double)(neg_dpar + dark);
        double ST2NR = jl_mulb(jl_mulb(p.k_Fe_ST2NR * qFe, dark), early) * p.is_nr;
        double NR2ST = p.k_Fe_NR2ST * qFeNR * (double)((dark & late) + light) * p.is_nr;
        const double ST2NF_cr = jl_mulb(jl_mulb(p.k_Fe_ST2NF * qFe, dark), early);
        const double NF2ST_cr = p.k_Fe_NF2ST * qFeNF * (double)((dark & late) + light);
        const double ST2NF_tr = jl_mulb(p.k_Fe_ST2NF * qFe, pos_dpar);
        const double NF2ST_tr = p.k_Fe_NF2ST * qFeNF * (double)(neg_dpar + dark);
        double ST2NF = ST2NF_cr * p.is_croc + ST2NF_tr * p.is_tric;
        double NF2ST = NF2ST_cr * p.is_croc + NF2ST_tr * p.is_tric;
        ST2PS = jl_min(ST2PS, qFe / dT);
        PS2ST = jl_min(PS2ST, qFePS / dT);
        ST2NR = jl_min(ST2NR, qFe / dT - ST2PS);
        NR2ST = jl_min(NR2ST, qFeNR / dT);
        ST2NF = jl_min(ST2NF, qFe / dT - ST2PS);
        NF2ST = jl_min(NF2ST, qFeNF / dT);
        /* update_biomass_kernel! (:296-312), update_cellsize_kernel! (:322-325) */
        const double Bm1 = Bm + dT * BS;
        CH -= dT * BS;
        qNH4 -= dT * BS * p.R_NC;
        qP -= dT * BS * p.R_PC;
        s.Chl[i] = Chl + dT * BS * p.R_NC * rChl;
        s.age[i] = s.age[i] + jl_mulb(dT / 3600.0, ac);
        s.qFe[i] = qFe + dT * (PS2ST - ST2PS + NR2ST - ST2NR + NF2ST - ST2NF);
        s.qFePS[i] = qFePS + dT * (ST2PS - PS2ST);
        s.qFeNR[i] = qFeNR + dT * (ST2NR - NR2ST);
        s.qFeNF[i] = qFeNF + dT * (ST2NF - NF2ST);
        s.Bm[i] = Bm1; s.CH[i] = CH; s.qNH4[i] = qNH4; s.qNO3[i] = qNO3; s.qP[i] = qP;
        s.Sz[i] = Bm1 / (p.Cquota * p.Nsuper);
        /* update_tdark_kernel! (:333-337): 1.0f0 − Bool is a Float32 */
        s.tdark[i] = s.tdark[i] * (1.0 - (double)light) + jl_mulb(dT, dark);
        s.exEn[i] = exEn;
        s.PS[i] = PS; s.CF[i] = CF; s.ECF[i] = ECF; s.RS[i] = RS; s.ERS[i] = ERS; s.NR[i] = NR; s.ENR[i] = ENR;
        s.NF[i] = NF; s.ENF[i] = ENF; s.BS[i] = BS; s.VNH4[i] = VNH4; s.VNO3[i] = VNO3; s.VPO4[i] = VPO4; s.VFe[i] = VFe;
        s.PS2ST[i] = PS2ST; s.ST2PS[i] = ST2PS; s.NR2ST[i] = NR2ST; s.ST2NR[i] = ST2NR; s.NF2ST[i] = NF2ST; s.ST2NF[i] = ST2NF;
        s.rChl[i] = rChl;
        /* calc_graz_quadratic!, calc_mort!, calc_dvid! (division_death_probability.jl:7-68) */
        s.graz[i] = jl_mulb(pop * p.grz_P, ac);
        s.mort[i] = jl_mulb(p.mort_P * shape_func_dec(s.Sz[i], p.mort_reg, F_1em5, 4), ac);
        double dv;
        const int ty = (int)p.dvid_type;
        if (ty == 1) dv = p.dvid_P * shape_func_inc(s.Sz[i], p.dvid_reg, F_2em3, 2);
        else if (ty == 2) dv = p.dvid_P * shape_func_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg, F_1em5, 4);
        else dv = p.dvid_P * shape_func_inc(s.Sz[i], p.dvid_reg, F_1em3, 4)
                  * shape_func_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg2, F_1em5, 4);
        s.dvid[i] = jl_mulb(dv, ac);
    }
    /* get_probability! (division_death_probability.jl:95-107) */
    for (int64_t i = 0; i < C; ++i) {
        double r0, r1, r2;
        pi_draw3(m->seed, (uint32_t)m->iteration, (uint32_t)spi, PI_DRAW_DECISION, (uint32_t)i, &r0, &r1, &r2);
        const int ac = s.ac[i];
        s.graz[i] = (double)(jl_isless(r0, s.graz[i] * dT) && ac);
        s.mort[i] = (double)(jl_isless(r1, s.mort[i] * dT) && ac);
        s.dvid[i] = (double)(jl_isless(r2, s.dvid[i] * dT) && ac);
    }
}

/* calc_loss_kernel! (IronEnergyMode/consume_loss.jl:17-32), then inactivate! */
void calc_loss_iron(orc_model* m, Species& s, const dvec& loss, double fC, double fN, double fP, double fFe) {
    const pi_iron_params& p = s.ipp;
    for (int64_t i = 0; i < m->C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        const double l = loss[i], Bm = s.Bm[i], CH = s.CH[i], qP = s.qP[i];
        const double fe = i_feq(s.qFe[i], s.qFePS[i], s.qFeNR[i], s.qFeNF[i]);
        m->plk[PI_NH4][c] += jl_mulb(s.qNH4[i], ac) * l;
        m->plk[PI_NO3][c] += jl_mulb(s.qNO3[i], ac) * l;
        m->plk[PI_DOC][c] += jl_mulb((Bm + CH) * fC, ac) * l;
        m->plk[PI_DON][c] += jl_mulb(Bm * p.R_NC * fN, ac) * l;
        m->plk[PI_DOP][c] += jl_mulb((Bm * p.R_PC + qP) * fP, ac) * l;
        m->plk[PI_DFe][c] += jl_mulb(fe * fFe, ac) * l;
        m->plk[PI_POC][c] += jl_mulb((Bm + CH) * (1.0 - fC), ac) * l;
        m->plk[PI_PON][c] += jl_mulb(Bm * p.R_NC * (1.0 - fN), ac) * l;
        m->plk[PI_POP][c] += jl_mulb((Bm * p.R_PC + qP) * (1.0 - fP), ac) * l;
        m->plk[PI_PFe_bio][c] += jl_mulb(fe * (1.0 - fFe), ac) * l;
    }
    for (int64_t i = 0; i < m->C; ++i) s.ac[i] = (uint8_t)(s.ac[i] && jl_isless(loss[i], 1.0));
}

/* plankton_update! (IronEnergyMode/plankton_update.jl:1-33) */
bool plankton_update_iron(orc_model* m, Species& s, int spi, double dT, double t) {
    const pi_iron_params& p = s.ipp;
    const int64_t C = m->C;
    diags_proc(m, s, s.d_graz, &s.graz);
    calc_loss_iron(m, s, s.graz, p.grazFracC, p.grazFracN, p.grazFracP, p.grazFracFe);
    diags_proc(m, s, s.d_mort, &s.mort);
    calc_loss_iron(m, s, s.mort, p.mortFracC, p.mortFracN, p.mortFracP, p.mortFracFe);
    for (int64_t i = 0; i < C; ++i) s.dvid[i] = jl_mulb(s.dvid[i], s.ac[i]);
    diags_proc(m, s, s.d_dvid, &s.dvid);
    double dvidnum = 0.0;
    std::vector<int64_t> free_slots;
    for (int64_t i = 0; i < C; ++i) {
        dvidnum += s.dvid[i] * (double)s.ac[i];
        if (!s.ac[i]) free_slots.push_back(i + 1);
    }
    if (dvidnum > (double)free_slots.size()) {
        m->err = capacity_message(t);
        m->err_flags |= ERR_CAPACITY;
        return false;
    }
    /* divide! (division_death.jl:84-92): copy_daughter_individuals! (:44-70), divide_to_half! (:73-82) */
    double acc = 0.0;
    for (int64_t i = 0; i < C; ++i) { acc += s.dvid[i]; m->tidc[i] = acc; m->tidc_int[i] = (int64_t)acc; }
    for (int64_t i = 0; i < C; ++i)
        if (s.dvid[i] == 1.0) s.idx[i] = free_slots[(size_t)m->tidc_int[i] - 1];
    dvec* copied[] = { &s.x, &s.y, &s.z, &s.Sz, &s.Bm, &s.CH, &s.qNO3, &s.qNH4, &s.qP, &s.qFe, &s.qFePS,
                       &s.qFeNR, &s.qFeNF, &s.exEn, &s.Chl, &s.gen };
    for (int64_t i = 0; i < C; ++i)
        if (s.dvid[i] == 1.0 && s.idx[i] != 0) {
            const int64_t d = s.idx[i] - 1;
            for (dvec* v : copied) (*v)[d] = (*v)[i];
            s.ac[d] = s.ac[i]; s.dvid[d] = s.dvid[i]; s.tdark[d] = s.tdark[i];
        }
    dvec* halved[] = { &s.Sz, &s.Bm, &s.CH, &s.qNO3, &s.qNH4, &s.qP, &s.qFe, &s.qFePS, &s.qFeNR, &s.qFeNF,
                       &s.exEn, &s.Chl };
    for (int64_t i = 0; i < C; ++i) {
        const double f = (2.0 - s.dvid[i]) / 2.0;
        for (dvec* v : halved) (*v)[i] *= f;
        s.gen[i] += s.dvid[i];
        s.age[i] *= (1.0 - s.dvid[i]);
    }
    for (int64_t i = 0; i < C; ++i) s.idx[i] = 0;
    plankton_growth_iron(m, s, spi, dT, t);
    /* calc_consume_kernel! (consume_loss.jl:2-9) */
    for (int64_t i = 0; i < C; ++i) {
        size_t c = cell_of(m, s, i);
        int ac = s.ac[i];
        m->plk[PI_DIC][c] += jl_mulb((s.RS[i] - s.PS[i]) * dT, ac);
        m->plk[PI_NH4][c] += jl_mulb(-s.VNH4[i] * dT, ac);
        m->plk[PI_NO3][c] += jl_mulb(-s.VNO3[i] * dT, ac);
        m->plk[PI_PO4][c] += jl_mulb(-s.VPO4[i] * dT, ac);
        m->plk[PI_DFe][c] += jl_mulb(-s.VFe[i] * dT, ac);
    }
    /* diags_spcs! (Diagnostics/diagnostics_kernels.jl:22-31), the IronEnergyMode processes */
    if (m->proc_mask) {
        const dvec* procs[PI_NIPROC] = { &s.PS, &s.CF, &s.ECF, &s.RS, &s.ERS, &s.NR, &s.ENR, &s.NF, &s.ENF, &s.BS,
                                         &s.VNH4, &s.VNO3, &s.VPO4, &s.VFe, &s.PS2ST, &s.ST2PS, &s.NR2ST, &s.ST2NR,
                                         &s.NF2ST, &s.ST2NF, &s.Bm, &s.exEn, &s.CH, &s.qNO3, &s.qNH4, &s.qP, &s.qFe,
                                         &s.qFePS, &s.qFeNR, &s.qFeNF, &s.Chl, &s.tdark };
        for (int q = 0; q < PI_NIPROC; ++q)
            if (m->proc_mask & (1u << q)) diags_proc(m, s, s.d_proc[q], procs[q]);
    }
    diags_proc(m, s, s.d_num, nullptr);
    return true;
}

struct Ops {
    const Grid& g;
    inline double dxp(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i + 1, j, k)] - c[g.id(i, j, k)], g.L(i + 1, j, k)), g.L(i, j, k)); }
    inline double dyp(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i, j + 1, k)] - c[g.id(i, j, k)], g.L(i, j + 1, k)), g.L(i, j, k)); }
    inline double dzp(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i, j, k)] - c[g.id(i, j, k + 1)], g.L(i, j, k + 1)), g.L(i, j, k)); }
    inline double dx0(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i, j, k)] - c[g.id(i - 1, j, k)], g.L(i, j, k)), g.L(i - 1, j, k)); }
    inline double dy0(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i, j, k)] - c[g.id(i, j - 1, k)], g.L(i, j, k)), g.L(i, j - 1, k)); }
    inline double dz0(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i, j, k - 1)] - c[g.id(i, j, k)], g.L(i, j, k)), g.L(i, j, k - 1)); }
    inline double dxm(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i - 1, j, k)] - c[g.id(i - 2, j, k)], g.L(i - 1, j, k)), g.L(i - 2, j, k)); }
    inline double dym(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i, j - 1, k)] - c[g.id(i, j - 2, k)], g.L(i, j - 1, k)), g.L(i, j - 2, k)); }
    inline double dzm(const dvec& c, long i, long j, long k) const { return jl_mulb(jl_mulb(c[g.id(i, j, k - 2)] - c[g.id(i, j, k - 1)], g.L(i, j, k - 1)), g.L(i, j, k - 2)); }
};

/* θ and Ψ of DST3FL.jl:19-53 */
inline double theta(double dnum, double d0) {
    return fabs(d0) * F_THMAX <= fabs(dnum) ? copysign(F_THMAX, dnum * d0) : dnum / d0;
}
inline double psi_lim(double cfl, double th) {
    double d0 = (2.0 - cfl) * (1.0 - cfl) / 6.0;
    double d1 = (1.0 - cfl * cfl) / 6.0;
    return jl_max(0.0, jl_min(jl_min(1.0, d0 + d1 * th), th * (1.0 - cfl) / (cfl + F_1em20)));
}

/* adv_flux_x/y/z, DST3FL.jl:63-73 */
double adv_flux_x(const Grid& g, const Ops& o, long i, long j, long k, const dvec& u, const dvec& c, double dT) {
    double uu = u[g.id(i, j, k)];
    double cfl = fabs(uu * dT / g.dxC(i, j));
    double tr = g.Axk(i, j, k) * uu;
    double d0 = o.dx0(c, i, j, k);
    double psp = psi_lim(cfl, theta(o.dxm(c, i, j, k), d0));
    double psm = psi_lim(cfl, theta(o.dxp(c, i, j, k), d0));
    return 0.5 * (tr + fabs(tr)) * (c[g.id(i - 1, j, k)] + psp * d0)
         + 0.5 * (tr - fabs(tr)) * (c[g.id(i, j, k)] - psm * d0);
}
double adv_flux_y(const Grid& g, const Ops& o, long i, long j, long k, const dvec& v, const dvec& c, double dT) {
    double vv = v[g.id(i, j, k)];
    double cfl = fabs(vv * dT / g.dyC(i, j));
    double tr = g.Ayk(i, j, k) * vv;
    double d0 = o.dy0(c, i, j, k);
    double psp = psi_lim(cfl, theta(o.dym(c, i, j, k), d0));
    double psm = psi_lim(cfl, theta(o.dyp(c, i, j, k), d0));
    return 0.5 * (tr + fabs(tr)) * (c[g.id(i, j - 1, k)] + psp * d0)
         + 0.5 * (tr - fabs(tr)) * (c[g.id(i, j, k)] - psm * d0);
}
double adv_flux_z(const Grid& g, const Ops& o, long i, long j, long k, const dvec& w, const dvec& c, double dT) {
    double ww = w[g.id(i, j, k)];
    double cfl = fabs(ww * dT / g.dzC1(k));
    double tr = g.Az(i, j) * ww;
    double d0 = o.dz0(c, i, j, k);
    double psp = psi_lim(cfl, theta(o.dzm(c, i, j, k), d0));   /* Ψz⁺ uses θz⁺ = δz⁻/δz⁰ */
    double psm = psi_lim(cfl, theta(o.dzp(c, i, j, k), d0));   /* Ψz⁻ uses θz⁻ = δz⁺/δz⁰ */
    return 0.5 * (tr + fabs(tr)) * (c[g.id(i, j, k)] + psm * d0)
         + 0.5 * (tr - fabs(tr)) * (c[g.id(i, j, k - 1)] - psp * d0);
}

/* tracer_advection!, Advection/multi_dim_adv.jl:111-135 */
void tracer_advection(orc_model* m, double dT) {
    const Grid& g = m->g;
    Ops o{g};
    for (int n = 0; n < PI_NTRACERS; ++n) m->tt[n] = m->tr[n];
    for (int dir = 0; dir < 3; ++dir) {
        const dvec& vel = dir == 0 ? m->u1 : dir == 1 ? m->v1 : m->w1;
        for (int n = 0; n < PI_NTRACERS; ++n) {
            dvec& Gc = m->Gcs[n];
            const dvec& cT = m->tt[n];
            #pragma omp parallel for schedule(static)
            for (long k = g.Hz + 1; k <= g.Hz + g.Nz; ++k)       /* calc_Gcˣ/ʸ/ᶻ_kernel! */
                for (long j = g.Hy + 1; j <= g.Hy + g.Ny; ++j)
                    for (long i = g.Hx + 1; i <= g.Hx + g.Nx; ++i)
                        Gc[g.id(i, j, k)] = dir == 0 ? adv_flux_x(g, o, i, j, k, vel, cT, dT)
                                          : dir == 1 ? adv_flux_y(g, o, i, j, k, vel, cT, dT)
                                                     : adv_flux_z(g, o, i, j, k, vel, cT, dT);
        }
        for (int n = 0; n < PI_NTRACERS; ++n) fill_halo_Gc(g, m->Gcs[n]);
        for (int n = 0; n < PI_NTRACERS; ++n) {                    /* multi_dim_x/y/z_kernel! */
            dvec& ct = m->tt[n];
            const dvec& Gc = m->Gcs[n];
            const dvec& c = m->tr[n];
            #pragma omp parallel for schedule(static)
            for (long k = g.Hz + 1; k <= g.Hz + g.Nz; ++k)
                for (long j = g.Hy + 1; j <= g.Hy + g.Ny; ++j)
                    for (long i = g.Hx + 1; i <= g.Hx + g.Nx; ++i) {
                        size_t q = g.id(i, j, k);
                        double ftr;
                        double dG;
                        if (dir == 0) {
                            dG = o.dxp(Gc, i, j, k);
                            ftr = jl_mulb(jl_mulb(g.Axk(i + 1, j, k) * vel[g.id(i + 1, j, k)] - g.Axk(i, j, k) * vel[q], g.L(i + 1, j, k)), g.L(i, j, k));
                        } else if (dir == 1) {
                            dG = o.dyp(Gc, i, j, k);
                            ftr = jl_mulb(jl_mulb(g.Ayk(i, j + 1, k) * vel[g.id(i, j + 1, k)] - g.Ayk(i, j, k) * vel[q], g.L(i, j + 1, k)), g.L(i, j, k));
                        } else {
                            dG = o.dzp(Gc, i, j, k);
                            ftr = jl_mulb(jl_mulb(g.Az(i, j) * vel[q] - g.Az(i, j) * vel[g.id(i, j, k + 1)], g.L(i, j, k + 1)), g.L(i, j, k));
                        }
                        ct[q] -= dT / g.vol(i, j, k) * (dG - c[q] * ftr);
                    }
        }
        for (int n = 0; n < PI_NTRACERS; ++n) fill_halo_tracer(g, m->tt[n]);
    }
    for (int n = 0; n < PI_NTRACERS; ++n) {                        /* calc_tracer_tendency! */
        #pragma omp parallel for schedule(static)
        for (size_t q = 0; q < g.G; ++q) m->Gcs[n][q] = m->tt[n][q] - m->tr[n][q];
    }
}

/* tracer_diffusion!, Advection/tracer_diffusion.jl:1-30 */
void tracer_diffusion(orc_model* m, double dT) {
    const Grid& g = m->g;
    Ops o{g};
    double kx = m->bgc.kappa_h, ky = m->bgc.kappa_h, kz = m->bgc.kappa_v;
    #pragma omp parallel for schedule(static)
    for (int n = 0; n < PI_NTRACERS; ++n) {
        const dvec& c = m->tr[n];
        dvec& Gc = m->Gcs[n];
        auto fx = [&](long i, long j, long k) { return kx * g.Axk(i, j, k) * (o.dx0(c, i, j, k) / g.dxF(i, j)); };
        auto fy = [&](long i, long j, long k) { return ky * g.Ayk(i, j, k) * (o.dy0(c, i, j, k) / g.dyF(i, j)); };
        auto fz = [&](long i, long j, long k) { return kz * g.Az(i, j) * (o.dz0(c, i, j, k) / g.dzF1(k)); };
        for (long k = g.Hz + 1; k <= g.Hz + g.Nz; ++k)
            for (long j = g.Hy + 1; j <= g.Hy + g.Ny; ++j)
                for (long i = g.Hx + 1; i <= g.Hx + g.Nx; ++i) {
                    double ax = jl_mulb(jl_mulb(fx(i + 1, j, k) - fx(i, j, k), g.L(i + 1, j, k)), g.L(i, j, k));
                    double ay = jl_mulb(jl_mulb(fy(i, j + 1, k) - fy(i, j, k), g.L(i, j + 1, k)), g.L(i, j, k));
                    double az = jl_mulb(jl_mulb(fz(i, j, k) - fz(i, j, k + 1), g.L(i, j, k + 1)), g.L(i, j, k));
                    double lap = 1.0 / g.vol(i, j, k) * (ax + ay + az);
                    size_t q = g.id(i, j, k);
                    Gc[q] = Gc[q] + lap * dT;
                }
    }
}

/* tracer_sinking!, Advection/tracer_sinking.jl:1-42 */
void tracer_sinking(orc_model* m, double dT) {
    const Grid& g = m->g;
    const int names[3] = { PI_PFe_inorg, PI_Dust, PI_PFe_bio };
    for (int q3 = 0; q3 < 3; ++q3) {
        int n = names[q3];
        double wsink = q3 < 2 ? m->bgc.w_sink_inorg : m->bgc.w_sink_org;
        for (size_t q = 0; q < g.G; ++q) m->flux_sink[q] = wsink * m->tr[n][q];
        for (int j = 1; j <= g.Gy; ++j)                  /* fill_halo_flux_sink!, halo_regions.jl:58-62 */
            for (int i = 1; i <= g.Gx; ++i) {
                for (int k = 1; k <= g.Hz; ++k) m->flux_sink[g.id(i, j, k)] = 0.0;
                for (int k = g.Nz + g.Hz; k <= g.Nz + 2 * g.Hz; ++k) m->flux_sink[g.id(i, j, k)] = 0.0;
            }
        dvec& Gc = m->Gcs[n];
        for (long k = 1; k <= g.Nz; ++k)
            for (long j = 1; j <= g.Ny; ++j)
                for (long i = 1; i <= g.Nx; ++i) {
                    long ii = i + g.Hx, jj = j + g.Hy, kk = k + g.Hz;
                    size_t q = g.id(ii, jj, kk);
                    Gc[q] = Gc[q] + (m->flux_sink[g.id(ii, jj, kk - 1)] - m->flux_sink[q]) / g.dzC1(k) * dT;
                }
    }
}

/* tracer_forcing!, tracer_forcings.jl:2-50 (interior; the halo part of Gcs is never read) */
void tracer_forcing(orc_model* m, double dT) {
    const Grid& g = m->g;
    const pi_bgc_params& b = m->bgc;
    #pragma omp parallel for schedule(static)
    for (long k = g.Hz + 1; k <= g.Hz + g.Nz; ++k)
        for (long j = g.Hy + 1; j <= g.Hy + g.Ny; ++j)
            for (long i = g.Hx + 1; i <= g.Hx + g.Nx; ++i) {
                size_t q = g.id(i, j, k);
                double T[PI_NTRACERS];
                for (int n = 0; n < PI_NTRACERS; ++n) T[n] = jl_max(0.0, m->tr[n][q]);
                std::vector<dvec>& F = m->Gcs;
                F[PI_DIC][q] = F[PI_DIC][q] + T[PI_DOC] * b.kDOC * dT;
                F[PI_DOC][q] = F[PI_DOC][q] - T[PI_DOC] * b.kDOC * dT + T[PI_POC] * b.kPOC * dT;
                F[PI_POC][q] = F[PI_POC][q] - T[PI_POC] * b.kPOC * dT;
                F[PI_NH4][q] = F[PI_NH4][q] + T[PI_DON] * b.kDON * dT - T[PI_NH4] * b.Nit * dT;
                F[PI_NO3][q] = F[PI_NO3][q] + T[PI_NH4] * b.Nit * dT;
                F[PI_DON][q] = F[PI_DON][q] - T[PI_DON] * b.kDON * dT + T[PI_PON] * b.kPON * dT;
                F[PI_PON][q] = F[PI_PON][q] - T[PI_PON] * b.kPON * dT;
                F[PI_PO4][q] = F[PI_PO4][q] + T[PI_DOP] * b.kDOP * dT;
                F[PI_DOP][q] = F[PI_DOP][q] - T[PI_DOP] * b.kDOP * dT + T[PI_POP] * b.kPOP * dT;
                F[PI_POP][q] = F[PI_POP][q] - T[PI_POP] * b.kPOP * dT;
                F[PI_DFe][q] = F[PI_DFe][q] + T[PI_PFe_bio] * b.kPOC * dT
                             - (b.lambda_POC * T[PI_POC] + b.lambda_min + b.lambda_dust * T[PI_Dust]) * T[PI_DFe] * b.DFeFrac * dT
                             + T[PI_PFe_inorg] * b.kdiss * dT
                             - jl_max((T[PI_DFe] - b.ligand), 0.0) * T[PI_DFe] * b.DFeFrac * b.lambda_Fe * dT;
                F[PI_PFe_bio][q] = F[PI_PFe_bio][q] + T[PI_POC] * T[PI_DFe] * b.DFeFrac * b.lambda_POC * dT
                                 - b.kPOC * T[PI_PFe_bio] * dT;
                F[PI_PFe_inorg][q] = F[PI_PFe_inorg][q] - T[PI_PFe_inorg] * b.kdiss * dT
                                   + (b.lambda_min + b.lambda_dust * T[PI_Dust]) * T[PI_DFe] * b.DFeFrac * dT
                                   + jl_max((T[PI_DFe] - b.ligand), 0.0) * T[PI_DFe] * b.DFeFrac * b.lambda_Fe * dT;
            }
}

/* getbc, HaloRegions/boundary_conditions.jl:44-52 (a, b are 1-based face indices) */
inline double getbc(const FluxBC& bc, int n1, int n2, long a, long b, int64_t it) {
    if (bc.kind == PI_BC_CONST) return bc.v[0];
    if (bc.kind == PI_BC_ARRAY2D) return bc.v[(size_t)(a - 1) + (size_t)n1 * (size_t)(b - 1)];
    const int64_t t = it < 1 ? 1 : (it > bc.nt ? bc.nt : it);   /* Julia would raise a BoundsError */
    return bc.v[(size_t)(a - 1) + (size_t)n1 * ((size_t)(b - 1) + (size_t)n2 * (size_t)(t - 1))];
}

/* apply_bcs!, HaloRegions/apply_bcs.jl:4-98 */
void apply_bcs(orc_model* m, double dT) {
    const Grid& g = m->g;
    int64_t it = m->iteration;
    for (int n = 0; n < PI_NTRACERS; ++n) {
        dvec& Gc = m->Gcs[n];
        const FluxBC* b = m->bc[n];
        if (b[PI_WEST].kind) for (long k = 1; k <= g.Nz; ++k) for (long j = 1; j <= g.Ny; ++j) {
            long jj = j + g.Hy, kk = k + g.Hz;
            Gc[g.id(1 + g.Hx, jj, kk)] += getbc(b[PI_WEST], g.Ny, g.Nz, j, k, it) * dT * g.Axk(1 + g.Hx, jj, kk) / g.vol(1 + g.Hx, jj, kk);
        }
        if (b[PI_EAST].kind) for (long k = 1; k <= g.Nz; ++k) for (long j = 1; j <= g.Ny; ++j) {
            long jj = j + g.Hy, kk = k + g.Hz;
            Gc[g.id(g.Nx + g.Hx, jj, kk)] -= getbc(b[PI_EAST], g.Ny, g.Nz, j, k, it) * dT * g.Axk(g.Nx + g.Hx, jj, kk) / g.vol(g.Nx + g.Hx, jj, kk);
        }
        if (b[PI_SOUTH].kind) for (long k = 1; k <= g.Nz; ++k) for (long i = 1; i <= g.Nx; ++i) {
            long ii = i + g.Hx, kk = k + g.Hz;
            Gc[g.id(ii, 1 + g.Hy, kk)] += getbc(b[PI_SOUTH], g.Nx, g.Nz, i, k, it) * dT * g.Ayk(ii, 1 + g.Hy, kk) / g.vol(ii, 1 + g.Hy, kk);
        }
        if (b[PI_NORTH].kind) for (long k = 1; k <= g.Nz; ++k) for (long i = 1; i <= g.Nx; ++i) {
            long ii = i + g.Hx, kk = k + g.Hz;
            Gc[g.id(ii, g.Ny + g.Hy, kk)] -= getbc(b[PI_NORTH], g.Nx, g.Nz, i, k, it) * dT * g.Ayk(ii, g.Ny + g.Hy, kk) / g.vol(ii, g.Ny + g.Hy, kk);
        }
        if (b[PI_BOTTOM].kind) for (long j = 1; j <= g.Ny; ++j) for (long i = 1; i <= g.Nx; ++i) {
            long ii = i + g.Hx, jj = j + g.Hy, kk = g.Nz + g.Hz;
            Gc[g.id(ii, jj, kk)] += getbc(b[PI_BOTTOM], g.Nx, g.Ny, i, j, it) * dT * g.Az(ii, jj) / g.vol(ii, jj, kk);
        }
        if (b[PI_TOP].kind) for (long j = 1; j <= g.Ny; ++j) for (long i = 1; i <= g.Nx; ++i) {
            long ii = i + g.Hx, jj = j + g.Hy, kk = 1 + g.Hz;
            Gc[g.id(ii, jj, kk)] -= getbc(b[PI_TOP], g.Nx, g.Ny, i, j, it) * dT * g.Az(ii, jj) / g.vol(ii, jj, kk);
        }
    }
}

/* apply_tendency!, tracer_update.jl:6-13 */
void apply_tendency(orc_model* m) {
    const Grid& g = m->g;
    for (int n = 0; n < PI_NTRACERS; ++n)
        #pragma omp parallel for schedule(static)
        for (long k = g.Hz + 1; k <= g.Hz + g.Nz; ++k)
            for (long j = g.Hy + 1; j <= g.Hy + g.Ny; ++j)
                for (long i = g.Hx + 1; i <= g.Hx + g.Nx; ++i) {
                    size_t q = g.id(i, j, k);
                    m->tr[n][q] += m->Gcs[n][q] + m->plk[n][q] / g.vol(i, j, k);
                }
}

/* tracer_update!, tracer_update.jl:22-43 */
void tracer_update(orc_model* m, double dT) {
    tracer_advection(m, dT);
    tracer_diffusion(m, dT);
    tracer_sinking(m, dT);
    tracer_forcing(m, dT);     /* zero_fields!(tracer_temp) + the forcing broadcasts */
    apply_bcs(m, dT);
    apply_tendency(m);
    for (int n = 0; n < PI_NTRACERS; ++n) fill_halo_tracer(m->g, m->tr[n]);
}

void zero(dvec& v) { std::fill(v.begin(), v.end(), 0.0); }

/* ---------------------------------------------------------------------------------------- */
/* Abiotic particles, src/Individuals/Abiotic/particle_interaction.jl                          */
/* ---------------------------------------------------------------------------------------- */

/* The capacity error of particle_release! and particles_from_bcs! (:128-130, :252-271). */
std::string abiotic_capacity_message(double t) {
    const std::string s = capacity_message(t);
    return "number of abiotic particles exceeds the capacity at timestep " + s.substr(s.find("timestep ") + 9);
}

/* particles_from_bcs!, :252-271, with calc_particle_bcs! (:142-229). A boundary cell of a face
 * with a particle flux becomes a particle when rnd·sz_min·Nsuper < flux·ΔT·area (rnd one draw per
 * cell and step). The faces write in the order top, bottom, east, west, north, south, so a later
 * face decides a cell two faces share (edges; top and bottom when Nz = 1). New particles take the
 * free slots in ascending order, cells in column-major order (findall), at cell − halo − 0.4 on
 * each axis, computed in Float32 (Int − Float32 promotes to Float32, :239-244). Their cell indices
 * stay as the slot held them until find_inds!. */
int particles_from_bcs(orc_model* m, Abiotic& a, int sa, double dT) {
    const Grid& g = m->g;
    const int64_t it = m->iteration;
    const FluxBC* b = a.bc;
    bool any = false;
    for (int f = 0; f < 6; ++f) any = any || b[f].kind != PI_BC_NONE;
    if (!any) return PI_OK;
    std::vector<uint8_t> flag(g.G, 0);
    auto set = [&](long i, long j, long k, double flux, double area) {
        double r0, r1, r2;
        pi_draw3(m->seed, (uint32_t)it, (uint32_t)sa, PI_DRAW_ABIO_BC, (uint32_t)g.id(i, j, k), &r0, &r1, &r2);
        flag[g.id(i, j, k)] = (uint8_t)jl_isless(r0 * a.p.sz_min * a.p.Nsuper, flux * dT * area);
    };
    if (b[PI_TOP].kind) for (long j = 1; j <= g.Ny; ++j) for (long i = 1; i <= g.Nx; ++i)
        set(i + g.Hx, j + g.Hy, 1 + g.Hz, getbc(b[PI_TOP], g.Nx, g.Ny, i, j, it), g.Az(i + g.Hx, j + g.Hy));
    if (b[PI_BOTTOM].kind) for (long j = 1; j <= g.Ny; ++j) for (long i = 1; i <= g.Nx; ++i)
        set(i + g.Hx, j + g.Hy, g.Nz + g.Hz, getbc(b[PI_BOTTOM], g.Nx, g.Ny, i, j, it), g.Az(i + g.Hx, j + g.Hy));
    if (b[PI_EAST].kind) for (long k = 1; k <= g.Nz; ++k) for (long j = 1; j <= g.Ny; ++j)
        set(g.Nx + g.Hx, j + g.Hy, k + g.Hz, getbc(b[PI_EAST], g.Ny, g.Nz, j, k, it), g.Axk(g.Nx + g.Hx, j + g.Hy, k + g.Hz));
    if (b[PI_WEST].kind) for (long k = 1; k <= g.Nz; ++k) for (long j = 1; j <= g.Ny; ++j)
        set(1 + g.Hx, j + g.Hy, k + g.Hz, getbc(b[PI_WEST], g.Ny, g.Nz, j, k, it), g.Axk(1 + g.Hx, j + g.Hy, k + g.Hz));
    if (b[PI_NORTH].kind) for (long k = 1; k <= g.Nz; ++k) for (long i = 1; i <= g.Nx; ++i)
        set(i + g.Hx, g.Ny + g.Hy, k + g.Hz, getbc(b[PI_NORTH], g.Nx, g.Nz, i, k, it), g.Ayk(i + g.Hx, g.Ny + g.Hy, k + g.Hz));
    if (b[PI_SOUTH].kind) for (long k = 1; k <= g.Nz; ++k) for (long i = 1; i <= g.Nx; ++i)
        set(i + g.Hx, 1 + g.Hy, k + g.Hz, getbc(b[PI_SOUTH], g.Nx, g.Nz, i, k, it), g.Ayk(i + g.Hx, 1 + g.Hy, k + g.Hz));
    size_t n = 0;
    for (size_t q = 0; q < g.G; ++q) n += flag[q];
    if (n == 0) return PI_OK;                                          /* sum(tr_temp) == 0 */
    std::vector<int64_t> freel;
    for (int64_t k = 0; k < m->C; ++k) if (!a.ac[k]) freel.push_back(k);
    if (n > freel.size()) { m->err = abiotic_capacity_message(m->t); return PI_ERR_CAPACITY; }
    size_t r = 0;
    for (size_t q = 0; q < g.G; ++q) {
        if (!flag[q]) continue;
        const long i = (long)(q % (size_t)g.Gx) + 1, j = (long)((q / (size_t)g.Gx) % (size_t)g.Gy) + 1;
        const long k = (long)(q / ((size_t)g.Gx * (size_t)g.Gy)) + 1;
        const int64_t d = freel[r++];
        a.ac[d] = 1;
        a.x[d] = (double)((float)(i - g.Hx) - 0.4f);
        a.y[d] = (double)((float)(j - g.Hy) - 0.4f);
        a.z[d] = (double)((float)(k - g.Hz) - 0.4f);
    }
    return PI_OK;
}

/* calc_distance, :3-15: the distance in metres of two particles whose find_inds! cells are equal
 * (ΔxF, ΔyF, ΔzF at the first one's cell), else 1.0f20. dx^2.0f0 is Float64^Float64 with an
 * integral exponent, which Julia evaluates as the integer power. */
inline double calc_distance(const Grid& g, int64_t xi1, int64_t yi1, int64_t zi1, double x1, double y1, double z1,
                            int64_t xi2, int64_t yi2, int64_t zi2, double x2, double y2, double z2) {
    if (xi1 == xi2 && yi1 == yi2 && zi1 == zi2) {
        const double dx = (x1 - x2) * g.dxF(xi1, yi1);
        const double dy = (y1 - y2) * g.dyF(xi1, yi1);
        const double dz = (z1 - z2) * g.dzF1(zi1);
        return sqrt(pi_pow_int(dx, 2) + pi_pow_int(dy, 2) + pi_pow_int(dz, 2));
    }
    return (double)1.0e20f;
}

/* particle_interaction!, :18-81, as a single-threaded run of its kernels leaves it.
 * calc_interaction_kernel! (:24-40) writes intac[(i % max_candidates) + 1, k] = i for every
 * active phytoplankton i (1-based, ascending) within Rd of active particle k, so an entry ends
 * with the largest such i; merge_particle_kernel! (:50-66) walks the particles in ascending k,
 * each merging into its first candidate whose ptc is below max_ptc (ptc += 1, the particle
 * inactive). This is the reference's scan over every pair. */
int particle_interaction(orc_model* m, Species& pl, Abiotic& a, int sp) {
    const Grid& g = m->g;
    const int64_t C = m->C, K = m->maxc;
    std::fill(m->intac.begin(), m->intac.end(), 0);                    /* reset_interaction! */
    for (int64_t i = 0; i < C; ++i) {
        if (!pl.ac[i]) continue;
        for (int64_t k = 0; k < C; ++k) {
            if (!a.ac[k]) continue;
            const double dist = calc_distance(g, pl.xi[i], pl.yi[i], pl.zi[i], pl.x[i], pl.y[i], pl.z[i],
                                              a.xi[k], a.yi[k], a.zi[k], a.x[k], a.y[k], a.z[k]);
            if (dist < a.p.Rd) m->intac[(size_t)k * (size_t)K + (size_t)((i + 1) % K)] = i + 1;
        }
    }
    for (int64_t k = 0; k < C; ++k) {
        if (!a.ac[k]) continue;
        for (int64_t j = 0; j < K; ++j) {
            const int64_t pid = m->intac[(size_t)k * (size_t)K + (size_t)j];
            if (pid <= 0) continue;
            const double mp = m->max_ptc[sp];
            if (mp != mp) { m->err = "type NamedTuple has no field max_ptc"; return PI_ERR_PARAM; }
            if (pl.ptc[pid - 1] < mp) { pl.ptc[pid - 1] += 1.0; a.ac[k] = 0; break; }
        }
    }
    return PI_OK;
}

/* particle_release!, :124-137, with get_release_probability! (:85-91), get_tind! (utils.jl:76-86)
 * and release_abiotic_particle_kernel! (:93-101). An active phytoplankton releases one particle
 * when rnd.x < release_P·ΔT·ptc; releasers take the free particle slots in ascending order. The
 * particle goes to the phytoplankton's position plus (rnd.x, rnd.y, rnd.z): rnd.x is the release
 * draw, rnd.y and rnd.z still hold the mortality and division draws of the last species'
 * get_probability! (calc_release_position!, :109-122, is not called). Its cell indices stay as
 * the slot held them until the next find_inds!. */
int particle_release(orc_model* m, Species& pl, Abiotic& a, int pair, double dT) {
    const int64_t C = m->C;
    std::vector<uint8_t> R((size_t)C, 0);
    dvec rx((size_t)C);
    int64_t nrel = 0;
    for (int64_t i = 0; i < C; ++i) {
        double r1, r2;
        pi_draw3(m->seed, (uint32_t)m->iteration, (uint32_t)pair, PI_DRAW_RELEASE, (uint32_t)i, &rx[i], &r1, &r2);
        R[i] = (uint8_t)(jl_isless(rx[i], a.p.release_P * dT * pl.ptc[i]) && pl.ac[i]);
        nrel += R[i];
    }
    std::vector<int64_t> freel;
    for (int64_t k = 0; k < C; ++k) if (!a.ac[k]) freel.push_back(k);
    if (nrel > (int64_t)freel.size()) { m->err = abiotic_capacity_message(m->t); return PI_ERR_CAPACITY; }
    size_t r = 0;
    for (int64_t i = 0; i < C; ++i) {
        if (!R[i]) continue;
        double d0, dy, dz;
        pi_draw3(m->seed, (uint32_t)m->iteration, (uint32_t)(m->nsp - 1), PI_DRAW_DECISION, (uint32_t)i, &d0, &dy, &dz);
        const int64_t d = freel[r++];
        a.ac[d] = 1;
        a.x[d] = pl.x[i] + rx[i];
        a.y[d] = pl.y[i] + dy;
        a.z[d] = pl.z[i] + dz;
        pl.ptc[i] -= 1.0;
    }
    return PI_OK;
}

/* The abiotic phase before the phytoplankton (time_step.jl:24-39). */
int abiotic_update(orc_model* m, double dT) {
    for (size_t sa = 0; sa < m->ab.size(); ++sa) {
        Abiotic& a = m->ab[sa];
        int st = particles_from_bcs(m, a, (int)sa, dT);
        if (st) return st;
        particle_advection(m, a, dT);
        particle_diffusion(m, a, (int)sa, dT, PI_DRAW_ABIO_DIFFUSION);
        find_inds(m, a);
    }
    return PI_OK;
}

/* Interaction, release and their diagnostics after the phytoplankton (time_step.jl:120-158). */
int abiotic_exchange(orc_model* m, double dT) {
    if (m->ab.empty()) return PI_OK;
    for (const auto& pr : m->pal_intac) {
        int st = particle_interaction(m, m->sp[pr.first], m->ab[pr.second], pr.first);
        if (st) return st;
    }
    for (size_t q = 0; q < m->pal_release.size(); ++q) {
        const auto& pr = m->pal_release[q];
        int st = particle_release(m, m->sp[pr.first], m->ab[pr.second], (int)q, dT);
        if (st) return st;
    }
    for (Species& S : m->sp) diags_proc(m, S, S.d_ptc, &S.ptc);
    for (Abiotic& a : m->ab)
        for (int64_t k = 0; k < m->C; ++k) a.d_num[cell_of(m, a, k)] += (double)(a.ac[k] && a.ac[k]);
    return PI_OK;
}

}  // namespace

/* ============================================================================================ */
/* C entry points (orc_* mirror the pi_* entry points of include/pib200.h)                       */
/* ============================================================================================ */

static std::string g_create_err;

extern "C" {

int orc_create(const pi_grid* grid, const pi_bgc_params* bgc, const pi_quota_params* species,
               int32_t nspecies, int64_t capacity, uint64_t seed, orc_model** out) {
    if (!grid || !bgc || !species || !out || nspecies < 1 || capacity < 1 || !grid->dzF || !grid->dzC) {
        g_create_err = "orc_create: bad argument"; return PI_ERR_ARG;
    }
    if (grid->topo[2] != PI_BOUNDED) { g_create_err = "z topology must be Bounded"; return PI_ERR_ARG; }
    orc_model* m = new orc_model();
    Grid& g = m->g;
    g.Nx = grid->Nx; g.Ny = grid->Ny; g.Nz = grid->Nz; g.Hx = grid->Hx; g.Hy = grid->Hy; g.Hz = grid->Hz;
    g.Gx = g.Nx + 2 * g.Hx; g.Gy = g.Ny + 2 * g.Hy; g.Gz = g.Nz + 2 * g.Hz;
    g.tx = grid->topo[0]; g.ty = grid->topo[1]; g.tz = grid->topo[2];
    g.dx = grid->dx; g.dy = grid->dy;
    g.dzF.assign(grid->dzF, grid->dzF + g.Gz);
    g.dzC.assign(grid->dzC, grid->dzC + g.Gz);
    g.G = (size_t)g.Gx * g.Gy * g.Gz;
    g.lm.assign(g.G, 1);
    if (grid->landmask) g.lm.assign(grid->landmask, grid->landmask + g.G);
    if (const pi_grid_metrics* mt = grid->metrics) {          /* LatLonGrid */
        const size_t G2 = (size_t)g.Gx * g.Gy;
        const double* a2[5] = { mt->dxC, mt->dyC, mt->dxF, mt->dyF, mt->Az };
        const double* a3[3] = { mt->Ax, mt->Ay, mt->Vol };
        for (const double* p : a2) if (!p) { delete m; g_create_err = "orc_create: LatLonGrid metrics incomplete"; return PI_ERR_ARG; }
        for (const double* p : a3) if (!p) { delete m; g_create_err = "orc_create: LatLonGrid metrics incomplete"; return PI_ERR_ARG; }
        g.ll = true;
        g.mdxC.assign(mt->dxC, mt->dxC + G2); g.mdyC.assign(mt->dyC, mt->dyC + G2);
        g.mdxF.assign(mt->dxF, mt->dxF + G2); g.mdyF.assign(mt->dyF, mt->dyF + G2);
        g.mAz.assign(mt->Az, mt->Az + G2);
        g.mAx.assign(mt->Ax, mt->Ax + g.G); g.mAy.assign(mt->Ay, mt->Ay + g.G); g.mVol.assign(mt->Vol, mt->Vol + g.G);
    }
    m->bgc = *bgc; m->nsp = nspecies; m->C = capacity; m->seed = seed;
    m->sp.resize(nspecies);
    size_t C = (size_t)capacity;
    for (int s = 0; s < nspecies; ++s) {
        Species& S = m->sp[s];
        S.p = species[s];
        for (dvec* v : { &S.x, &S.y, &S.z, &S.Sz, &S.Bm, &S.Cq, &S.Nq, &S.Pq, &S.Chl, &S.gen, &S.age,
                         &S.PS, &S.VDOC, &S.VNH4, &S.VNO3, &S.VPO4, &S.rChl, &S.resp, &S.BS, &S.exu,
                         &S.graz, &S.mort, &S.dvid, &S.ptc }) v->assign(C, 0.0);
        S.xi.assign(C, 0); S.yi.assign(C, 0); S.zi.assign(C, 0); S.idx.assign(C, 0);
        S.ac.assign(C, 0);
        for (dvec* v : { &S.d_num, &S.d_graz, &S.d_mort, &S.d_dvid, &S.d_ptc }) v->assign(g.G, 0.0);
    }
    m->tr.assign(PI_NTRACERS, dvec(g.G, 0.0));
    m->Gcs.assign(PI_NTRACERS, dvec(g.G, 0.0));
    m->tt.assign(PI_NTRACERS, dvec(g.G, 0.0));
    m->plk.assign(PI_NTRACERS, dvec(g.G, 0.0));
    for (dvec* v : { &m->u0, &m->v0, &m->w0, &m->u1, &m->v1, &m->w1, &m->uh, &m->vh, &m->wh,
                     &m->temp, &m->flux_sink, &m->par, &m->par0, &m->Chl, &m->pop, &m->d_PAR }) v->assign(g.G, 0.0);
    m->PARF.assign((size_t)g.Nx * g.Ny, 0.0);
    for (dvec* v : { &m->rx, &m->ry, &m->rz, &m->vx, &m->vy, &m->vz, &m->vu1, &m->vv1, &m->vw1,
                     &m->vu2, &m->vv2, &m->vw2, &m->tNH4, &m->tNO3, &m->tPO4, &m->tDOC, &m->tDFe,
                     &m->tpar, &m->tT, &m->tpop, &m->tdpar, &m->tidc }) v->assign(C, 0.0);
    m->tidc_int.assign(C, 0);
    m->iteration = 0; m->t = 0.0; m->err_flags = 0;
    *out = m;
    return PI_OK;
}

/* A CarbonMode model: the QuotaMode setup with the shared parameters filled in, then the species
 * switched to CarbonMode (their Cq, Nq, Pq stay zero). */
int orc_create_carbon(const pi_grid* grid, const pi_bgc_params* bgc, const pi_carbon_params* species,
                      int32_t nspecies, int64_t capacity, uint64_t seed, orc_model** out) {
    if (!species || nspecies < 1) { g_create_err = "orc_create_carbon: bad argument"; return PI_ERR_ARG; }
    std::vector<pi_quota_params> q((size_t)nspecies);
    for (int s = 0; s < nspecies; ++s) {
        const pi_carbon_params& c = species[s];
        pi_quota_params& p = q[s];
        memset(&p, 0, sizeof p);
        p.Nsuper = c.Nsuper; p.Cquota = c.Cquota; p.mean = c.mean; p.var = c.var; p.alpha = c.alpha;
        p.Phi = c.Phi; p.Topt = c.Topt; p.Tmax = c.Tmax; p.Ea = c.Ea; p.PCmax = c.PCmax; p.respir = c.respir;
        p.grz_P = c.grz_P; p.dvid_type = c.dvid_type; p.dvid_P = c.dvid_P; p.dvid_reg = c.dvid_reg;
        p.dvid_reg2 = c.dvid_reg2; p.mort_P = c.mort_P; p.mort_reg = c.mort_reg;
        p.grazFracC = c.grazFracC; p.mortFracC = c.mortFracC;
    }
    int st = orc_create(grid, bgc, q.data(), nspecies, capacity, seed, out);
    if (st) return st;
    for (int s = 0; s < nspecies; ++s) {
        Species& S = (*out)->sp[s];
        S.carbon = 1;
        S.cp = species[s];
        for (dvec* v : { &S.Bd, &S.RP, &S.RS, &S.TD }) v->assign((size_t)capacity, 0.0);
    }
    return PI_OK;
}

/* A MacroMolecularMode model: the QuotaMode setup with the shared parameters, then the species
 * switched to MacroMolecularMode (Sz, Bm and the quotas stay zero). */
int orc_create_macro(const pi_grid* grid, const pi_bgc_params* bgc, const pi_macro_params* species,
                     int32_t nspecies, int64_t capacity, uint64_t seed, orc_model** out) {
    if (!species || nspecies < 1) { g_create_err = "orc_create_macro: bad argument"; return PI_ERR_ARG; }
    std::vector<pi_quota_params> q((size_t)nspecies);
    for (int s = 0; s < nspecies; ++s) {
        const pi_macro_params& c = species[s];
        pi_quota_params& p = q[s];
        memset(&p, 0, sizeof p);
        p.Nsuper = c.Nsuper; p.var = c.var; p.alpha = c.alpha; p.Phi = c.Phi; p.Topt = c.Topt; p.Tmax = c.Tmax;
        p.Ea = c.Ea; p.PCmax = c.PCmax; p.respir = c.respir; p.grz_P = c.grz_P; p.dvid_type = 1.0;
        p.dvid_P = c.dvid_P; p.mort_P = c.mort_P; p.mort_reg = c.mort_reg;
        p.grazFracC = c.grazFracC; p.grazFracN = c.grazFracN; p.grazFracP = c.grazFracP;
        p.mortFracC = c.mortFracC; p.mortFracN = c.mortFracN; p.mortFracP = c.mortFracP;
    }
    int st = orc_create(grid, bgc, q.data(), nspecies, capacity, seed, out);
    if (st) return st;
    for (int s = 0; s < nspecies; ++s) {
        Species& S = (*out)->sp[s];
        S.macro = 1;
        S.mp = species[s];
        for (dvec* v : { &S.PRO, &S.DNA, &S.RNA, &S.CH, &S.NST, &S.PST, &S.S_PRO, &S.S_DNA, &S.S_RNA })
            v->assign((size_t)capacity, 0.0);
    }
    return PI_OK;
}

/* An IronEnergyMode model: the QuotaMode setup with the shared parameters, then the species switched
 * to IronEnergyMode (their Cq, Nq, Pq stay zero). */
int orc_create_iron(const pi_grid* grid, const pi_bgc_params* bgc, const pi_iron_params* species,
                    int32_t nspecies, int64_t capacity, uint64_t seed, orc_model** out) {
    if (!species || nspecies < 1) { g_create_err = "orc_create_iron: bad argument"; return PI_ERR_ARG; }
    std::vector<pi_quota_params> q((size_t)nspecies);
    for (int s = 0; s < nspecies; ++s) {
        const pi_iron_params& c = species[s];
        pi_quota_params& p = q[s];
        memset(&p, 0, sizeof p);
        p.Nsuper = c.Nsuper; p.Cquota = c.Cquota; p.mean = c.mean; p.var = c.var; p.Chl2Cint = c.Chl2Cint;
        p.alpha = c.alpha; p.Topt = c.Topt; p.Tmax = c.Tmax; p.Ea = c.Ea; p.PCmax = c.PCmax;
        p.R_NC = c.R_NC; p.R_PC = c.R_PC; p.grz_P = c.grz_P; p.dvid_type = c.dvid_type; p.dvid_P = c.dvid_P;
        p.dvid_reg = c.dvid_reg; p.dvid_reg2 = c.dvid_reg2; p.mort_P = c.mort_P; p.mort_reg = c.mort_reg;
        p.grazFracC = c.grazFracC; p.grazFracN = c.grazFracN; p.grazFracP = c.grazFracP;
        p.mortFracC = c.mortFracC; p.mortFracN = c.mortFracN; p.mortFracP = c.mortFracP;
    }
    int st = orc_create(grid, bgc, q.data(), nspecies, capacity, seed, out);
    if (st) return st;
    for (int s = 0; s < nspecies; ++s) {
        Species& S = (*out)->sp[s];
        S.iron = 1;
        S.ipp = species[s];
        for (dvec* v : { &S.CH, &S.RS, &S.qNO3, &S.qNH4, &S.qP, &S.qFe, &S.qFePS, &S.qFeNR, &S.qFeNF, &S.exEn, &S.tdark,
                         &S.CF, &S.ECF, &S.NF, &S.ENF, &S.VFe, &S.PS2ST, &S.ST2PS, &S.NR2ST, &S.ST2NR, &S.NF2ST,
                         &S.ST2NF, &S.ERS, &S.NR, &S.ENR })
            v->assign((size_t)capacity, 0.0);
    }
    return PI_OK;
}

int orc_destroy(orc_model* m) { delete m; return PI_OK; }

int orc_set_individuals(orc_model* m, int32_t sp, const pi_individuals* in) {
    if (!m || sp < 0 || sp >= m->nsp || !in) return PI_ERR_ARG;
    Species& S = m->sp[sp];
    size_t C = (size_t)m->C;
    auto cp = [&](dvec& d, const double* s) { d.assign(s, s + C); };
    cp(S.x, in->x); cp(S.y, in->y); cp(S.z, in->z);
    S.xi.assign(in->xi, in->xi + C); S.yi.assign(in->yi, in->yi + C); S.zi.assign(in->zi, in->zi + C);
    if (S.macro) {
        const double* cols[6] = { in->PRO, in->DNA, in->RNA, in->CH, in->NST, in->PST };
        dvec* dst[6] = { &S.PRO, &S.DNA, &S.RNA, &S.CH, &S.NST, &S.PST };
        for (int q = 0; q < 6; ++q) { if (!cols[q]) return PI_ERR_ARG; cp(*dst[q], cols[q]); }
        for (dvec* v : { &S.Sz, &S.Bm, &S.Cq, &S.Nq, &S.Pq }) v->assign(C, 0.0);
    } else {
    cp(S.Sz, in->Sz); cp(S.Bm, in->Bm);
    for (auto pr : { std::make_pair(&S.Cq, in->Cq), std::make_pair(&S.Nq, in->Nq), std::make_pair(&S.Pq, in->Pq) }) {
        if (pr.second) cp(*pr.first, pr.second);
        else if (S.carbon || S.iron) pr.first->assign(C, 0.0);
        else return PI_ERR_ARG;
    }
    }
    cp(S.Chl, in->Chl); cp(S.gen, in->gen); cp(S.age, in->age);
    S.ac.assign(in->ac, in->ac + C);
    cp(S.graz, in->graz); cp(S.mort, in->mort); cp(S.dvid, in->dvid);
    if (S.carbon) { if (in->Bd) cp(S.Bd, in->Bd); else S.Bd.assign(C, 0.0); }
    if (in->ptc) cp(S.ptc, in->ptc); else S.ptc.assign(C, 0.0);
    if (S.iron) {
        const double* cols[8] = { in->CH, in->qNO3, in->qNH4, in->qP, in->qFe, in->qFePS, in->qFeNR, in->qFeNF };
        dvec* dst[8] = { &S.CH, &S.qNO3, &S.qNH4, &S.qP, &S.qFe, &S.qFePS, &S.qFeNR, &S.qFeNF };
        for (int q = 0; q < 8; ++q) { if (!cols[q]) return PI_ERR_ARG; cp(*dst[q], cols[q]); }
        if (in->exEn) cp(S.exEn, in->exEn); else S.exEn.assign(C, 0.0);
        if (in->tdark) cp(S.tdark, in->tdark); else S.tdark.assign(C, 0.0);
    }
    return PI_OK;
}

int orc_get_individuals(orc_model* m, int32_t sp, pi_individuals* out) {
    if (!m || sp < 0 || sp >= m->nsp || !out) return PI_ERR_ARG;
    Species& S = m->sp[sp];
    auto cp = [&](double* d, const dvec& s) { if (d) std::copy(s.begin(), s.end(), d); };
    auto ci = [&](int64_t* d, const std::vector<int64_t>& s) { if (d) std::copy(s.begin(), s.end(), d); };
    cp(out->x, S.x); cp(out->y, S.y); cp(out->z, S.z);
    ci(out->xi, S.xi); ci(out->yi, S.yi); ci(out->zi, S.zi);
    cp(out->Sz, S.Sz); cp(out->Bm, S.Bm); cp(out->Cq, S.Cq); cp(out->Nq, S.Nq); cp(out->Pq, S.Pq);
    cp(out->Chl, S.Chl); cp(out->gen, S.gen); cp(out->age, S.age);
    if (out->ac) std::copy(S.ac.begin(), S.ac.end(), out->ac);
    cp(out->graz, S.graz); cp(out->mort, S.mort); cp(out->dvid, S.dvid);
    if (S.carbon) cp(out->Bd, S.Bd);
    if (S.macro) {
        cp(out->PRO, S.PRO); cp(out->DNA, S.DNA); cp(out->RNA, S.RNA);
        cp(out->CH, S.CH); cp(out->NST, S.NST); cp(out->PST, S.PST);
    }
    cp(out->ptc, S.ptc);
    if (S.iron) {
        cp(out->CH, S.CH); cp(out->qNO3, S.qNO3); cp(out->qNH4, S.qNH4); cp(out->qP, S.qP); cp(out->qFe, S.qFe);
        cp(out->qFePS, S.qFePS); cp(out->qFeNR, S.qFeNR); cp(out->qFeNF, S.qFeNF); cp(out->exEn, S.exEn);
        cp(out->tdark, S.tdark);
    }
    return PI_OK;
}

/* abiotic_setup / Palat / max_candidates of PlanktonModel (models.jl:99-146) */
int orc_set_abiotics(orc_model* m, int32_t nsa, const pi_abiotic_params* params, int32_t n_intac, const int32_t* intac,
                     int32_t n_release, const int32_t* release, int32_t max_candidates, const double* max_ptc) {
    if (!m || nsa < 1 || !params || max_candidates < 1 || !max_ptc || n_intac < 0 || n_release < 0 ||
        (n_intac && !intac) || (n_release && !release) || !m->ab.empty()) return PI_ERR_ARG;
    for (int32_t q = 0; q < n_intac + n_release; ++q) {
        const int32_t* pr = q < n_intac ? intac + 2 * q : release + 2 * (q - n_intac);
        if (pr[0] < 0 || pr[0] >= m->nsp || pr[1] < 0 || pr[1] >= nsa) return PI_ERR_ARG;
    }
    const size_t C = (size_t)m->C;
    m->ab.resize((size_t)nsa);
    for (int32_t a = 0; a < nsa; ++a) {
        Abiotic& A = m->ab[a];
        A.p = params[a];
        for (dvec* v : { &A.x, &A.y, &A.z }) v->assign(C, 0.0);
        A.xi.assign(C, 0); A.yi.assign(C, 0); A.zi.assign(C, 0);
        A.ac.assign(C, 0);
        A.d_num.assign(m->g.G, 0.0);
    }
    for (int32_t q = 0; q < n_intac; ++q) m->pal_intac.emplace_back(intac[2 * q], intac[2 * q + 1]);
    for (int32_t q = 0; q < n_release; ++q) m->pal_release.emplace_back(release[2 * q], release[2 * q + 1]);
    m->maxc = max_candidates;
    m->max_ptc.assign(max_ptc, max_ptc + m->nsp);
    m->intac.assign((size_t)max_candidates * C, 0);
    return PI_OK;
}

int orc_set_abiotic_particles(orc_model* m, int32_t sa, const pi_abiotic_particles* in) {
    if (!m || sa < 0 || sa >= (int32_t)m->ab.size() || !in || !in->x || !in->y || !in->z || !in->ac) return PI_ERR_ARG;
    Abiotic& A = m->ab[sa];
    const size_t C = (size_t)m->C;
    A.x.assign(in->x, in->x + C); A.y.assign(in->y, in->y + C); A.z.assign(in->z, in->z + C);
    A.ac.assign(in->ac, in->ac + C);
    for (auto pr : { std::make_pair(&A.xi, in->xi), std::make_pair(&A.yi, in->yi), std::make_pair(&A.zi, in->zi) }) {
        if (pr.second) pr.first->assign(pr.second, pr.second + C);
        else pr.first->assign(C, 0);
    }
    return PI_OK;
}

int orc_get_abiotic_particles(orc_model* m, int32_t sa, pi_abiotic_particles* out) {
    if (!m || sa < 0 || sa >= (int32_t)m->ab.size() || !out) return PI_ERR_ARG;
    const Abiotic& A = m->ab[sa];
    auto cp = [&](double* d, const dvec& s) { if (d) std::copy(s.begin(), s.end(), d); };
    auto ci = [&](int64_t* d, const std::vector<int64_t>& s) { if (d) std::copy(s.begin(), s.end(), d); };
    cp(out->x, A.x); cp(out->y, A.y); cp(out->z, A.z);
    ci(out->xi, A.xi); ci(out->yi, A.yi); ci(out->zi, A.zi);
    if (out->ac) std::copy(A.ac.begin(), A.ac.end(), out->ac);
    return PI_OK;
}

int orc_count_abiotic(orc_model* m, int32_t sa, int64_t* n) {
    if (!m || sa < 0 || sa >= (int32_t)m->ab.size() || !n) return PI_ERR_ARG;
    int64_t c = 0;
    for (uint8_t a : m->ab[sa].ac) c += a;
    *n = c;
    return PI_OK;
}

int orc_set_abiotic_bc(orc_model* m, int32_t sa, int32_t face, int32_t kind, const double* values, int64_t nt) {
    if (!m || sa < 0 || sa >= (int32_t)m->ab.size() || face < 0 || face > 5 || kind < 0 || kind > 3) return PI_ERR_ARG;
    const Grid& g = m->g;
    FluxBC& b = m->ab[sa].bc[face];
    b.kind = kind; b.nt = nt; b.v.clear();
    size_t n1 = face <= PI_EAST ? g.Ny : g.Nx, n2 = face <= PI_NORTH ? g.Nz : g.Ny;
    size_t n = kind == PI_BC_CONST ? 1 : kind == PI_BC_ARRAY2D ? n1 * n2 : kind == PI_BC_ARRAY3D ? n1 * n2 * (size_t)nt : 0;
    if (n && !values) return PI_ERR_ARG;
    if (n) b.v.assign(values, values + n);
    return PI_OK;
}

/* Physiological rates of the last step (PS, VDOC, VNH4, VNO3, VPO4, ρChl, resp, BS, exu). */
int orc_get_rates(orc_model* m, int32_t sp, double* out9) {
    if (!m || sp < 0 || sp >= m->nsp || !out9) return PI_ERR_ARG;
    Species& S = m->sp[sp];
    const dvec* r[9] = { &S.PS, &S.VDOC, &S.VNH4, &S.VNO3, &S.VPO4, &S.rChl, &S.resp, &S.BS, &S.exu };
    for (int q = 0; q < 9; ++q) std::copy(r[q]->begin(), r[q]->end(), out9 + (size_t)q * m->C);
    return PI_OK;
}

int orc_set_tracer(orc_model* m, int32_t idx, const double* data) {
    if (!m || idx < 0 || idx >= PI_NTRACERS || !data) return PI_ERR_ARG;
    m->tr[idx].assign(data, data + m->g.G);
    return PI_OK;
}
int orc_get_tracer(orc_model* m, int32_t idx, double* out) {
    if (!m || idx < 0 || idx >= PI_NTRACERS || !out) return PI_ERR_ARG;
    std::copy(m->tr[idx].begin(), m->tr[idx].end(), out);
    return PI_OK;
}

/* Scratch fields for tests: 0 par, 1 Chl, 2 pop, 3..16 plk[0..13], 17..30 Gcs[0..13],
 * 31 u1, 32 v1, 33 w1, 34 u0, 35 temp. */
int orc_get_field(orc_model* m, int32_t which, double* out) {
    if (!m || !out) return PI_ERR_ARG;
    const dvec* f = nullptr;
    if (which == 0) f = &m->par; else if (which == 1) f = &m->Chl; else if (which == 2) f = &m->pop;
    else if (which >= 3 && which < 17) f = &m->plk[which - 3];
    else if (which >= 17 && which < 31) f = &m->Gcs[which - 17];
    else if (which == 31) f = &m->u1; else if (which == 32) f = &m->v1; else if (which == 33) f = &m->w1;
    else if (which == 34) f = &m->u0; else if (which == 35) f = &m->temp;
    if (!f) return PI_ERR_ARG;
    std::copy(f->begin(), f->end(), out);
    return PI_OK;
}

/* vel_copy!, Simulation/utils.jl:5-34 */
int orc_set_velocity(orc_model* m, const double* u, const double* v, const double* w) {
    if (!m || !u || !v || !w) return PI_ERR_ARG;
    const Grid& g = m->g;
    int ex = g.tx == PI_BOUNDED, ey = g.ty == PI_BOUNDED, ez = g.tz == PI_BOUNDED;
    auto copy_in = [&](dvec& f, const double* s, int nx, int ny, int nz) {
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
            f[g.id(i + g.Hx, j + g.Hy, k + g.Hz)] = s[(size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1))];
    };
    copy_in(m->u1, u, g.Nx + ex, g.Ny, g.Nz);
    copy_in(m->v1, v, g.Nx, g.Ny + ey, g.Nz);
    copy_in(m->w1, w, g.Nx, g.Ny, g.Nz + ez);
    fill_halo_u(g, m->u1); fill_halo_v(g, m->v1); fill_halo_w(g, m->w1);
    return PI_OK;
}

int orc_set_velocity0(orc_model* m, const double* u, const double* v, const double* w) {
    if (!m) return PI_ERR_ARG;
    dvec su = m->u1, sv = m->v1, sw = m->w1;
    int r = orc_set_velocity(m, u, v, w);
    std::swap(m->u0, m->u1); std::swap(m->v0, m->v1); std::swap(m->w0, m->w1);
    m->u1 = su; m->v1 = sv; m->w1 = sw;
    return r;
}

int orc_set_PARF(orc_model* m, const double* parf) {
    if (!m || !parf) return PI_ERR_ARG;
    m->PARF.assign(parf, parf + (size_t)m->g.Nx * m->g.Ny);
    return PI_OK;
}

int orc_set_temp(orc_model* m, const double* temp) {   /* copy_interior!, Simulation/utils.jl:13-15 */
    if (!m || !temp) return PI_ERR_ARG;
    const Grid& g = m->g;
    for (int k = 1; k <= g.Nz; ++k) for (int j = 1; j <= g.Ny; ++j) for (int i = 1; i <= g.Nx; ++i)
        m->temp[g.id(i + g.Hx, j + g.Hy, k + g.Hz)] = temp[(size_t)(i - 1) + (size_t)g.Nx * ((size_t)(j - 1) + (size_t)g.Ny * (size_t)(k - 1))];
    return PI_OK;
}

int orc_set_flux_bc(orc_model* m, int32_t tracer, int32_t face, int32_t kind, const double* values, int64_t nt) {
    if (!m || tracer < 0 || tracer >= PI_NTRACERS || face < 0 || face > 5 || kind < 0 || kind > 3) return PI_ERR_ARG;
    const Grid& g = m->g;
    FluxBC& b = m->bc[tracer][face];
    b.kind = kind; b.nt = nt; b.v.clear();
    size_t n1 = face <= PI_EAST ? g.Ny : g.Nx, n2 = face <= PI_NORTH ? g.Nz : g.Ny;
    size_t n = kind == PI_BC_CONST ? 1 : kind == PI_BC_ARRAY2D ? n1 * n2 : kind == PI_BC_ARRAY3D ? n1 * n2 * (size_t)nt : 0;
    if (n && !values) return PI_ERR_ARG;
    if (n) b.v.assign(values, values + n);
    return PI_OK;
}

/* TimeStep!, Model/time_step.jl:12-180 */
int orc_time_step(orc_model* m, double dT) {
    if (!m) return PI_ERR_ARG;
    const Grid& g = m->g;
    m->iteration = m->iteration + 1;
    m->t = (double)m->iteration * dT;
    #pragma omp parallel for schedule(static)
    for (size_t q = 0; q < g.G; ++q) {                                           /* :17-19 */
        m->uh[q] = (m->u0[q] + m->u1[q]) * 0.5;
        m->vh[q] = (m->v0[q] + m->v1[q]) * 0.5;
        m->wh[q] = (m->w0[q] + m->w1[q]) * 0.5;
    }
    for (int n = 0; n < PI_NTRACERS; ++n) zero(m->plk[n]);                        /* :21-22 */
    zero(m->Chl);
    bool ok = true;
    if (int st = abiotic_update(m, dT)) return st;                                 /* :24-39 */
    if (m->bgc.shared_graz == 1.0) {
        zero(m->pop);
        for (int s = 0; s < m->nsp; ++s) {
            particle_advection(m, m->sp[s], dT);
            particle_diffusion(m, m->sp[s], s, dT);
            find_inds(m, m->sp[s]);
            acc_chl(m, m->sp[s]);
            acc_counts(m, m->sp[s]);
        }
        for (int ki = 1; ki <= g.Nz; ++ki) calc_par(m, ki);
        for (int s = 0; s < m->nsp && ok; ++s) {
            find_NPT(m, m->sp[s]);
            ok = plankton_update(m, m->sp[s], s, dT, m->t);
        }
    } else {
        for (int s = 0; s < m->nsp; ++s) {
            particle_advection(m, m->sp[s], dT);
            particle_diffusion(m, m->sp[s], s, dT);
            find_inds(m, m->sp[s]);
            acc_chl(m, m->sp[s]);
        }
        for (int ki = 1; ki <= g.Nz; ++ki) calc_par(m, ki);
        for (int s = 0; s < m->nsp && ok; ++s) {
            zero(m->pop);
            acc_counts(m, m->sp[s]);
            find_NPT(m, m->sp[s]);
            ok = plankton_update(m, m->sp[s], s, dT, m->t);
        }
    }
    if (!ok) return PI_ERR_CAPACITY;
    if (int st = abiotic_exchange(m, dT)) return st;                               /* :120-158 */
    tracer_update(m, dT);
    for (size_t q = 0; q < g.G; ++q) m->d_PAR[q] += m->par[q];                  /* :167 */
    for (int n = 0; n < PI_NTRACERS; ++n)                                          /* :168-172 */
        if (m->tr_mask & (1u << n))
            for (size_t q = 0; q < g.G; ++q) m->d_tr[n][q] += m->tr[n][q];
    m->u0 = m->u1; m->v0 = m->v1; m->w0 = m->w1;                                  /* :174-177 */
    m->par0 = m->par;
    if (m->err_flags & ERR_DOMAIN) { m->err = "an individual left the halo-padded grid"; return PI_ERR_DOMAIN; }
    return PI_OK;
}

int orc_get_time(orc_model* m, int64_t* it, double* t) {
    if (!m) return PI_ERR_ARG;
    if (it) *it = m->iteration;
    if (t) *t = m->t;
    return PI_OK;
}
int orc_set_time(orc_model* m, int64_t it, double t) { if (!m) return PI_ERR_ARG; m->iteration = it; m->t = t; return PI_OK; }

int orc_count_active(orc_model* m, int32_t sp, int64_t* n) {
    if (!m || sp < 0 || sp >= m->nsp || !n) return PI_ERR_ARG;
    int64_t c = 0;
    for (uint8_t a : m->sp[sp].ac) c += a;
    *n = c;
    return PI_OK;
}

/* PlanktonDiagnostics(model; tracer, phytoplankton) optional fields: enabling clears them. */
int orc_set_diags(orc_model* m, uint32_t tr_mask, uint32_t proc_mask) {
    const int nproc = m ? (m->sp[0].iron ? (int)PI_NIPROC : m->sp[0].macro ? (int)PI_NMPROC
                           : m->sp[0].carbon ? (int)PI_NCPROC : (int)PI_NPROC) : 0;
    if (!m || tr_mask >> PI_NTRACERS || (nproc < 32 && proc_mask >> nproc)) return PI_ERR_ARG;
    m->tr_mask = tr_mask; m->proc_mask = proc_mask;
    m->d_tr.assign(tr_mask ? PI_NTRACERS : 0, dvec(tr_mask ? m->g.G : 0, 0.0));
    for (Species& S : m->sp) S.d_proc.assign(proc_mask ? nproc : 0, dvec(proc_mask ? m->g.G : 0, 0.0));
    return PI_OK;
}

int orc_get_diag(orc_model* m, int32_t kind, int32_t sp, double* out) {
    if (!m || !out) return PI_ERR_ARG;
    const dvec* f = nullptr;
    if (kind == PI_DIAG_PAR) f = &m->d_PAR;
    else if (kind >= PI_DIAG_TRACER && kind < PI_DIAG_TRACER + PI_NTRACERS) {
        if (!(m->tr_mask & (1u << (kind - PI_DIAG_TRACER)))) return PI_ERR_ARG;
        f = &m->d_tr[kind - PI_DIAG_TRACER];
    } else if (kind >= PI_DIAG_PROC && kind < PI_DIAG_PROC + PI_NIPROC) {
        if (sp < 0 || sp >= m->nsp || !(m->proc_mask & (1u << (kind - PI_DIAG_PROC)))) return PI_ERR_ARG;
        if ((size_t)(kind - PI_DIAG_PROC) >= m->sp[sp].d_proc.size()) return PI_ERR_ARG;
        f = &m->sp[sp].d_proc[kind - PI_DIAG_PROC];
    } else if (kind == PI_DIAG_ABIO_NUM) {
        if (sp < 0 || sp >= (int32_t)m->ab.size()) return PI_ERR_ARG;
        f = &m->ab[sp].d_num;
    } else {
        if (sp < 0 || sp >= m->nsp) return PI_ERR_ARG;
        Species& S = m->sp[sp];
        f = kind == PI_DIAG_NUM ? &S.d_num : kind == PI_DIAG_GRAZ ? &S.d_graz
          : kind == PI_DIAG_MORT ? &S.d_mort : kind == PI_DIAG_DVID ? &S.d_dvid
          : kind == PI_DIAG_PTC ? &S.d_ptc : nullptr;
    }
    if (!f) return PI_ERR_ARG;
    std::copy(f->begin(), f->end(), out);
    return PI_OK;
}

int orc_last_error(orc_model* m, char* buf, size_t len) {
    const std::string& e = m ? m->err : g_create_err;
    if (buf && len) { size_t n = std::min(len - 1, e.size()); memcpy(buf, e.c_str(), n); buf[n] = 0; }
    return PI_OK;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Numeric primitives exposed for tests of the shared header. */
double orc_exp(double x) { return pi_exp(x); }
double orc_pow_int(double x, int n) { return pi_pow_int(x, n); }
double orc_log(double x) { return pi_log(x); }
double orc_pow(double x, double y) { return pi_pow(x, y); }
void orc_draw3(uint64_t seed, uint32_t it, uint32_t sp, uint32_t purpose, uint32_t slot, double* r) {
    pi_draw3(seed, it, sp, purpose, slot, &r[0], &r[1], &r[2]);
}

}  // extern "C"
