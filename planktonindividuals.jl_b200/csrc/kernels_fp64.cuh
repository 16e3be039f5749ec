// FP64 plain-form kernels of the model time step (the abiotic particles' own kernels are in
// kernels_abiotic.cuh).
//
// Every arithmetic expression below is written in the operation order of the reference Julia
// code it cites, and the library is compiled with -fmad=false, so each result is the same IEEE
// double the CPU oracle produces. Scatters that the reference does with float atomics are done
// here by binning individuals per cell (sorted by species then slot, the order of a sequential
// reference run) and summing each cell's contributions in that order.
#pragma once

#include "pib200_internal.h"

namespace pib {

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t bit) { atomicOr(err, bit); }

__device__ __forceinline__ int clamp_idx(long long v, int lo, int hi, uint32_t* err) {
    if (v < lo) { set_err(err, PI_DEVERR_DOMAIN); return lo; }
    if (v > hi) { set_err(err, PI_DEVERR_DOMAIN); return hi; }
    return (int)v;
}

__device__ __forceinline__ double dzF1(const DGrid& g, int k) { return g.dzF[k - 1]; }
__device__ __forceinline__ double dzC1(const DGrid& g, int k) { return g.dzC[k - 1]; }
// Grids/areas_volumes_spacings.jl:9-38 with 1-based halo-inclusive indices. LL = false: a
// RectilinearGrid, whose metrics are formed from Δx, Δy and dzF in the reference's operation order;
// LL = true: a LatLonGrid, whose arrays are read. The kernels that use them are instantiated for
// both, so the RectilinearGrid code reads no metric array.
__device__ __forceinline__ int gidx2(const DGrid& g, int i, int j) { return (i - 1) + g.Gx * (j - 1); }
__device__ __forceinline__ long long gidx3l(const DGrid& g, int i, int j, int k) {
    return (i - 1) + (long long)g.Gx * ((j - 1) + (long long)g.Gy * (k - 1));
}
template <bool LL> __device__ __forceinline__ double vol(const DGrid& g, int i, int j, int k) {
    return LL ? g.mVol[gidx3l(g, i, j, k)] : g.dx * g.dy * dzF1(g, k);
}
template <bool LL> __device__ __forceinline__ double Axm(const DGrid& g, int i, int j, int k) {
    return LL ? g.mAx[gidx3l(g, i, j, k)] : g.dy * dzF1(g, k);
}
template <bool LL> __device__ __forceinline__ double Aym(const DGrid& g, int i, int j, int k) {
    return LL ? g.mAy[gidx3l(g, i, j, k)] : g.dx * dzF1(g, k);
}
template <bool LL> __device__ __forceinline__ double Azm(const DGrid& g, int i, int j) { return LL ? g.mAz[gidx2(g, i, j)] : g.dx * g.dy; }
template <bool LL> __device__ __forceinline__ double dxCm(const DGrid& g, int i, int j) { return LL ? g.mdxC[gidx2(g, i, j)] : g.dx; }
template <bool LL> __device__ __forceinline__ double dyCm(const DGrid& g, int i, int j) { return LL ? g.mdyC[gidx2(g, i, j)] : g.dy; }
template <bool LL> __device__ __forceinline__ double dxFm(const DGrid& g, int i, int j) { return LL ? g.mdxF[gidx2(g, i, j)] : g.dx; }
template <bool LL> __device__ __forceinline__ double dyFm(const DGrid& g, int i, int j) { return LL ? g.mdyF[gidx2(g, i, j)] : g.dy; }
// volume of a RectilinearGrid cell at level k (pi_tracer_advection_noalloc takes only these)
__device__ __forceinline__ double vol(const DGrid& g, int k) { return g.dx * g.dy * dzF1(g, k); }
__device__ __forceinline__ int lmask(const DGrid& g, int i, int j, int k) {
    return g.all_water ? 1 : (int)g.lm[gidx(g, i, j, k)];
}

// ------------------------------------------------------------------------------------------
// (a) RK4 advection + random-walk diffusion + cell lookup
//     particle_advection.jl:2-56, particle_advection_kernels.jl:2-50, interpolation.jl:3-83,
//     particle_diffusion.jl:2-33, Individuals/utils.jl:2-7
// ------------------------------------------------------------------------------------------

// particle_boundary_condition, particle_advection_kernels.jl:2-11
__device__ __forceinline__ double bc_pos(double x, double xr, int topo) {
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

// Trilinear interpolation in grid-index units (u_itpl/v_itpl/w_itpl). HALF = 1 samples
// vel½ = (vel₀ + vel₁) * 0.5 corner by corner, which is the array time_step.jl:17-19 builds.
template <int COMP, int HALF, bool LL>
__device__ __forceinline__ double itpl(const DGrid& g, const double* __restrict__ f0,
                                       const double* __restrict__ f1, double x, double y,
                                       double z, int ac, uint32_t* err) {
    double fx = jl_mulb(COMP == 0 ? x + 1.0 : x + 0.5, ac);
    double fy = jl_mulb(COMP == 1 ? y + 1.0 : y + 0.5, ac);
    double fz = jl_mulb(COMP == 2 ? z + 1.0 : z + 0.5, ac);
    double xd = jl_mod1(fx), yd = jl_mod1(fy), zd = jl_mod1(fz);
    int i = clamp_idx(jl_trunc(fx) + g.Hx, 1, g.Gx - 1, err);
    int j = clamp_idx(jl_trunc(fy) + g.Hy, 1, g.Gy - 1, err);
    int k = clamp_idx(jl_trunc(fz) + g.Hz, 1, g.Gz - 1, err);
    int q000 = gidx(g, i, j, k);
    int sx = 1, sy = g.Gx, sz = g.Gx * g.Gy;
    auto F = [&](int q) -> double { return HALF ? (f0[q] + f1[q]) * 0.5 : f0[q]; };
    double c000 = F(q000), c001 = F(q000 + sz), c010 = F(q000 + sy), c011 = F(q000 + sy + sz);
    double c100 = F(q000 + sx), c101 = F(q000 + sx + sz), c110 = F(q000 + sx + sy);
    double c111 = F(q000 + sx + sy + sz);
    double w000 = (1.0 - xd) * (1.0 - yd) * (1.0 - zd);
    double w001 = (1.0 - xd) * (1.0 - yd) * zd;
    double w010 = (1.0 - xd) * yd * (1.0 - zd);
    double w011 = (1.0 - xd) * yd * zd;
    double w100 = xd * (1.0 - yd) * (1.0 - zd);
    double w101 = xd * (1.0 - yd) * zd;
    double w110 = xd * yd * (1.0 - zd);
    double w111 = xd * yd * zd;
    // each corner divided by ΔxC, ΔyC or ΔzC at that corner (interpolation.jl:23-50)
    auto D = [&](int a, int b, int c) -> double {
        return COMP == 0 ? dxCm<LL>(g, i + a, j + b) : COMP == 1 ? dyCm<LL>(g, i + a, j + b) : dzC1(g, k + c);
    };
    return w000 * c000 / D(0, 0, 0) + w001 * c001 / D(0, 0, 1) + w010 * c010 / D(0, 1, 0) + w011 * c011 / D(0, 1, 1)
         + w100 * c100 / D(1, 0, 0) + w101 * c101 / D(1, 0, 1) + w110 * c110 / D(1, 1, 0) + w111 * c111 / D(1, 1, 1);
}


// vel½ = (vel₀ + vel₁) * 0.5 (time_step.jl:17-19), once per step for the three components.
__global__ void k_velhalf(long long G, const double* __restrict__ u0, const double* __restrict__ v0,
                          const double* __restrict__ w0, const double* __restrict__ u1,
                          const double* __restrict__ v1, const double* __restrict__ w1,
                          double* __restrict__ uh, double* __restrict__ vh, double* __restrict__ wh,
                          const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < G; q += (long long)gridDim.x * blockDim.x) {
        uh[q] = (u0[q] + u1[q]) * 0.5;
        vh[q] = (v0[q] + v1[q]) * 0.5;
        wh[q] = (w0[q] + w1[q]) * 0.5;
    }
}

struct VelPtrs { const double *u0, *v0, *w0, *uh, *vh, *wh, *u1, *v1, *w1; };

// RK4 + diffusion + find_inds! of one active particle at `slot` of the columns x, y, z, cell of P
// (a phytoplankton species, SpcDev, or an abiotic species, AbioDev, whose steps are the same
// kernels, time_step.jl:29-38); the diffusion draw is keyed by (dsp, purpose). BIN: writes the
// binning key and count of a phytoplankton individual.
template <bool LL, bool BIN = true, class PV>
__device__ __forceinline__ void particle_step(const DGrid& g, const PV& P, uint32_t dsp, uint32_t purpose, long long slot,
                                              long long gid, double dT, uint64_t seed, uint32_t iter,
                                              const VelPtrs& vel, double kappa_h, double kappa_v,
                                              uint32_t* __restrict__ cnt, uint32_t* __restrict__ key,
                                              uint32_t* err) {
    const int ac = 1;
    int oxi, oyi, ozi;
    unpack_cell(g, P.cell[slot], oxi, oyi, ozi);
    int kdz = clamp_idx((long long)ozi + g.Hz, 1, g.Gz, err);   // ΔzC at the stored zi + Hz
    const double X = P.x[slot], Y = P.y[slot], Z = P.z[slot];
    const double NX = (double)g.Nx, NY = (double)g.Ny, NZ = (double)g.Nz;
    // stage 1 at vel₀
    double u1 = jl_mulb(itpl<0, 0, LL>(g, vel.u0, vel.u0, X, Y, Z, ac, err), ac);
    double v1 = jl_mulb(itpl<1, 0, LL>(g, vel.v0, vel.v0, X, Y, Z, ac, err), ac);
    double w1 = jl_mulb(itpl<2, 0, LL>(g, vel.w0, vel.w0, X, Y, Z, ac, err), ac);
    double u2 = u1, v2 = v1, w2 = w1;
    double vx = X + jl_mulb(0.5 * u1 * dT, ac);
    double vy = Y + jl_mulb(0.5 * v1 * dT, ac);
    double vz = Z - jl_mulb(0.5 * w1 * dT, ac);
    vx = jl_mulb(bc_pos(vx, NX, g.tx), ac); vy = jl_mulb(bc_pos(vy, NY, g.ty), ac); vz = jl_mulb(bc_pos(vz, NZ, g.tz), ac);
    // stage 2 at vel½
    u1 = jl_mulb(itpl<0, 0, LL>(g, vel.uh, vel.uh, vx, vy, vz, ac, err), ac);
    v1 = jl_mulb(itpl<1, 0, LL>(g, vel.vh, vel.vh, vx, vy, vz, ac, err), ac);
    w1 = jl_mulb(itpl<2, 0, LL>(g, vel.wh, vel.wh, vx, vy, vz, ac, err), ac);
    u2 = u2 + u1 * 2.0; v2 = v2 + v1 * 2.0; w2 = w2 + w1 * 2.0;
    vx = X + jl_mulb(0.5 * u1 * dT, ac);
    vy = Y + jl_mulb(0.5 * v1 * dT, ac);
    vz = Z - jl_mulb(0.5 * w1 * dT, ac);
    vx = jl_mulb(bc_pos(vx, NX, g.tx), ac); vy = jl_mulb(bc_pos(vy, NY, g.ty), ac); vz = jl_mulb(bc_pos(vz, NZ, g.tz), ac);
    // stage 3 at vel½
    u1 = jl_mulb(itpl<0, 0, LL>(g, vel.uh, vel.uh, vx, vy, vz, ac, err), ac);
    v1 = jl_mulb(itpl<1, 0, LL>(g, vel.vh, vel.vh, vx, vy, vz, ac, err), ac);
    w1 = jl_mulb(itpl<2, 0, LL>(g, vel.wh, vel.wh, vx, vy, vz, ac, err), ac);
    u2 = u2 + u1 * 2.0; v2 = v2 + v1 * 2.0; w2 = w2 + w1 * 2.0;
    vx = X + jl_mulb(1.0 * u1 * dT, ac);
    vy = Y + jl_mulb(1.0 * v1 * dT, ac);
    vz = Z - jl_mulb(1.0 * w1 * dT, ac);
    vx = jl_mulb(bc_pos(vx, NX, g.tx), ac); vy = jl_mulb(bc_pos(vy, NY, g.ty), ac); vz = jl_mulb(bc_pos(vz, NZ, g.tz), ac);
    // stage 4 at vel₁
    u1 = jl_mulb(itpl<0, 0, LL>(g, vel.u1, vel.u1, vx, vy, vz, ac, err), ac);
    v1 = jl_mulb(itpl<1, 0, LL>(g, vel.v1, vel.v1, vx, vy, vz, ac, err), ac);
    w1 = jl_mulb(itpl<2, 0, LL>(g, vel.w1, vel.w1, vx, vy, vz, ac, err), ac);
    u2 = u2 + u1; v2 = v2 + v1; w2 = w2 + w1;
    u2 = u2 / 6.0; v2 = v2 / 6.0; w2 = w2 / 6.0;
    double x = X + jl_mulb(1.0 * u2 * dT, ac);
    double y = Y + jl_mulb(1.0 * v2 * dT, ac);
    double z = Z - jl_mulb(1.0 * w2 * dT, ac);
    x = jl_mulb(bc_pos(x, NX, g.tx), ac); y = jl_mulb(bc_pos(y, NY, g.ty), ac); z = jl_mulb(bc_pos(z, NZ, g.tz), ac);
    // diffusion: rnd ∈ [0,1) → (rnd - 0.5) * 2 → · √(κΔT) / Δ
    double r0, r1, r2;
    pi_draw3(seed, iter, dsp, purpose, (uint32_t)slot, &r0, &r1, &r2);
    r0 = (r0 - 0.5) * 2.0; r1 = (r1 - 0.5) * 2.0; r2 = (r2 - 0.5) * 2.0;
    // ΔxC/ΔyC at (xi+Hx, yi+Hy) of the stored indices (particle_diffusion.jl:4-5); the reference
    // reads past the metric array there when x = Nx exactly, which is held at the last column here
    const int dxi = min(max(oxi + g.Hx, 1), g.Gx), dyi = min(max(oyi + g.Hy, 1), g.Gy);
    r0 = r0 * sqrt(kappa_h * dT) / dxCm<LL>(g, dxi, dyi);
    r1 = r1 * sqrt(kappa_h * dT) / dyCm<LL>(g, dxi, dyi);
    r2 = r2 * sqrt(kappa_v * dT) / dzC1(g, kdz);
    x = x + jl_mulb(r0, ac); y = y + jl_mulb(r1, ac); z = z + jl_mulb(r2, ac);
    x = jl_mulb(bc_pos(x, NX, g.tx), ac); y = jl_mulb(bc_pos(y, NY, g.ty), ac); z = jl_mulb(bc_pos(z, NZ, g.tz), ac);
    P.x[slot] = x; P.y[slot] = y; P.z[slot] = z;
    // find_inds!
    int xi = clamp_idx(jl_trunc(jl_mulb(x + 1.0, ac)) + g.Hx, 1, g.Gx, err);
    int yi = clamp_idx(jl_trunc(jl_mulb(y + 1.0, ac)) + g.Hy, 1, g.Gy, err);
    int zi = clamp_idx(jl_trunc(jl_mulb(z + 1.0, ac)) + g.Hz, 1, g.Gz, err);
    P.cell[slot] = pack_cell(g, xi, yi, zi);
    if (BIN) {
        int c = gidx(g, xi, yi, zi);
        key[gid] = (uint32_t)c;
        atomicAdd(&cnt[c], 1u);
    }
}

// Slot-order pass over every (species, slot): inactive slots (every stage multiplies by ac, so
// their positions end as zeros and their cell is (Hx, Hy, Hz)), and active individuals that were
// not binned in the previous step (new daughters, uploaded state). The others are moved by
// k_particles_sorted in cell order.
template <bool LL>
__global__ void k_particles(DGrid g, const SpcDev* __restrict__ spc, int nsp, long long C,
                            double dT, uint64_t seed, uint32_t iter, VelPtrs vel,
                            double kappa_h, double kappa_v, uint32_t* __restrict__ cnt,
                            uint32_t* __restrict__ key, uint32_t sentinel, uint32_t* err) {
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nsp * C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    int s = (int)(gid / C);
    long long slot = gid - (long long)s * C;
    const SpcDev& P = spc[s];
    if (!(P.flags[slot] & FL_AC)) {
        int oxi, oyi, ozi;
        unpack_cell(g, P.cell[slot], oxi, oyi, ozi);
        clamp_idx((long long)ozi + g.Hz, 1, g.Gz, err);
        if (P.x[slot] != 0.0) P.x[slot] = 0.0;
        if (P.y[slot] != 0.0) P.y[slot] = 0.0;
        if (P.z[slot] != 0.0) P.z[slot] = 0.0;
        P.cell[slot] = pack_cell(g, g.Hx, g.Hy, g.Hz);
        key[gid] = sentinel;
        return;
    }
    if (P.stat[slot] & ST_AC0) return;                // moved by k_particles_sorted
    particle_step<LL>(g, P, (uint32_t)s, PI_DRAW_DIFFUSION, slot, gid, dT, seed, iter, vel, kappa_h, kappa_v, cnt, key,
                      err);
}

// Cell-order pass: the individuals binned in the previous step (prev_sorted[0 .. off[G]), which
// were active then) that are still active. Neighbouring threads interpolate in neighbouring cells.
template <bool LL>
__global__ void k_particles_sorted(DGrid g, const SpcDev* __restrict__ spc, long long C,
                                   const uint32_t* __restrict__ prev_sorted,
                                   const uint32_t* __restrict__ prev_off, long long Gcells,
                                   double dT, uint64_t seed, uint32_t iter, VelPtrs vel,
                                   double kappa_h, double kappa_v, uint32_t* __restrict__ cnt,
                                   uint32_t* __restrict__ key, uint32_t* err) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (*err & PI_DEVERR_CAPACITY) return;
    if (p >= (long long)prev_off[Gcells]) return;
    uint32_t gd = prev_sorted[p];
    int s = (int)(gd / C);
    long long slot = gd - (long long)s * C;
    const SpcDev& P = spc[s];
    if (!(P.flags[slot] & FL_AC) || !(P.stat[slot] & ST_AC0)) return;
    particle_step<LL>(g, P, (uint32_t)s, PI_DRAW_DIFFUSION, slot, gd, dT, seed, iter, vel, kappa_h, kappa_v, cnt, key,
                      err);
}

// pos[gid] = position of gid in the cell-sorted entry list.
__global__ void k_setpos(const uint32_t* __restrict__ off, long long G,
                         const uint32_t* __restrict__ gid_sorted, int32_t* __restrict__ pos,
                         long long n, const uint32_t* err) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (*err & PI_DEVERR_CAPACITY) return;
    if (p >= n || p >= (long long)off[G]) return;
    pos[gid_sorted[p]] = (int32_t)p;
}

// ------------------------------------------------------------------------------------------
// PAR: calc_par! down each column (Individuals/utils.jl:55-63, time_step.jl:63-67) with the Chl
// of acc_chl! (utils.jl:33-36) summed per cell in species-then-slot order, and
// diags.tracer.PAR .+= par (time_step.jl:167).
// ------------------------------------------------------------------------------------------
template <bool LL>
__global__ void k_par(DGrid g, const SpcDev* __restrict__ spc, long long C,
                      const uint32_t* __restrict__ off, const uint32_t* __restrict__ gid_sorted,
                      double* __restrict__ PARF, const double* __restrict__ PARF_src,
                      double* __restrict__ par, double* __restrict__ diag_par, double kc, double kw,
                      const uint32_t* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y + 1;
    if (i > g.Nx) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    int f = (i - 1) + g.Nx * (j - 1);
    double parf = PARF_src[f];
    int ii = i + g.Hx, jj = j + g.Hy;
    for (int k = 1; k <= g.Nz; ++k) {
        int kk = k + g.Hz;
        int c = gidx(g, ii, jj, kk);
        double chl = 0.0;
        for (uint32_t p = off[c]; p < off[c + 1]; ++p) {
            uint32_t gd = gid_sorted[p];
            int s = (int)(gd / C);
            chl += spc[s].Chl[gd - (long long)s * C];
        }
        double atten = (chl / vol<LL>(g, ii, jj, kk) * kc + kw) * dzF1(g, kk);
        double e = pi_exp(-atten);
        double pv = parf * (1.0 - e) / atten;
        par[c] = pv;
        parf = parf * e;
        diag_par[c] = diag_par[c] + pv;
    }
    PARF[f] = parf;
}

// ------------------------------------------------------------------------------------------
// (e) grazing, mortality, division — plankton_update.jl:5-24, division_death.jl:2-77,
//     consume_loss.jl:17-26, Diagnostics/diagnostics_kernels.jl:4-7
// ------------------------------------------------------------------------------------------

// total_C/N/P_biomass (MacroMolecularMode/plankton_generation.jl:82-93)
__host__ __device__ __forceinline__ double m_totC(double PRO, double DNA, double RNA, double CH, double Chl) {
    return PRO + DNA + RNA + CH + Chl / F_CHL * 55.0;
}
__host__ __device__ __forceinline__ double m_totN(double PRO, double DNA, double RNA, double NST, double Chl,
                                                  const pi_macro_params& p) {
    return PRO * p.R_NC_PRO + DNA * p.R_NC_DNA + RNA * p.R_NC_RNA + NST + Chl / F_CHL * 4.0;
}
__host__ __device__ __forceinline__ double m_totP(double DNA, double RNA, double PST, const pi_macro_params& p) {
    return DNA * p.R_PC_DNA + RNA * p.R_PC_RNA + PST;
}

// Applies last step's grazing/mortality decisions, writes the loss contributions of the
// individuals lost, the division/free flags for the slot scan and the graz/mort/dvid diags.
// mode MODE_CARBON: CarbonMode losses (CarbonMode/consume_loss.jl:12-16), DOC and POC from Bm only;
// MODE_MACRO: MacroMolecularMode losses (MacroMolecularMode/consume_loss.jl:14-24) from the total
// C, N and P biomass (mp holds its R_NC_* and R_PC_* ratios).
__global__ void k_decide(DGrid g, SpcDev P, pi_quota_params p, pi_macro_params mp, pi_iron_params ip, long long C, int s,
                         const int32_t* __restrict__ pos, double* __restrict__ loss,
                         uint8_t* __restrict__ evk, unsigned long long* __restrict__ flag64,
                         double* __restrict__ d_graz, double* __restrict__ d_mort,
                         double* __restrict__ d_dvid, uint32_t* err, int mode) {
    long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    uint8_t f = P.flags[slot];
    int ac0 = f & FL_AC, gz = (f & FL_GRAZ) != 0, mt = (f & FL_MORT) != 0, dv = (f & FL_DVID) != 0;
    P.stat[slot] = ac0 ? ST_AC0 : 0;
    int ac1 = ac0 && !gz;          // inactivate!(plank, graz): ac &= isless(graz, 1)
    int ac2 = ac1 && !mt;          // inactivate!(plank, mort)
    int dv2 = dv && ac2;           // plank.dvid .*= plank.ac
    if (ac0) {
        int xi, yi, zi;
        unpack_cell(g, P.cell[slot], xi, yi, zi);
        int c = gidx(g, xi, yi, zi);
        if (gz) atomicAdd(&d_graz[c], 1.0);
        if (ac1 && mt) atomicAdd(&d_mort[c], 1.0);
        if (dv2) atomicAdd(&d_dvid[c], 1.0);
        long long e = pos[(long long)s * C + slot];
        uint8_t kind = gz ? 1 : (ac1 && mt) ? 2 : 0;
        evk[e] = kind;
        if (kind) {
            double fC = kind == 1 ? p.grazFracC : p.mortFracC;
            double fN = kind == 1 ? p.grazFracN : p.mortFracN;
            double fP = kind == 1 ? p.grazFracP : p.mortFracP;
            if (mode == MODE_IRON) {
                // IronEnergyMode/consume_loss.jl:17-32: NH4, NO3, DOC, DON, DOP, DFe, POC, PON, POP, PFe_bio
                double* L = loss + e * 10;
                const double fFe = kind == 1 ? ip.grazFracFe : ip.mortFracFe;
                const double Bm = P.Bm[slot], CH = P.CH[slot], qP = P.qP[slot];
                const double fe = P.qFe[slot] + P.qFePS[slot] + P.qFeNF[slot] + P.qFeNR[slot];
                L[0] = jl_mulb(P.qNH4[slot], 1) * 1.0;
                L[1] = jl_mulb(P.qNO3[slot], 1) * 1.0;
                L[2] = jl_mulb((Bm + CH) * fC, 1) * 1.0;
                L[3] = jl_mulb(Bm * ip.R_NC * fN, 1) * 1.0;
                L[4] = jl_mulb((Bm * ip.R_PC + qP) * fP, 1) * 1.0;
                L[5] = jl_mulb(fe * fFe, 1) * 1.0;
                L[6] = jl_mulb((Bm + CH) * (1.0 - fC), 1) * 1.0;
                L[7] = jl_mulb(Bm * ip.R_NC * (1.0 - fN), 1) * 1.0;
                L[8] = jl_mulb((Bm * ip.R_PC + qP) * (1.0 - fP), 1) * 1.0;
                L[9] = jl_mulb(fe * (1.0 - fFe), 1) * 1.0;
            } else {
            double* L = loss + e * 6;
            if (mode == MODE_CARBON) {
                const double Bm = P.Bm[slot];
                L[0] = jl_mulb(Bm * fC, 1) * 1.0;                     // DOC
                L[3] = jl_mulb(Bm * (1.0 - fC), 1) * 1.0;             // POC
                L[1] = 0.0; L[2] = 0.0; L[4] = 0.0; L[5] = 0.0;
            } else if (mode == MODE_MACRO) {
                const double tC = m_totC(P.PRO[slot], P.DNA[slot], P.RNA[slot], P.CH[slot], P.Chl[slot]);
                const double tN = m_totN(P.PRO[slot], P.DNA[slot], P.RNA[slot], P.NST[slot], P.Chl[slot], mp);
                const double tP = m_totP(P.DNA[slot], P.RNA[slot], P.PST[slot], mp);
                L[0] = jl_mulb(tC * fC, 1) * 1.0;                     // DOC
                L[1] = jl_mulb(tN * fN, 1) * 1.0;                     // DON
                L[2] = jl_mulb(tP * fP, 1) * 1.0;                     // DOP
                L[3] = jl_mulb(tC * (1.0 - fC), 1) * 1.0;             // POC
                L[4] = jl_mulb(tN * (1.0 - fN), 1) * 1.0;             // PON
                L[5] = jl_mulb(tP * (1.0 - fP), 1) * 1.0;             // POP
            } else {
            double Bm = P.Bm[slot], Cq = P.Cq[slot], Nq = P.Nq[slot], Pq = P.Pq[slot];
            L[0] = jl_mulb((Bm + Cq) * fC, 1) * 1.0;                  // DOC
            L[1] = jl_mulb((Bm * p.R_NC + Nq) * fN, 1) * 1.0;         // DON
            L[2] = jl_mulb((Bm * p.R_PC + Pq) * fP, 1) * 1.0;         // DOP
            L[3] = jl_mulb((Bm + Cq) * (1.0 - fC), 1) * 1.0;          // POC
            L[4] = jl_mulb((Bm * p.R_NC + Nq) * (1.0 - fN), 1) * 1.0; // PON
            L[5] = jl_mulb((Bm * p.R_PC + Pq) * (1.0 - fP), 1) * 1.0; // POP
            }
            }
        }
    }
    P.flags[slot] = (uint8_t)((ac2 ? FL_AC : 0) | (dv2 ? FL_DVID : 0));
    flag64[slot] = ((unsigned long long)dv2 << 32) | (unsigned long long)(!ac2);
}

// After the exclusive scan of flag64: the k-th divider (slot order) and the k-th free slot
// (findall(!ac), ascending) — get_tind!, Individuals/utils.jl:76-86. Checks capacity
// (plankton_update.jl:18-22).
__global__ void k_lists(const unsigned long long* __restrict__ flag64,
                        const unsigned long long* __restrict__ rank64, long long C,
                        int32_t* __restrict__ divlist, int32_t* __restrict__ freelist,
                        uint32_t* ndiv, uint32_t* err, int64_t* err_iter, int64_t iter,
                        uint32_t errbits = PI_DEVERR_CAPACITY) {
    long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    unsigned long long tot = rank64[C - 1] + flag64[C - 1];
    unsigned long long tdiv = tot >> 32, tfree = tot & 0xffffffffull;
    if (tdiv > tfree) {
        if (slot == 0) { *ndiv = 0; *err_iter = iter; }
        __threadfence();
        // every thread sees the same totals; one flag write is enough but all are harmless
        if (slot == 0) set_err(err, errbits);
        return;
    }
    if (slot == 0) *ndiv = (uint32_t)tdiv;
    unsigned long long f = flag64[slot], r = rank64[slot];
    if (f >> 32) divlist[r >> 32] = (int32_t)slot;
    if (f & 1ull) {
        unsigned long long fr = r & 0xffffffffull;
        if (fr < tdiv) freelist[fr] = (int32_t)slot;
    }
}

// copy_daughter_individuals! then divide_to_half! for the dividers and their daughters
// (division_death.jl:28-63). Other slots are unchanged by divide_to_half (factor 1, +0, ×1).
// CarbonMode (CarbonMode/division_death.jl:28-57): x, y, z, Sz, Bm, Chl and gen are copied, Bd is
// not — the daughter halves the damaged biomass its slot held before.
__global__ void k_daughters(SpcDev P, const int32_t* __restrict__ divlist,
                            const int32_t* __restrict__ freelist, const uint32_t* ndiv,
                            const uint32_t* err, int mode) {
    if (*err & PI_DEVERR_CAPACITY) return;
    uint32_t n = *ndiv;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        long long p = divlist[k], d = freelist[k];
        const double h = (2.0 - 1.0) / 2.0;
        if (mode == MODE_IRON) {
            // IronEnergyMode/division_death.jl:44-82: x, y, z, tdark and gen copied; Sz, Bm, CH, the
            // quotas, exEn and Chl copied and halved in both; age not copied
            double* pools[12] = { P.Sz, P.Bm, P.CH, P.qNO3, P.qNH4, P.qP, P.qFe, P.qFePS, P.qFeNR, P.qFeNF, P.exEn, P.Chl };
            const double gen = P.gen[p];
            P.x[d] = P.x[p]; P.y[d] = P.y[p]; P.z[d] = P.z[p]; P.tdark[d] = P.tdark[p];
#pragma unroll
            for (int q = 0; q < 12; ++q) { const double v = pools[q][p] * h; pools[q][d] = v; pools[q][p] = v; }
            P.gen[d] = gen + 1.0; P.age[d] = P.age[d] * (1.0 - 1.0);
            P.flags[d] = FL_AC | FL_DVID;
            P.gen[p] = gen + 1.0; P.age[p] = P.age[p] * (1.0 - 1.0);
            continue;
        }
        if (mode == MODE_MACRO) {
            // MacroMolecularMode/division_death.jl:28-62: the seven pools, x, y, z and gen are
            // copied and halved in both (not age)
            double* pools[7] = { P.PRO, P.DNA, P.RNA, P.CH, P.NST, P.PST, P.Chl };
            const double gen = P.gen[p];
            P.x[d] = P.x[p]; P.y[d] = P.y[p]; P.z[d] = P.z[p];
#pragma unroll
            for (int q = 0; q < 7; ++q) { const double v = pools[q][p] * h; pools[q][d] = v; pools[q][p] = v; }
            P.gen[d] = gen + 1.0; P.age[d] = P.age[d] * (1.0 - 1.0);
            P.flags[d] = FL_AC | FL_DVID;
            P.gen[p] = gen + 1.0; P.age[p] = P.age[p] * (1.0 - 1.0);
            continue;
        }
        if (mode == MODE_CARBON) {
            double Sz = P.Sz[p], Bm = P.Bm[p], Chl = P.Chl[p], gen = P.gen[p];
            P.x[d] = P.x[p]; P.y[d] = P.y[p]; P.z[d] = P.z[p];
            P.Sz[d] = Sz * h; P.Bm[d] = Bm * h; P.Bd[d] = P.Bd[d] * h; P.Chl[d] = Chl * h;
            P.gen[d] = gen + 1.0; P.age[d] = P.age[d] * (1.0 - 1.0);
            P.flags[d] = FL_AC | FL_DVID;
            P.Sz[p] = Sz * h; P.Bm[p] = Bm * h; P.Bd[p] = P.Bd[p] * h; P.Chl[p] = Chl * h;
            P.gen[p] = gen + 1.0; P.age[p] = P.age[p] * (1.0 - 1.0);
            continue;
        }
        double Sz = P.Sz[p], Bm = P.Bm[p], Cq = P.Cq[p], Nq = P.Nq[p], Pq = P.Pq[p], Chl = P.Chl[p];
        double gen = P.gen[p];
        P.x[d] = P.x[p]; P.y[d] = P.y[p]; P.z[d] = P.z[p];
        P.Sz[d] = Sz * h; P.Bm[d] = Bm * h; P.Cq[d] = Cq * h; P.Nq[d] = Nq * h; P.Pq[d] = Pq * h;
        P.Chl[d] = Chl * h; P.gen[d] = gen + 1.0; P.age[d] = P.age[d] * (1.0 - 1.0);
        P.flags[d] = FL_AC | FL_DVID;
        P.Sz[p] = Sz * h; P.Bm[p] = Bm * h; P.Cq[p] = Cq * h; P.Nq[p] = Nq * h; P.Pq[p] = Pq * h;
        P.Chl[p] = Chl * h; P.gen[p] = gen + 1.0; P.age[p] = P.age[p] * (1.0 - 1.0);
    }
}

// ------------------------------------------------------------------------------------------
// (b) physiology — QuotaMode/plankton_growth.jl:2-24, growth_kernels.jl:2-166,
//     division_death_probability.jl:7-107, find_NPT! (utils.jl:14-25), calc_consume!
//     (consume_loss.jl:2-9), diags_proc!(num) (plankton_update.jl:33)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ double shape_dec(double x, double xmax, double k, int pw) {
    double fx = jl_max(0.0, jl_min(1.0, 1.0 - x / xmax));
    return pi_pow_int(fx, pw) / (k + pi_pow_int(fx, pw));
}
__device__ __forceinline__ double shape_inc(double x, double xmax, double k, int pw) {
    double fx = jl_max(0.0, jl_min(1.0, 1.0 - x / xmax));
    double reg = pi_pow_int(fx, pw) / (k + pi_pow_int(fx, pw));
    return 1.0 - reg;
}
__device__ __forceinline__ double tempFunc_PS(double T, const pi_quota_params& p) {
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double regT = shape_dec(x, xmax, F_4em2, 4);
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * regT;
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
__device__ __forceinline__ double tempFunc(double T, const pi_quota_params& p) {
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0)));
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}

struct TracerPtrs { const double* c[PI_NTRACERS]; };

__global__ void k_physiology(DGrid g, SpcDev P, pi_quota_params p, long long C, int s,
                             double dT, double t, uint64_t seed, uint32_t iter, int shared_graz,
                             const double* __restrict__ NH4f, const double* __restrict__ NO3f,
                             const double* __restrict__ PO4f, const double* __restrict__ DOCf,
                             const double* __restrict__ par, const double* __restrict__ temp,
                             const uint32_t* __restrict__ off, const uint32_t* __restrict__ gid_sorted,
                             const int32_t* __restrict__ pos, double* __restrict__ contrib,
                             double* __restrict__ d_num, double* __restrict__ procv, const uint32_t* err) {
    long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    uint8_t f = P.flags[slot];
    int ac = f & FL_AC;
    int ac0 = P.stat[slot] & ST_AC0;
    long long e = ac0 ? pos[(long long)s * C + slot] : -1;
    if (!ac) {
        // Inactive after this step's deaths: every rate is multiplied by ac, the state is left
        // as it is (quotas of a lost individual are non-negative) and its decisions are 0.
        if (ac0) {
            double* K = contrib + e * 5;
            K[0] = 0.0; K[1] = 0.0; K[2] = 0.0; K[3] = 0.0; K[4] = 0.0;
        }
        return;
    }
    int xi, yi, zi;
    unpack_cell(g, P.cell[slot], xi, yi, zi);
    int c = gidx(g, xi, yi, zi);
    // find_NPT!: environment at the cell, times ac at gather time
    double NH4 = 0.0, NO3 = 0.0, PO4 = 0.0, DOC = 0.0, parv = 0.0, T = 0.0, pop = 0.0;
    if (ac0) {
        NH4 = jl_max(0.0, NH4f[c]); NO3 = jl_max(0.0, NO3f[c]); PO4 = jl_max(0.0, PO4f[c]);
        DOC = jl_max(0.0, DOCf[c]); parv = par[c]; T = temp[c];
        if (shared_graz) {
            pop = (double)(off[c + 1] - off[c]);
        } else {
            uint32_t n = 0;
            for (uint32_t q = off[c]; q < off[c + 1]; ++q) n += (gid_sorted[q] / (uint32_t)C) == (uint32_t)s;
            pop = (double)n;
        }
    }
    double Bm = P.Bm[slot], Cq = P.Cq[slot], Nq = P.Nq[slot], Pq = P.Pq[slot], Chl = P.Chl[slot];
    double age = P.age[slot];
    // calc_inorganic_uptake_kernel! (growth_kernels.jl:48-56)
    double aI = parv * p.alpha * p.Phi;
    double PCm = p.PCmax * tempFunc_PS(T, p);
    double PS = PCm * (1.0 - pi_exp(-aI / jl_max(F_1em30, PCm) * Chl / jl_max(F_1em30, Bm))) * Bm;
    PS = jl_mulb(PS, ac);
    double VNH4, VNO3, VPO4;
    {
        double Qn = (Nq + Bm * p.R_NC) / jl_max(F_1em30, Bm + Cq);
        double Qp = (Pq + Bm * p.R_PC) / jl_max(F_1em30, Bm + Cq);
        double regQN = shape_dec(Qn, p.Nqmax, F_1em4, 4);
        double regQP = shape_dec(Qp, p.Pqmax, F_1em4, 4);
        double a = jl_mulb(p.VNH4max * regQN * NH4 / jl_max(F_1em30, NH4 + p.KsatNH4) * tempFunc(T, p) * Bm, ac);
        double b = jl_mulb(p.VNO3max * regQN * NO3 / jl_max(F_1em30, NO3 + p.KsatNO3) * tempFunc(T, p) * Bm, ac);
        double cc = jl_mulb(p.VPO4max * regQP * PO4 / jl_max(F_1em30, PO4 + p.KsatPO4) * tempFunc(T, p) * Bm, ac);
        VNH4 = jl_min(a, NH4 / dT / jl_max(1.0, pop));
        VNO3 = jl_min(b, NO3 / dT / jl_max(1.0, pop));
        VPO4 = jl_min(cc, PO4 / dT / jl_max(1.0, pop));
    }
    // update_quotas_1_kernel! (:64-69)
    Cq += PS * dT;
    Pq += VPO4 * dT;
    Nq += (VNH4 + VNO3) * dT;
    // calc_organic_uptake_kernel! (:78-84)
    double VDOC;
    {
        double Qc = Cq / jl_max(F_1em30, Bm + Cq);
        double regQ = shape_dec(Qc, p.Cqmax, F_1em4, 4);
        double VN = p.VDOCmax * regQ * DOC / jl_max(F_1em30, DOC + p.KsatDOC) * tempFunc(T, p) * Bm;
        VDOC = jl_mulb(jl_min(VN, DOC / dT / jl_max(1.0, pop)), ac);
        VDOC = jl_mulb(VDOC, jl_isless(F_1em2, PS / (VDOC + PS)));
    }
    // calc_ρChl_kernel! (:92-97)
    double rChl = jl_mulb(jl_mulb(PS / jl_max(F_1em30, Bm) * p.Chl2N /
                                  jl_max(F_1em30, parv * p.alpha * p.Phi * Chl / Bm),
                                  jl_isless(F_1em1, parv)), ac);
    // calc_respir_kernel! (:105-108)
    double resp = jl_mulb(p.respir * Bm * tempFunc(T, p), ac);
    // update_quotas_2_kernel! (:117-124)
    Cq = Cq + (VDOC - resp) * dT;
    Bm = Bm - jl_max(0.0, (0.0 - Cq));
    Nq = Nq + jl_max(0.0, (0.0 - Cq)) * p.R_NC;
    Pq = Pq + jl_max(0.0, (0.0 - Cq)) * p.R_PC;
    Cq = Cq + jl_max(0.0, (0.0 - Cq));
    // calc_BS_kernel! (:132-138)
    double mn = jl_min(jl_min(Cq, Nq / p.R_NC), Pq / p.R_PC);
    double BS = jl_mulb(mn * p.k_mtb, ac);
    double exu = jl_mulb(jl_max(0.0, Cq - mn) * p.k_mtb, ac);
    // update_biomass_kernel! (:146-154)
    Bm += dT * BS;
    Cq -= dT * (BS + exu);
    Nq -= dT * BS * p.R_NC;
    Pq -= dT * BS * p.R_PC;
    Chl += dT * BS * p.R_NC * rChl;
    age += jl_mulb(dT / 3600.0, ac);
    // update_cellsize_kernel! (:163-166)
    double Sz = Bm / (p.Cquota * p.Nsuper);
    // probabilities (division_death_probability.jl:49-68, 26-30)
    double graz = jl_mulb(pop * p.grz_P, ac);
    double mort = jl_mulb(p.mort_P * shape_dec(Sz, p.mort_reg, F_1em5, 4), ac);
    double dv;
    int ty = (int)p.dvid_type;
    if (ty == 1) dv = p.dvid_P * shape_inc(Sz, p.dvid_reg, F_2em3, 2);
    else if (ty == 2) dv = p.dvid_P * shape_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg, F_1em5, 4);
    else dv = p.dvid_P * shape_inc(Sz, p.dvid_reg, F_1em3, 4) * shape_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg2, F_1em5, 4);
    double dvid = jl_mulb(dv, ac);
    // get_probability! (:95-107)
    double r0, r1, r2;
    pi_draw3(seed, iter, (uint32_t)s, PI_DRAW_DECISION, (uint32_t)slot, &r0, &r1, &r2);
    int dg = jl_isless(r0, graz * dT) && ac;
    int dm = jl_isless(r1, mort * dT) && ac;
    int dd = jl_isless(r2, dvid * dT) && ac;
    P.Bm[slot] = Bm; P.Cq[slot] = Cq; P.Nq[slot] = Nq; P.Pq[slot] = Pq; P.Chl[slot] = Chl;
    P.age[slot] = age; P.Sz[slot] = Sz;
    P.flags[slot] = (uint8_t)(FL_AC | (dg ? FL_GRAZ : 0) | (dm ? FL_MORT : 0) | (dd ? FL_DVID : 0));
    // calc_consume_kernel!: contributions kept per cell entry, summed in order later
    if (ac0) {
        double* K = contrib + e * 5;
        K[0] = jl_mulb((resp - PS) * dT, ac);
        K[1] = jl_mulb((exu - VDOC) * dT, ac);
        K[2] = jl_mulb(-VNH4 * dT, ac);
        K[3] = jl_mulb(-VNO3 * dT, ac);
        K[4] = jl_mulb(-VPO4 * dT, ac);
    }
    // diags_spcs! values of the slot (PI_PROC_* order), summed per cell in slot order later
    if (procv) {
        const double v[PI_NPROC] = { PS, BS, VDOC, VNH4, VNO3, VPO4, resp, exu, Bm, Cq, Nq, Pq, Chl };
        for (int q = 0; q < PI_NPROC; ++q) procv[(long long)q * C + slot] = v[q];
    }
    // diags_proc!(num, ac, ac) at the slot's (possibly stale) cell
    atomicAdd(&d_num[c], 1.0);
}

// ------------------------------------------------------------------------------------------
// CarbonMode physiology — CarbonMode/plankton_growth.jl:2-29, growth_kernels.jl:2-120,
// division_death_probability.jl:7-107, calc_consume! (consume_loss.jl:2-5)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double c_tempFunc_PS(double T, const pi_carbon_params& p) {
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double regT = shape_dec(x, xmax, F_1em1, 4);
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * regT;
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
__device__ __forceinline__ double c_tempFunc(double T, const pi_carbon_params& p) {
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0)));
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
// gamma_alloc (growth_kernels.jl:22-26)
__device__ __forceinline__ double c_gamma(double Bm, double Bd, const pi_carbon_params& p) {
    double gm = jl_mulb(Bd / jl_max(F_1em30, Bm), jl_isless(0.0, Bd));
    return jl_mulb(jl_min(1.0, gm), p.thermal == 1.0);
}

__global__ void k_physiology_carbon(DGrid g, SpcDev P, pi_carbon_params p, long long C, int s,
                                    double dT, double t, uint64_t seed, uint32_t iter, int shared_graz,
                                    const double* __restrict__ par, const double* __restrict__ temp,
                                    const uint32_t* __restrict__ off, const uint32_t* __restrict__ gid_sorted,
                                    const int32_t* __restrict__ pos, double* __restrict__ contrib,
                                    double* __restrict__ d_num, double* __restrict__ procv, const uint32_t* err) {
    long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    uint8_t f = P.flags[slot];
    int ac = f & FL_AC;
    int ac0 = P.stat[slot] & ST_AC0;
    long long e = ac0 ? pos[(long long)s * C + slot] : -1;
    if (!ac) {
        // inactive after this step's deaths: every rate that carries ac is 0. Thermal damage does
        // not (growth_kernels.jl:69-75), and an individual killed in this step gathered its
        // temperature while it was active, so its damaged biomass still grows by TD·ΔT; the
        // state of a slot inactive before the step keeps its values (T = 0 gives TD = 0).
        if (ac0) {
            double* K = contrib + e * 5;
            K[0] = 0.0; K[1] = 0.0; K[2] = 0.0; K[3] = 0.0; K[4] = 0.0;
            int xi, yi, zi;
            unpack_cell(g, P.cell[slot], xi, yi, zi);
            const double T = temp[gidx(g, xi, yi, zi)];
            const double Bm = P.Bm[slot], Bd = P.Bd[slot];
            double TD = jl_mulb(jl_mulb(jl_mulb((T - p.Topt) * p.f_T2B * (Bm - Bd), jl_isless(p.Topt, T)),
                                        jl_isless(Bd, Bm)), p.thermal == 1.0);
            TD = jl_max(0.0, jl_min(TD, (Bm - Bd) / dT));
            P.Bd[slot] = Bd + (TD - 0.0) * dT;           // RP = PS·γ = 0 (PS carries ac)
        }
        return;
    }
    int xi, yi, zi;
    unpack_cell(g, P.cell[slot], xi, yi, zi);
    int c = gidx(g, xi, yi, zi);
    double parv = 0.0, T = 0.0, pop = 0.0;
    if (ac0) {
        parv = par[c]; T = temp[c];
        if (shared_graz) {
            pop = (double)(off[c + 1] - off[c]);
        } else {
            uint32_t n = 0;
            for (uint32_t q = off[c]; q < off[c + 1]; ++q) n += (gid_sorted[q] / (uint32_t)C) == (uint32_t)s;
            pop = (double)n;
        }
    }
    double Bm = P.Bm[slot], Bd = P.Bd[slot], Chl = P.Chl[slot], age = P.age[slot];
    // calc_PS! (calc_photosynthesis, growth_kernels.jl:29-36)
    double aI = parv * p.alpha * p.Phi;
    double PCm = p.PCmax * (c_tempFunc(T, p) * p.thermal + c_tempFunc_PS(T, p) * (1.0 - p.thermal));
    double light = 1.0 - pi_exp(-aI / jl_max(F_1em30, PCm) * Chl / jl_max(F_1em30, Bm));
    double PS = jl_mulb(PCm * jl_max(0.0, Bm - Bd) * (light * (1.0 - p.is_bact) + p.is_bact), ac);
    // calc_BS!, calc_repair! (:55-64), calc_thermal_damage! (:69-75), calc_respir! (:82-85)
    double BS = PS * (1.0 - c_gamma(Bm, Bd, p));
    double RP = PS * c_gamma(Bm, Bd, p);
    double TD = jl_mulb(jl_mulb(jl_mulb((T - p.Topt) * p.f_T2B * (Bm - Bd), jl_isless(p.Topt, T)),
                                jl_isless(Bd, Bm)), p.thermal == 1.0);
    TD = jl_max(0.0, jl_min(TD, (Bm - Bd) / dT));
    double RS = jl_mulb(p.respir * Bm * c_tempFunc(T, p), ac);
    // update_quotas! (:92-97), update_cellsize! (:104-108)
    Bm += (BS - RS) * dT;
    Bd += (TD - RP) * dT;
    age += jl_mulb(dT / 3600.0, ac);
    double Sz = Bm / (p.Cquota * p.Nsuper);
    Chl = Bm * p.Chl2C;
    // probabilities (division_death_probability.jl:26-30, 49-52, 60-77)
    double graz = jl_mulb(pop * p.grz_P, ac);
    double dv;
    int ty = (int)p.dvid_type;
    if (ty == 1) dv = p.dvid_P * shape_inc(Sz, p.dvid_reg, F_2em3, 2);
    else if (ty == 2) dv = p.dvid_P * shape_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg, F_1em5, 4);
    else dv = p.dvid_P * shape_inc(Sz, p.dvid_reg, F_1em3, 4) * shape_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg2, F_1em5, 4);
    double dvid = jl_mulb(dv, ac);
    double mort = p.thermal == 1.0 ? jl_mulb(p.mort_P * shape_inc(Bd / jl_max(F_1em30, Bm), F_0p99, F_1em6, 4), ac)
                                   : jl_mulb(p.mort_P * shape_dec(Sz, p.mort_reg, F_1em5, 4), ac);
    // get_probability! (:95-107)
    double r0, r1, r2;
    pi_draw3(seed, iter, (uint32_t)s, PI_DRAW_DECISION, (uint32_t)slot, &r0, &r1, &r2);
    int dg = jl_isless(r0, graz * dT) && ac;
    int dm = jl_isless(r1, mort * dT) && ac;
    int dd = jl_isless(r2, dvid * dT) && ac;
    P.Bm[slot] = Bm; P.Bd[slot] = Bd; P.Chl[slot] = Chl; P.age[slot] = age; P.Sz[slot] = Sz;
    P.flags[slot] = (uint8_t)(FL_AC | (dg ? FL_GRAZ : 0) | (dm ? FL_MORT : 0) | (dd ? FL_DVID : 0));
    // calc_consume_kernel!: DIC only
    if (ac0) {
        double* K = contrib + e * 5;
        K[0] = jl_mulb((RS - PS) * dT, ac);
        K[1] = 0.0; K[2] = 0.0; K[3] = 0.0; K[4] = 0.0;
    }
    // diags_spcs! values of the slot (PI_CPROC_* order)
    if (procv) {
        const double v[PI_NCPROC] = { PS, BS, RP, RS, TD, Bm, Bd, Chl };
        for (int q = 0; q < PI_NCPROC; ++q) procv[(long long)q * C + slot] = v[q];
    }
    atomicAdd(&d_num[c], 1.0);
}

// ------------------------------------------------------------------------------------------
// MacroMolecularMode physiology — MacroMolecularMode/plankton_growth.jl:2-28, growth_kernels.jl:1-200,
// division_death_probability.jl:37-40, 49-52, 84-107, calc_consume! (consume_loss.jl:2-9)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double m_tempFunc_PS(double T, const pi_macro_params& p) {
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double regT = shape_dec(x, xmax, F_4em2, 4);
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * regT;
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
__device__ __forceinline__ double m_tempFunc(double T, const pi_macro_params& p) {
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0)));
    k = jl_max(0.0, k);
    double OGT_rate = pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0)));
    return jl_min(1.0, k / OGT_rate);
}
// Every slot is updated: the synthesis and exudation terms carry no ac, so the state of an
// inactive slot keeps changing as in the reference, from zero light, temperature and nutrients
// unless it was active when they were gathered (an individual grazed or dead in this step).
__global__ void k_physiology_macro(DGrid g, SpcDev P, pi_macro_params p, long long C, int s,
                                   double dT, uint64_t seed, uint32_t iter, int shared_graz,
                                   const double* __restrict__ NH4f, const double* __restrict__ NO3f,
                                   const double* __restrict__ PO4f, const double* __restrict__ DOCf,
                                   const double* __restrict__ par, const double* __restrict__ temp,
                                   const uint32_t* __restrict__ off, const uint32_t* __restrict__ gid_sorted,
                                   const int32_t* __restrict__ pos, double* __restrict__ contrib,
                                   double* __restrict__ d_num, double* __restrict__ procv, const uint32_t* err) {
    long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    const int ac = P.flags[slot] & FL_AC;
    const int ac0 = P.stat[slot] & ST_AC0;
    int c = -1;
    double NH4 = 0.0, NO3 = 0.0, PO4 = 0.0, DOC = 0.0, parv = 0.0, T = 0.0, pop = 0.0;
    if (ac0) {                                         // find_NPT! (utils.jl:14-25), × ac at gathering
        int xi, yi, zi;
        unpack_cell(g, P.cell[slot], xi, yi, zi);
        c = gidx(g, xi, yi, zi);
        NH4 = jl_max(0.0, NH4f[c]); NO3 = jl_max(0.0, NO3f[c]); PO4 = jl_max(0.0, PO4f[c]); DOC = jl_max(0.0, DOCf[c]);
        parv = par[c]; T = temp[c];
        if (shared_graz) {
            pop = (double)(off[c + 1] - off[c]);
        } else {
            uint32_t n = 0;
            for (uint32_t q = off[c]; q < off[c + 1]; ++q) n += (gid_sorted[q] / (uint32_t)C) == (uint32_t)s;
            pop = (double)n;
        }
    }
    double PRO = P.PRO[slot], DNA = P.DNA[slot], RNA = P.RNA[slot], CH = P.CH[slot];
    double NST = P.NST[slot], PST = P.PST[slot], Chl = P.Chl[slot], age = P.age[slot];
    // calc_inorganic_uptake_kernel! (growth_kernels.jl:45-54): calc_PS (:20-25), calc_NP_uptake (:28-42)
    double aI = parv * p.alpha * p.Phi;
    double PCm = p.PCmax * m_tempFunc_PS(T, p);
    double PS = jl_mulb(PCm * (1.0 - pi_exp(-aI / jl_max(F_1em30, PCm) * Chl / jl_max(F_1em30, PRO))) * PRO, ac);
    double R_NST = NST / jl_max(F_1em30, m_totN(PRO, DNA, RNA, NST, Chl, p));
    double R_PST = PST / jl_max(F_1em30, m_totP(DNA, RNA, PST, p));
    double regQN = shape_dec(R_NST, p.NSTmax, F_1em4, 4), regQP = shape_dec(R_PST, p.PSTmax, F_1em4, 4);
    double VNH4 = jl_mulb(p.VNH4max * regQN * NH4 / jl_max(F_1em30, NH4 + p.KsatNH4) * m_tempFunc(T, p) * PRO, ac);
    double VNO3 = jl_mulb(p.VNO3max * regQN * NO3 / jl_max(F_1em30, NO3 + p.KsatNO3) * m_tempFunc(T, p) * PRO, ac);
    double VPO4 = jl_mulb(p.VPO4max * regQP * PO4 / jl_max(F_1em30, PO4 + p.KsatPO4) * m_tempFunc(T, p) * PRO, ac);
    VNH4 = jl_min(VNH4, NH4 / dT / jl_max(1.0, pop));
    VNO3 = jl_min(VNO3, NO3 / dT / jl_max(1.0, pop));
    VPO4 = jl_min(VPO4, PO4 / dT / jl_max(1.0, pop));
    // update_quotas_1_kernel! (:63-67)
    CH += PS * dT; PST += VPO4 * dT; NST += (VNH4 + VNO3) * dT;
    // calc_organic_uptake_kernel! (:82-90), calc_DOC_uptake (:73-80)
    double R_CH = CH / jl_max(F_1em30, m_totC(PRO, DNA, RNA, CH, Chl));
    double regQ = shape_dec(R_CH, p.CHmax, F_1em4, 4);
    double VN = p.VDOCmax * regQ * DOC / jl_max(F_1em30, DOC + p.KsatDOC) * m_tempFunc(T, p) * PRO;
    double VDOC = jl_mulb(jl_min(VN, DOC / dT / jl_max(1.0, pop)), ac);
    VDOC = jl_mulb(VDOC, jl_isless(F_5em2, PS / (VDOC + PS)));
    // calc_ρChl_kernel! (:98-103), calc_respir_kernel! (:111-114)
    double rChl = jl_mulb(jl_mulb(PS / jl_max(F_1em30, PRO) / jl_max(F_1em30, parv * p.alpha * p.Phi * Chl / jl_max(F_1em30, PRO)),
                                  jl_isless(F_1em1, parv)), ac);
    double resp = jl_mulb(p.respir * PRO * m_tempFunc(T, p), ac);
    // update_quotas_2_kernel! (:124-130)
    CH = CH + (VDOC - resp) * dT;
    PRO = PRO - jl_max(0.0, 0.0 - CH);
    NST = NST + jl_max(0.0, 0.0 - CH) * p.R_NC_PRO;
    CH = CH + jl_max(0.0, 0.0 - CH);
    // calc_BS_kernel! (:136-152)
    double tf = m_tempFunc(T, p);
    double limit_PRO = jl_min(CH / (CH + p.k_sat_pro * p.Nsuper), NST / (NST + p.k_sat_pro * p.Nsuper * p.R_NC_PRO));
    double limit_DNA = jl_min(jl_min(CH / (CH + p.k_sat_dna * p.Nsuper), NST / (NST + p.k_sat_dna * p.Nsuper * p.R_NC_DNA)),
                              PST / (PST + p.k_sat_dna * p.Nsuper * p.R_PC_DNA));
    double limit_RNA = jl_min(jl_min(CH / (CH + p.k_sat_rna * p.Nsuper), NST / (NST + p.k_sat_rna * p.Nsuper * p.R_NC_RNA)),
                              PST / (PST + p.k_sat_rna * p.Nsuper * p.R_PC_RNA));
    double S_PRO = p.k_pro * RNA * limit_PRO * tf;
    double S_DNA = jl_mulb(p.k_dna * PRO * limit_DNA * tf, jl_isless(DNA / (p.C_DNA * p.Nsuper), 2.0));
    double S_RNA = p.k_rna * PRO * limit_RNA * tf;
    // update_biomass_kernel! (:159-171)
    PRO += dT * S_PRO;
    DNA += dT * S_DNA;
    RNA += dT * S_RNA;
    CH -= dT * (S_PRO + S_DNA + S_RNA + S_PRO * rChl);
    NST -= dT * (S_PRO * p.R_NC_PRO + S_DNA * p.R_NC_DNA + S_RNA * p.R_NC_RNA + S_PRO * rChl * 4.0 / 55.0);
    PST -= dT * (S_DNA * p.R_PC_DNA + S_RNA * p.R_PC_RNA);
    Chl += dT * S_PRO * rChl * F_CHL / 55.0;
    age += jl_mulb(dT / 3600.0, ac);
    // calc_exudation_kernel! (:179-183), update_CH_kernel! (:190-193)
    double exu = jl_max(0.0, CH - p.CHmax * m_totC(PRO, DNA, RNA, CH, Chl));
    CH -= exu;
    // calc_graz_quadratic!, calc_MM_mort!, calc_MM_dvid!, get_probability!
    double graz = jl_mulb(pop * p.grz_P, ac);
    double mort = jl_mulb(p.mort_P * shape_inc(age, p.mort_reg, F_1em4, 4), ac);
    double dvid = jl_mulb(p.dvid_P, jl_isless(2.0, DNA / (p.C_DNA * p.Nsuper)));
    double r0, r1, r2;
    pi_draw3(seed, iter, (uint32_t)s, PI_DRAW_DECISION, (uint32_t)slot, &r0, &r1, &r2);
    int dg = jl_isless(r0, graz * dT) && ac;
    int dm = jl_isless(r1, mort * dT) && ac;
    int dd = jl_isless(r2, dvid * dT) && ac;
    P.PRO[slot] = PRO; P.DNA[slot] = DNA; P.RNA[slot] = RNA; P.CH[slot] = CH;
    P.NST[slot] = NST; P.PST[slot] = PST; P.Chl[slot] = Chl; P.age[slot] = age;
    P.flags[slot] = (uint8_t)((ac ? FL_AC : 0) | (dg ? FL_GRAZ : 0) | (dm ? FL_MORT : 0) | (dd ? FL_DVID : 0));
    // calc_consume_kernel! (consume_loss.jl:2-9) for the individuals binned this step
    if (ac0) {
        double* K = contrib + (long long)pos[(long long)s * C + slot] * 5;
        K[0] = jl_mulb((resp - PS) * dT, ac);
        K[1] = jl_mulb((exu - VDOC) * dT, ac);
        K[2] = jl_mulb(-VNH4 * dT, ac);
        K[3] = jl_mulb(-VNO3 * dT, ac);
        K[4] = jl_mulb(-VPO4 * dT, ac);
    }
    // diags_spcs! (Diagnostics/diagnostics_kernels.jl:20-21) in PI_MPROC_* order: VNH4 (listed
    // there as :VHN4) and exu are never accumulated
    if (procv) {
        const double v[PI_NMPROC] = { PS, VDOC, 0.0, VNO3, VPO4, resp, rChl, S_PRO, S_DNA, S_RNA, 0.0,
                                      CH, NST, PST, PRO, DNA, RNA, Chl };
        for (int q = 0; q < PI_NMPROC; ++q) procv[(long long)q * C + slot] = v[q];
    }
    if (ac) {
        int xi, yi, zi;
        unpack_cell(g, P.cell[slot], xi, yi, zi);
        atomicAdd(&d_num[gidx(g, xi, yi, zi)], 1.0);
    }
}

// diags_spcs! (Diagnostics/diagnostics_kernels.jl:14-33): the cell of every slot active after the
// species' update (its find_inds! cell), G for the others, for a stable sort by cell.
__global__ void k_diag_keys(DGrid g, SpcDev P, long long C, uint32_t* __restrict__ key, uint32_t* __restrict__ val,
                            const uint32_t* err) {
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    uint32_t k = (uint32_t)g.G;
    if (!(*err & PI_DEVERR_CAPACITY) && (P.flags[slot] & FL_AC)) {
        int xi, yi, zi;
        unpack_cell(g, P.cell[slot], xi, yi, zi);
        k = (uint32_t)gidx(g, xi, yi, zi);
    }
    key[slot] = k;
    val[slot] = (uint32_t)slot;
}

// d[cell] += value of each of the cell's slots in ascending slot order (the sorted run of the
// cell), for the enabled processes; one thread per run.
__global__ void k_diag_sum(long long C, long long G, const uint32_t* __restrict__ key, const uint32_t* __restrict__ val,
                           const double* __restrict__ procv, uint32_t mask, double* __restrict__ d) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    const uint32_t c = key[i];
    if (c >= (uint32_t)G || (i > 0 && key[i - 1] == c)) return;
    for (int q = 0; q < PI_MAXPROC; ++q) {
        if (!(mask >> q & 1u)) continue;
        double x = d[(long long)q * G + c];
        for (long long j = i; j < C && key[j] == c; ++j) x = x + procv[(long long)q * C + val[j]];
        d[(long long)q * G + c] = x;
    }
}

// diags.tracer[name] .+= tracer (time_step.jl:168-172) for the enabled tracers, halos included.
__global__ void k_diag_tracers(double* __restrict__ d, const double* __restrict__ tr, uint32_t mask, long long G,
                               const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < (long long)PI_NTRACERS * G;
         q += (long long)gridDim.x * blockDim.x)
        if (mask >> (q / G) & 1u) d[q] = d[q] + tr[q];
}

// ------------------------------------------------------------------------------------------
// (d) tracer update — Biogeochemistry/tracer_update.jl:22-43, Advection/DST3FL.jl:1-73,
//     Advection/multi_dim_adv.jl:1-135, operaters.jl:1-27, tracer_diffusion.jl, tracer_sinking.jl,
//     tracer_forcings.jl, HaloRegions/apply_bcs.jl
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ double theta(double dnum, double d0) {
    return fabs(d0) * F_THMAX <= fabs(dnum) ? copysign(F_THMAX, dnum * d0) : dnum / d0;
}
__device__ __forceinline__ double psi_lim(double cfl, double th) {
    double d0 = (2.0 - cfl) * (1.0 - cfl) / 6.0;
    double d1 = (1.0 - cfl * cfl) / 6.0;
    return jl_max(0.0, jl_min(jl_min(1.0, d0 + d1 * th), th * (1.0 - cfl) / (cfl + F_1em20)));
}
// DST3FL face flux on one axis from the 4 values around the face (cm2 = c[i-2], cm1 = c[i-1],
// c0 = c[i], cp1 = c[i+1]) and the landmask at those points. UP = 1 for x/y (upwind cell i-1),
// UP = 0 for z (index grows downward: upwind cell is k for upward flow), adv_flux_x/y/z.
__device__ __forceinline__ double dst3_flux_xy(double cm2, double cm1, double c0, double cp1,
                                               int lm2, int lm1, int l0, int lp1,
                                               double vel, double area, double dxc, double dT) {
    double cfl = fabs(vel * dT / dxc);
    double tr = area * vel;
    double d0 = jl_mulb(jl_mulb(c0 - cm1, l0), lm1);     // δ⁰ = (c[i] - c[i-1])
    double dm = jl_mulb(jl_mulb(cm1 - cm2, lm1), lm2);   // δ⁻ = (c[i-1] - c[i-2])
    double dp = jl_mulb(jl_mulb(cp1 - c0, lp1), l0);     // δ⁺ = (c[i+1] - c[i])
    double psp = psi_lim(cfl, theta(dm, d0));
    double psm = psi_lim(cfl, theta(dp, d0));
    return 0.5 * (tr + fabs(tr)) * (cm1 + psp * d0) + 0.5 * (tr - fabs(tr)) * (c0 - psm * d0);
}
// z: cm2 = c[k-2], cm1 = c[k-1], c0 = c[k], cp1 = c[k+1]
__device__ __forceinline__ double dst3_flux_z(double cm2, double cm1, double c0, double cp1,
                                              int lm2, int lm1, int l0, int lp1,
                                              double w, double area, double dzc, double dT) {
    double cfl = fabs(w * dT / dzc);
    double tr = area * w;
    double d0 = jl_mulb(jl_mulb(cm1 - c0, l0), lm1);     // δz⁰ = c[k-1] - c[k]
    double dm = jl_mulb(jl_mulb(cm2 - cm1, lm1), lm2);   // δz⁻ = c[k-2] - c[k-1]
    double dp = jl_mulb(jl_mulb(c0 - cp1, lp1), l0);     // δz⁺ = c[k] - c[k+1]
    double psp = psi_lim(cfl, theta(dm, d0));            // Ψz⁺
    double psm = psi_lim(cfl, theta(dp, d0));            // Ψz⁻
    return 0.5 * (tr + fabs(tr)) * (c0 + psm * d0) + 0.5 * (tr - fabs(tr)) * (cm1 - psp * d0);
}

// Index maps that stand in for the halo fill of tracer_temp between sweeps.
__device__ __forceinline__ int wrap_axis(int a, int N, int H, int topo) {
    if (topo == PI_PERIODIC) {
        while (a < H + 1) a += N;
        while (a > N + H) a -= N;
        return a;
    }
    return a < H + 1 ? H + 1 : (a > N + H ? N + H : a);
}

// Per-face quantities of DST3FL that do not depend on the tracer (CFL, transport, d₀ and d₁ of
// DST3FL.jl:5-11, the factors of adv_flux): computed once per face and shared by the 14 tracers.
// Each is the same IEEE expression the per-tracer formula evaluates, so results are unchanged.
struct FaceCoef { double d0c, d1c, omc, cpe, hp, hm; };

__device__ __forceinline__ FaceCoef face_coef(double vel, double area, double dxc, double dT) {
    FaceCoef f;
    double cfl = fabs(vel * dT / dxc);
    double tr = area * vel;
    f.d0c = (2.0 - cfl) * (1.0 - cfl) / 6.0;
    f.d1c = (1.0 - cfl * cfl) / 6.0;
    f.omc = 1.0 - cfl;
    f.cpe = cfl + F_1em20;
    f.hp = 0.5 * (tr + fabs(tr));
    f.hm = 0.5 * (tr - fabs(tr));
    return f;
}
__device__ __forceinline__ double psi_c(const FaceCoef& f, double th) {
    return jl_max(0.0, jl_min(jl_min(1.0, f.d0c + f.d1c * th), th * f.omc / f.cpe));
}
// adv_flux_x / adv_flux_y at face i from c[i-2], c[i-1], c[i], c[i+1]
__device__ __forceinline__ double flux_xy_c(const FaceCoef& f, double cm2, double cm1, double c0, double cp1,
                                            int lm2, int lm1, int l0, int lp1) {
    double d0 = jl_mulb(jl_mulb(c0 - cm1, l0), lm1);
    double dm = jl_mulb(jl_mulb(cm1 - cm2, lm1), lm2);
    double dp = jl_mulb(jl_mulb(cp1 - c0, lp1), l0);
    double psp = psi_c(f, theta(dm, d0));
    double psm = psi_c(f, theta(dp, d0));
    return f.hp * (cm1 + psp * d0) + f.hm * (c0 - psm * d0);
}
// adv_flux_z at face k from c[k-2], c[k-1], c[k], c[k+1] (index grows downward)
__device__ __forceinline__ double flux_z_c(const FaceCoef& f, double cm2, double cm1, double c0, double cp1,
                                           int lm2, int lm1, int l0, int lp1) {
    double d0 = jl_mulb(jl_mulb(cm1 - c0, l0), lm1);
    double dm = jl_mulb(jl_mulb(cm2 - cm1, lm1), lm2);
    double dp = jl_mulb(jl_mulb(c0 - cp1, lp1), l0);
    double psp = psi_c(f, theta(dm, d0));
    double psm = psi_c(f, theta(dp, d0));
    return f.hp * (c0 + psm * d0) + f.hm * (cm1 - psp * d0);
}

// x sweep (calc_Gcˣ + fill_halo_Gcs + multi_dim_x on tracer_temp = tracer). Each warp owns 31
// cells of one row and 32 faces: lane l computes the flux of face i0 + l once, and the east-face
// flux of its cell comes from lane l + 1 by shuffle. The face after the last interior cell follows
// fill_halo_Gcs!: the periodic image of face H+1, or zero when Bounded.
#define SWX_WARPS 4
template <bool LL>
__global__ void __launch_bounds__(32 * SWX_WARPS) k_sweep_x(DGrid g, const double* __restrict__ tr,
                                                            double* __restrict__ tta,
                                                            const double* __restrict__ u, double dT,
                                                            const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * SWX_WARPS + (threadIdx.x >> 5);
    const int i0 = wid * 31 + 1 + g.Hx;
    if (i0 > g.Nx + g.Hx) return;                    // uniform per warp
    const int j = blockIdx.y + 1 + g.Hy, k = blockIdx.z + 1 + g.Hz;
    const int f = i0 + lane;                         // this lane's face (west face of cell f)
    const int last = g.Nx + g.Hx;
    const bool has_face = f <= last + 1;
    const bool has_cell = lane < 31 && f <= last;
    const bool special = f == last + 1;
    const bool zero_face = !has_face || (special && g.tx != PI_PERIODIC);
    const int fs = special ? g.Hx + 1 : f;           // face whose stencil gives the flux
    const long long G = g.G;
    const double ax = g.dy * dzF1(g, k);             // Ax of a RectilinearGrid
    const int qf = gidx(g, has_face ? fs : i0, j, k);
    FaceCoef fc{};
    int lm2 = 1, lm1 = 1, l0 = 1, lp1 = 1;
    if (!zero_face) {
        fc = face_coef(u[qf], LL ? Axm<LL>(g, fs, j, k) : ax, dxCm<LL>(g, fs, j), dT);
        lm2 = lmask(g, fs - 2, j, k); lm1 = lmask(g, fs - 1, j, k); l0 = lmask(g, fs, j, k); lp1 = lmask(g, fs + 1, j, k);
    }
    const int qc = gidx(g, has_cell ? f : i0, j, k);
    double ftr = 0.0, dtv = 0.0;
    int cl0 = 1, clp = 1;
    if (has_cell) {
        cl0 = lmask(g, f, j, k); clp = lmask(g, f + 1, j, k);
        ftr = jl_mulb(jl_mulb((LL ? Axm<LL>(g, f + 1, j, k) : ax) * u[qc + 1] - (LL ? Axm<LL>(g, f, j, k) : ax) * u[qc], clp), cl0);
        dtv = dT / vol<LL>(g, f, j, k);
    }
#pragma unroll 2
    for (int n = 0; n < PI_NTRACERS; ++n) {
        const double* c = tr + n * G;
        double F = zero_face ? 0.0 : flux_xy_c(fc, c[qf - 2], c[qf - 1], c[qf], c[qf + 1], lm2, lm1, l0, lp1);
        double Fe = __shfl_down_sync(0xffffffffu, F, 1);
        if (has_cell) {
            double c0 = c[qc];
            double dG = jl_mulb(jl_mulb(Fe - F, clp), cl0);
            tta[n * G + qc] = c0 - dtv * (dG - c0 * ftr);
        }
    }
}

// y sweep on tracer_temp after x (multi_dim_y, original tracer in the update term). Each thread
// walks SWY_L cells along y carrying the face flux (each face computed once, plus one shared face
// per segment), tracer by tracer so a thread holds one running flux; lanes run along x for
// coalesced access. Rows outside the interior are read through the periodic or clamped map the
// halo fill of tracer_temp produces.
#define SWY_L 8
#define SWY_TY 4
template <bool LL>
__device__ __forceinline__ double yface_flux(const DGrid& g, const double* __restrict__ c,
                                             const double* __restrict__ v, int i, int f, int k,
                                             double ay, double dT) {
    const bool special = f == g.Ny + g.Hy + 1;
    if (special && g.ty != PI_PERIODIC) return 0.0;            // fill_halo_north_Gc! (Bounded)
    const int fs = special ? g.Hy + 1 : f;                      // periodic: Gc[N+H+1] = Gc[H+1]
    FaceCoef fc = face_coef(v[gidx(g, i, fs, k)], LL ? Aym<LL>(g, i, fs, k) : ay, dyCm<LL>(g, i, fs), dT);
    int r0 = gidx(g, i, wrap_axis(fs - 2, g.Ny, g.Hy, g.ty), k), r1 = gidx(g, i, wrap_axis(fs - 1, g.Ny, g.Hy, g.ty), k);
    int r2 = gidx(g, i, wrap_axis(fs, g.Ny, g.Hy, g.ty), k), r3 = gidx(g, i, wrap_axis(fs + 1, g.Ny, g.Hy, g.ty), k);
    return flux_xy_c(fc, c[r0], c[r1], c[r2], c[r3], lmask(g, i, fs - 2, k), lmask(g, i, fs - 1, k),
                     lmask(g, i, fs, k), lmask(g, i, fs + 1, k));
}

template <bool LL>
__global__ void __launch_bounds__(32 * SWY_TY, 8) k_sweep_y(DGrid g, const double* __restrict__ tr,
                                                         const double* __restrict__ tta,
                                                         double* __restrict__ ttb,
                                                         const double* __restrict__ v, double dT,
                                                         const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    const int i = blockIdx.x * 32 + threadIdx.x + 1 + g.Hx;
    const int j0 = (blockIdx.y * SWY_TY + threadIdx.y) * SWY_L + 1 + g.Hy;
    const int k = blockIdx.z + 1 + g.Hz;
    if (i > g.Nx + g.Hx || j0 > g.Ny + g.Hy) return;
    const int jend = min(j0 + SWY_L - 1, g.Ny + g.Hy);
    const long long G = g.G;
    // the face area and ΔT/volume of a RectilinearGrid are the same for every row
    const double ay = g.dx * dzF1(g, k);
    const double dtv0 = dT / vol<false>(g, i, j0, k);
#pragma unroll 1
    for (int t = 0; t < PI_NTRACERS; ++t) {
        const double* c = tta + t * G;
        double Ft = yface_flux<LL>(g, c, v, i, j0, k, ay, dT);
        for (int jj = j0; jj <= jend; ++jj) {
            double Fb = yface_flux<LL>(g, c, v, i, jj + 1, k, ay, dT);
            const int q = gidx(g, i, jj, k);
            const int cl0 = lmask(g, i, jj, k), clp = lmask(g, i, jj + 1, k);
            const double dtv = LL ? dT / vol<LL>(g, i, jj, k) : dtv0;
            const double ayp = LL ? Aym<LL>(g, i, jj + 1, k) : ay, ay0 = LL ? Aym<LL>(g, i, jj, k) : ay;
            const double ftr = jl_mulb(jl_mulb(ayp * v[q + g.Gx] - ay0 * v[q], clp), cl0);
            double dG = jl_mulb(jl_mulb(Fb - Ft, clp), cl0);
            ttb[t * G + q] = c[q] - dtv * (dG - tr[t * G + q] * ftr);
            Ft = Fb;
        }
    }
}

struct ZFinalArgs {
    DGrid g;
    const double* gadv;      // 14 × G, advective tendency from k_sweep_z
    const double* tr;        // 14 × G, current tracers
    const double* ttb;       // 14 × G, tracer_temp after x and y
    double* tr_next;         // 14 × G
    const double* w;
    double dT;
    pi_bgc_params b;
    int diffuse;             // κh or κv nonzero
    int any_bc;
    const FluxBCDev* bcs;    // [14][6]
    int64_t iter;
    // particle contributions (plk)
    const SpcDev* spc;
    long long C;
    const uint32_t* off;
    const uint32_t* gid_sorted;
    const uint8_t* evk;
    const double* loss;
    const double* contrib;
    int nsp;
    const uint32_t* err;
};

__device__ __forceinline__ double getbc_dev(const FluxBCDev& b, int a, int c, int64_t it) {
    if (b.kind == PI_BC_CONST) return b.v[0];
    if (b.kind == PI_BC_ARRAY2D) return b.v[(a - 1) + (long long)b.n1 * (c - 1)];
    const int64_t t = it < 1 ? 1 : (it > b.nt ? b.nt : it);   // the host rejects steps past nt
    return b.v[(a - 1) + (long long)b.n1 * ((c - 1) + (long long)b.n2 * (t - 1))];
}

#define SWZ_L 8
#define SWZ_TZ 4
// z sweep of multi_dim_z then calc_tracer_tendency!: Gc_adv = tracer_temp - tracer, written to
// `gadv`. Each thread walks SWZ_L levels of one column carrying the z face flux, tracer by tracer;
// levels outside the interior are read through the clamped map of the Bounded halo fill.
__device__ __forceinline__ double zface_flux(const DGrid& g, const double* __restrict__ c,
                                             const double* __restrict__ w, int i, int j, int f,
                                             int qcol, int slab, double az, double dT) {
    if (f == g.Nz + g.Hz + 1) return 0.0;                      // fill_halo_bottom_Gc! (Bounded)
    FaceCoef fc = face_coef(w[qcol + (f - 1) * slab], az, dzC1(g, f), dT);
    auto lev = [&](int kk) { return qcol + (wrap_axis(kk, g.Nz, g.Hz, PI_BOUNDED) - 1) * slab; };
    return flux_z_c(fc, c[lev(f - 2)], c[lev(f - 1)], c[lev(f)], c[lev(f + 1)], lmask(g, i, j, f - 2),
                    lmask(g, i, j, f - 1), lmask(g, i, j, f), lmask(g, i, j, f + 1));
}

template <bool LL>
__global__ void __launch_bounds__(32 * SWZ_TZ, 8) k_sweep_z(DGrid g, const double* __restrict__ tr,
                                                         const double* __restrict__ ttb,
                                                         double* __restrict__ gadv,
                                                         const double* __restrict__ w, double dT,
                                                         const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    const int i = blockIdx.x * 32 + threadIdx.x + 1 + g.Hx;
    const int j = blockIdx.y + 1 + g.Hy;
    const int k0 = (blockIdx.z * SWZ_TZ + threadIdx.y) * SWZ_L + 1 + g.Hz;
    if (i > g.Nx + g.Hx || k0 > g.Nz + g.Hz) return;
    const int kend = min(k0 + SWZ_L - 1, g.Nz + g.Hz);
    const long long G = g.G;
    const double az = Azm<LL>(g, i, j);
    const int slab = g.Gx * g.Gy;
    const int qcol = gidx(g, i, j, 1);
#pragma unroll 1
    for (int t = 0; t < PI_NTRACERS; ++t) {
        const double* c = ttb + t * G;
        double Ft = zface_flux(g, c, w, i, j, k0, qcol, slab, az, dT);
        for (int k = k0; k <= kend; ++k) {
            double Fb = zface_flux(g, c, w, i, j, k + 1, qcol, slab, az, dT);
            const int q = qcol + (k - 1) * slab;
            const int cl0 = lmask(g, i, j, k), clp = lmask(g, i, j, k + 1);
            const double ftr = jl_mulb(jl_mulb(az * w[q] - az * w[q + slab], clp), cl0);
            const double dG = jl_mulb(jl_mulb(Ft - Fb, clp), cl0);
            const double cc = tr[t * G + q];
            const double ct = c[q] - dT / vol<LL>(g, i, j, k) * (dG - cc * ftr);
            gadv[t * G + q] = ct - cc;                          // calc_tracer_tendency!
            Ft = Fb;
        }
    }
}

template <bool LL, bool IRON>
__device__ __forceinline__ void z_final_cell(const ZFinalArgs& a, int i, int j, int k, int q, double volk, double* Gc);

// Per interior cell: diffusion, sinking, forcing, flux BCs, particle terms and apply_tendency!
// on top of the advective tendency of k_sweep_z (tracer_update.jl:22-43).
template <bool LL, bool IRON = false>
__global__ void __launch_bounds__(128, 6) k_tracer_tail(ZFinalArgs a) {
    const DGrid& g = a.g;
    if (*a.err & PI_DEVERR_CAPACITY) return;
    const int i = blockIdx.x * 128 + threadIdx.x + 1 + g.Hx;
    const int j = blockIdx.y + 1 + g.Hy;
    const int k = blockIdx.z + 1 + g.Hz;
    if (i > g.Nx + g.Hx) return;
    const int q = gidx(g, i, j, k);
    const long long G = g.G;
    double Gc[PI_NTRACERS];
#pragma unroll
    for (int t = 0; t < PI_NTRACERS; ++t) Gc[t] = a.gadv[t * G + q];
    z_final_cell<LL, IRON>(a, i, j, k, q, vol<LL>(g, i, j, k), Gc);
}

// The rest of tracer_update! for one interior cell, given its advective tendency Gc.
template <bool LL, bool IRON>
__device__ __forceinline__ void z_final_cell(const ZFinalArgs& a, int i, int j, int k, int q, double volk, double* Gc) {
    const DGrid& g = a.g;
    const long long G = g.G;
    const double dT = a.dT;
    const double az = Azm<LL>(g, i, j);
    const int slab = g.Gx * g.Gy;
    const pi_bgc_params& b = a.b;
    // tracer_diffusion! (κ∇², tracer_diffusion.jl:1-21) on the original tracer
    if (a.diffuse) {
        double kx = b.kappa_h, ky = b.kappa_h, kz = b.kappa_v;
        int li = lmask(g, i, j, k);
#pragma unroll
        for (int n = 0; n < PI_NTRACERS; ++n) {
            const double* c = a.tr + n * G;
            auto dx0 = [&](int ii) { return jl_mulb(jl_mulb(c[gidx(g, ii, j, k)] - c[gidx(g, ii - 1, j, k)], lmask(g, ii, j, k)), lmask(g, ii - 1, j, k)); };
            auto dy0 = [&](int jj) { return jl_mulb(jl_mulb(c[gidx(g, i, jj, k)] - c[gidx(g, i, jj - 1, k)], lmask(g, i, jj, k)), lmask(g, i, jj - 1, k)); };
            auto dz0 = [&](int kk) { return jl_mulb(jl_mulb(c[gidx(g, i, j, kk - 1)] - c[gidx(g, i, j, kk)], lmask(g, i, j, kk)), lmask(g, i, j, kk - 1)); };
            double fx1 = kx * Axm<LL>(g, i + 1, j, k) * (dx0(i + 1) / dxFm<LL>(g, i + 1, j)), fx0 = kx * Axm<LL>(g, i, j, k) * (dx0(i) / dxFm<LL>(g, i, j));
            double fy1 = ky * Aym<LL>(g, i, j + 1, k) * (dy0(j + 1) / dyFm<LL>(g, i, j + 1)), fy0 = ky * Aym<LL>(g, i, j, k) * (dy0(j) / dyFm<LL>(g, i, j));
            double fz0 = kz * az * (dz0(k) / dzF1(g, k)), fz1 = kz * az * (dz0(k + 1) / dzF1(g, k + 1));
            double ax_ = jl_mulb(jl_mulb(fx1 - fx0, lmask(g, i + 1, j, k)), li);
            double ay_ = jl_mulb(jl_mulb(fy1 - fy0, lmask(g, i, j + 1, k)), li);
            double az_ = jl_mulb(jl_mulb(fz0 - fz1, lmask(g, i, j, k + 1)), li);
            double lap = 1.0 / volk * (ax_ + ay_ + az_);
            Gc[n] = Gc[n] + lap * dT;
        }
    }
    // tracer_sinking! (tracer_sinking.jl:1-42); flux_sink is zero on k <= Hz and k >= Nz+Hz
    {
        auto sink = [&](int n, double ws) {
            const double* c = a.tr + n * G;
            double fup = (k - 1 <= g.Hz || k - 1 >= g.Nz + g.Hz) ? 0.0 : ws * c[q - slab];
            double fdn = (k >= g.Nz + g.Hz) ? 0.0 : ws * c[q];
            return (fup - fdn) / dzC1(g, k - g.Hz) * dT;
        };
        Gc[PI_PFe_inorg] = Gc[PI_PFe_inorg] + sink(PI_PFe_inorg, b.w_sink_inorg);
        Gc[PI_Dust] = Gc[PI_Dust] + sink(PI_Dust, b.w_sink_inorg);
        Gc[PI_PFe_bio] = Gc[PI_PFe_bio] + sink(PI_PFe_bio, b.w_sink_org);
    }
    // tracer_forcing! (tracer_forcings.jl:2-50) on max(0, tracer)
    {
        double T[PI_NTRACERS];
#pragma unroll
        for (int n = 0; n < PI_NTRACERS; ++n) T[n] = jl_max(0.0, a.tr[n * G + q]);
        Gc[PI_DIC] = Gc[PI_DIC] + T[PI_DOC] * b.kDOC * dT;
        Gc[PI_DOC] = Gc[PI_DOC] - T[PI_DOC] * b.kDOC * dT + T[PI_POC] * b.kPOC * dT;
        Gc[PI_POC] = Gc[PI_POC] - T[PI_POC] * b.kPOC * dT;
        Gc[PI_NH4] = Gc[PI_NH4] + T[PI_DON] * b.kDON * dT - T[PI_NH4] * b.Nit * dT;
        Gc[PI_NO3] = Gc[PI_NO3] + T[PI_NH4] * b.Nit * dT;
        Gc[PI_DON] = Gc[PI_DON] - T[PI_DON] * b.kDON * dT + T[PI_PON] * b.kPON * dT;
        Gc[PI_PON] = Gc[PI_PON] - T[PI_PON] * b.kPON * dT;
        Gc[PI_PO4] = Gc[PI_PO4] + T[PI_DOP] * b.kDOP * dT;
        Gc[PI_DOP] = Gc[PI_DOP] - T[PI_DOP] * b.kDOP * dT + T[PI_POP] * b.kPOP * dT;
        Gc[PI_POP] = Gc[PI_POP] - T[PI_POP] * b.kPOP * dT;
        Gc[PI_DFe] = Gc[PI_DFe] + T[PI_PFe_bio] * b.kPOC * dT
                   - (b.lambda_POC * T[PI_POC] + b.lambda_min + b.lambda_dust * T[PI_Dust]) * T[PI_DFe] * b.DFeFrac * dT
                   + T[PI_PFe_inorg] * b.kdiss * dT
                   - jl_max((T[PI_DFe] - b.ligand), 0.0) * T[PI_DFe] * b.DFeFrac * b.lambda_Fe * dT;
        Gc[PI_PFe_bio] = Gc[PI_PFe_bio] + T[PI_POC] * T[PI_DFe] * b.DFeFrac * b.lambda_POC * dT
                       - b.kPOC * T[PI_PFe_bio] * dT;
        Gc[PI_PFe_inorg] = Gc[PI_PFe_inorg] - T[PI_PFe_inorg] * b.kdiss * dT
                         + (b.lambda_min + b.lambda_dust * T[PI_Dust]) * T[PI_DFe] * b.DFeFrac * dT
                         + jl_max((T[PI_DFe] - b.ligand), 0.0) * T[PI_DFe] * b.DFeFrac * b.lambda_Fe * dT;
    }
    // apply_bcs! (apply_bcs.jl:4-98), faces in the reference's order
    if (a.any_bc) {
        int ii = i - g.Hx, jj = j - g.Hy, kk = k - g.Hz;
        double axk = Axm<LL>(g, i, j, k), ayk = Aym<LL>(g, i, j, k);
#pragma unroll
        for (int n = 0; n < PI_NTRACERS; ++n) {
            const FluxBCDev* B = a.bcs + n * 6;
            if (B[PI_WEST].kind && i == 1 + g.Hx) Gc[n] += getbc_dev(B[PI_WEST], jj, kk, a.iter) * dT * axk / volk;
            if (B[PI_EAST].kind && i == g.Nx + g.Hx) Gc[n] -= getbc_dev(B[PI_EAST], jj, kk, a.iter) * dT * axk / volk;
            if (B[PI_SOUTH].kind && j == 1 + g.Hy) Gc[n] += getbc_dev(B[PI_SOUTH], ii, kk, a.iter) * dT * ayk / volk;
            if (B[PI_NORTH].kind && j == g.Ny + g.Hy) Gc[n] -= getbc_dev(B[PI_NORTH], ii, kk, a.iter) * dT * ayk / volk;
            if (B[PI_BOTTOM].kind && k == g.Nz + g.Hz) Gc[n] += getbc_dev(B[PI_BOTTOM], ii, jj, a.iter) * dT * az / volk;
            if (B[PI_TOP].kind && k == 1 + g.Hz) Gc[n] -= getbc_dev(B[PI_TOP], ii, jj, a.iter) * dT * az / volk;
        }
    }
    // plk: per-cell particle losses and consumption in reference summation order
    double plk_DIC = 0.0, plk_NH4 = 0.0, plk_NO3 = 0.0, plk_PO4 = 0.0, plk_DOC = 0.0;
    double plk_DON = 0.0, plk_DOP = 0.0, plk_POC = 0.0, plk_PON = 0.0, plk_POP = 0.0;
    double plk_DFe = 0.0, plk_PFe = 0.0;         // IronEnergyMode only
    {
        uint32_t p0 = a.off[q], p1 = a.off[q + 1];
        uint32_t p = p0;
        while (p < p1) {
            uint32_t s = a.gid_sorted[p] / (uint32_t)a.C;
            uint32_t e = p;
            while (e < p1 && a.gid_sorted[e] / (uint32_t)a.C == s) ++e;
            for (int pass = 1; pass <= 2; ++pass)
                for (uint32_t r = p; r < e; ++r)
                    if (a.evk[r] == pass) {
                        if (IRON) {                  // NH4, NO3, DOC, DON, DOP, DFe, POC, PON, POP, PFe_bio
                            const double* L = a.loss + (long long)r * 10;
                            plk_NH4 += L[0]; plk_NO3 += L[1]; plk_DOC += L[2]; plk_DON += L[3]; plk_DOP += L[4];
                            plk_DFe += L[5]; plk_POC += L[6]; plk_PON += L[7]; plk_POP += L[8]; plk_PFe += L[9];
                        } else {
                            const double* L = a.loss + (long long)r * 6;
                            plk_DOC += L[0]; plk_DON += L[1]; plk_DOP += L[2];
                            plk_POC += L[3]; plk_PON += L[4]; plk_POP += L[5];
                        }
                    }
            for (uint32_t r = p; r < e; ++r) {
                const double* K = a.contrib + (long long)r * 5;
                if (IRON) { plk_DIC += K[0]; plk_NH4 += K[1]; plk_NO3 += K[2]; plk_PO4 += K[3]; plk_DFe += K[4]; }
                else { plk_DIC += K[0]; plk_DOC += K[1]; plk_NH4 += K[2]; plk_NO3 += K[3]; plk_PO4 += K[4]; }
            }
            p = e;
        }
    }
    // apply_tendency!: tracer += Gc + plk / volume
#pragma unroll
    for (int n = 0; n < PI_NTRACERS; ++n) {
        double pk = n == PI_DIC ? plk_DIC : n == PI_NH4 ? plk_NH4 : n == PI_NO3 ? plk_NO3 : n == PI_PO4 ? plk_PO4
                  : n == PI_DOC ? plk_DOC : n == PI_DON ? plk_DON : n == PI_DOP ? plk_DOP : n == PI_POC ? plk_POC
                  : n == PI_PON ? plk_PON : n == PI_POP ? plk_POP
                  : (IRON && n == PI_DFe) ? plk_DFe : (IRON && n == PI_PFe_bio) ? plk_PFe : 0.0;
        a.tr_next[n * G + q] = a.tr[n * G + q] + (Gc[n] + pk / volk);
    }
}

// fill_halo_tracer! in three passes (x, y, z). Each thread owns one line along the axis and
// reads all its source values before writing, as Julia's broadcast unaliases views.
template <int AXIS>
__global__ void k_halo(DGrid g, double* __restrict__ f, int nfields, const uint32_t* err) {
    int a = blockIdx.x * blockDim.x + threadIdx.x + 1;   // first transverse index
    int b = blockIdx.y + 1;                              // second transverse index
    int n = blockIdx.z;
    int na = AXIS == 0 ? g.Gy : g.Gx;
    if (a > na || n >= nfields) return;
    if (err && (*err & PI_DEVERR_CAPACITY)) return;
    int N = AXIS == 0 ? g.Nx : AXIS == 1 ? g.Ny : g.Nz;
    int H = AXIS == 0 ? g.Hx : AXIS == 1 ? g.Hy : g.Hz;
    int topo = AXIS == 0 ? g.tx : AXIS == 1 ? g.ty : g.tz;
    double* c = f + (long long)n * g.G;
    auto at = [&](int t) -> double& {
        if (AXIS == 0) return c[gidx(g, t, a, b)];
        if (AXIS == 1) return c[gidx(g, a, t, b)];
        return c[gidx(g, a, b, t)];
    };
    double wv[8], ev[8];
    for (int h = 1; h <= H; ++h) {
        wv[h - 1] = topo == PI_PERIODIC ? at(N + h) : at(H + 1);
        ev[h - 1] = topo == PI_PERIODIC ? at(H + h) : at(N + H);
    }
    for (int h = 1; h <= H; ++h) {
        at(h) = wv[h - 1];
        at(N + H + h) = ev[h - 1];
    }
}

// Interior array (reference layout nx×ny×nz, x fastest) into a halo-padded field at offset
// (Hx, Hy, Hz): copy_interior! / copy_interior_u! (Simulation/utils.jl:13-34).
__global__ void k_scatter_interior(DGrid g, double* __restrict__ dst, const double* __restrict__ src,
                                   int nx, int ny, int nz) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)nx * ny * nz;
    if (q >= n) return;
    int i = (int)(q % nx);
    long long r = q / nx;
    int j = (int)(r % ny);
    int k = (int)(r / ny);
    dst[gidx(g, i + 1 + g.Hx, j + 1 + g.Hy, k + 1 + g.Hz)] = src[q];
}

// Velocity halo rule along one axis (fill_halo_u/v/w!, halo_regions.jl:64-99) when the field is a
// face field on that axis and the axis is Bounded: the high halo copies the extra face N+H+1.
// Otherwise the tracer rule. One thread per line; sources are read before writes.
template <int AXIS>
__global__ void k_halo_vel(DGrid g, double* __restrict__ c, int face_axis) {
    int a = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int b = blockIdx.y + 1;
    int na = AXIS == 0 ? g.Gy : g.Gx;
    if (a > na) return;
    int N = AXIS == 0 ? g.Nx : AXIS == 1 ? g.Ny : g.Nz;
    int H = AXIS == 0 ? g.Hx : AXIS == 1 ? g.Hy : g.Hz;
    int topo = AXIS == 0 ? g.tx : AXIS == 1 ? g.ty : g.tz;
    auto at = [&](int t) -> double& {
        if (AXIS == 0) return c[gidx(g, t, a, b)];
        if (AXIS == 1) return c[gidx(g, a, t, b)];
        return c[gidx(g, a, b, t)];
    };
    double wv[8], ev[8];
    int velrule = (face_axis == AXIS) && topo == PI_BOUNDED;
    for (int h = 1; h <= H; ++h) {
        wv[h - 1] = topo == PI_PERIODIC ? at(N + h) : at(H + 1);
        ev[h - 1] = topo == PI_PERIODIC ? at(H + h) : at(N + H);
    }
    double face = velrule ? at(N + H + 1) : 0.0;
    for (int h = 1; h <= H; ++h) at(h) = wv[h - 1];
    if (velrule) {
        for (int h = N + H + 2; h <= N + 2 * H; ++h) at(h) = face;
    } else {
        for (int h = 1; h <= H; ++h) at(N + H + h) = ev[h - 1];
    }
}

// Active individuals of one species (calc_active_individuals, models.jl:157-164).
// Index of the first non-finite value of a[0, n) (atomicMin into *first, which starts at ~0).
__global__ void k_first_nonfinite(const double* __restrict__ a, long long n, unsigned long long* first) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        if (!isfinite(a[q])) atomicMin(first, (unsigned long long)q);
}

// First active slot of a species with a non-finite Float64 attribute.
__global__ void k_first_nonfinite_inds(SpcDev s, long long C, unsigned long long* first) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < C; q += (long long)gridDim.x * blockDim.x) {
        if (!(s.flags[q] & FL_AC)) continue;
        const double v[11] = { s.x[q], s.y[q], s.z[q], s.Sz[q], s.Bm[q], s.Cq[q], s.Nq[q], s.Pq[q], s.Chl[q], s.gen[q], s.age[q] };
        bool bad = false;
        for (int k = 0; k < 11; ++k) bad |= !isfinite(v[k]);
        if (s.PRO) {                                  // MacroMolecularMode pools
            const double w[6] = { s.PRO[q], s.DNA[q], s.RNA[q], s.CH[q], s.NST[q], s.PST[q] };
            for (int k = 0; k < 6; ++k) bad |= !isfinite(w[k]);
        }
        if (bad) atomicMin(first, (unsigned long long)q);
    }
}

// Mass budgets (no counterpart in the reference): block partials of the interior Σ vol·c of the
// carbon (DIC+DOC+POC), nitrogen (NH4+NO3+DON+PON) and phosphorus (PO4+DOP+POP) tracers, and of the
// active individuals' C (Bm+Cq), N (Bm·R_NC+Nq) and P (Bm·R_PC+Pq). Each block sums a fixed set of
// cells (slots) in a fixed order, so the result does not depend on the run.
__device__ __forceinline__ void block_sum3(double c, double n, double p, double* partial) {
    __shared__ double sh[3][256];
    sh[0][threadIdx.x] = c; sh[1][threadIdx.x] = n; sh[2][threadIdx.x] = p;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) for (int r = 0; r < 3; ++r) sh[r][threadIdx.x] += sh[r][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) for (int r = 0; r < 3; ++r) partial[blockIdx.x * 3 + r] = sh[r][0];
}
__global__ void __launch_bounds__(256) k_budget_cells(DGrid g, const double* __restrict__ tr, double* __restrict__ partial) {
    double c = 0.0, n = 0.0, p = 0.0;
    const long long V = (long long)g.Nx * g.Ny * g.Nz, G = g.G;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < V; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % g.Nx) + 1 + g.Hx;
        const long long r = q / g.Nx;
        const int j = (int)(r % g.Ny) + 1 + g.Hy, k = (int)(r / g.Ny) + 1 + g.Hz;
        const long long cq = gidx(g, i, j, k);
        const double vol = g.mVol ? pib::vol<true>(g, i, j, k) : pib::vol<false>(g, i, j, k);
        c += vol * (tr[PI_DIC * G + cq] + tr[PI_DOC * G + cq] + tr[PI_POC * G + cq]);
        n += vol * (tr[PI_NH4 * G + cq] + tr[PI_NO3 * G + cq] + tr[PI_DON * G + cq] + tr[PI_PON * G + cq]);
        p += vol * (tr[PI_PO4 * G + cq] + tr[PI_DOP * G + cq] + tr[PI_POP * G + cq]);
    }
    block_sum3(c, n, p, partial);
}
__global__ void __launch_bounds__(256) k_budget_inds(SpcDev s, long long C, double R_NC, double R_PC, double* __restrict__ partial) {
    double c = 0.0, n = 0.0, p = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < C; q += (long long)gridDim.x * blockDim.x) {
        if (!(s.flags[q] & FL_AC)) continue;
        const double Bm = s.Bm[q];
        c += Bm + s.Cq[q];
        n += Bm * R_NC + s.Nq[q];
        p += Bm * R_PC + s.Pq[q];
    }
    block_sum3(c, n, p, partial);
}

// MacroMolecularMode individuals: total_C/N/P_biomass (plankton_generation.jl:82-93) of the active ones
__global__ void __launch_bounds__(256) k_budget_inds_macro(SpcDev s, long long C, pi_macro_params mp, double* __restrict__ partial) {
    double c = 0.0, n = 0.0, p = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < C; q += (long long)gridDim.x * blockDim.x) {
        if (!(s.flags[q] & FL_AC)) continue;
        c += m_totC(s.PRO[q], s.DNA[q], s.RNA[q], s.CH[q], s.Chl[q]);
        n += m_totN(s.PRO[q], s.DNA[q], s.RNA[q], s.NST[q], s.Chl[q], mp);
        p += m_totP(s.DNA[q], s.RNA[q], s.PST[q], mp);
    }
    block_sum3(c, n, p, partial);
}

__global__ void k_count_active(const uint8_t* __restrict__ flags, long long C, unsigned long long* out) {
    unsigned long long n = 0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < C; q += (long long)gridDim.x * blockDim.x)
        n += (flags[q] & FL_AC) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(out, n);
}

// After a capacity error the step stops where the reference throws: the tracers keep their
// values, so the buffer that becomes current is a copy of the old one.
__global__ void k_copy_if_err(double* __restrict__ dst, const double* __restrict__ src, long long n,
                              const uint32_t* err) {
    if (!(*err & PI_DEVERR_CAPACITY)) return;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = src[q];
}

}  // namespace pib
