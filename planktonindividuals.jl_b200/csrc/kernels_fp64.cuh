// FP64 plain-form kernels of the model time step (QuotaMode, no abiotic particles).
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
template <int COMP, int HALF>
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
    double d0, d1;
    if (COMP == 0) { d0 = g.dx; d1 = g.dx; }
    else if (COMP == 1) { d0 = g.dy; d1 = g.dy; }
    else { d0 = dzC1(g, k); d1 = dzC1(g, k + 1); }
    return w000 * c000 / d0 + w001 * c001 / d1 + w010 * c010 / d0 + w011 * c011 / d1
         + w100 * c100 / d0 + w101 * c101 / d1 + w110 * c110 / d0 + w111 * c111 / d1;
}

struct VelPtrs { const double *u0, *v0, *w0, *u1, *v1, *w1; };

// One thread per (species, slot). Writes the new position, the packed cell of find_inds!, the
// binning key and the per-cell count of active individuals.
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
    int ac = P.flags[slot] & FL_AC;
    int oxi, oyi, ozi;
    unpack_cell(g, P.cell[slot], oxi, oyi, ozi);
    // ΔzC at the stored zi + Hz (particle_diffusion.jl:5), checked for every slot
    int kdz = clamp_idx((long long)ozi + g.Hz, 1, g.Gz, err);
    if (!ac) {
        // Inactive slots: every stage multiplies by ac, so positions end as zeros and the cell
        // is (Hx, Hy, Hz).
        if (P.x[slot] != 0.0) P.x[slot] = 0.0;
        if (P.y[slot] != 0.0) P.y[slot] = 0.0;
        if (P.z[slot] != 0.0) P.z[slot] = 0.0;
        P.cell[slot] = pack_cell(g, g.Hx, g.Hy, g.Hz);
        key[gid] = sentinel;
        return;
    }
    const double X = P.x[slot], Y = P.y[slot], Z = P.z[slot];
    const double NX = (double)g.Nx, NY = (double)g.Ny, NZ = (double)g.Nz;
    // stage 1 at vel₀
    double u1 = jl_mulb(itpl<0, 0>(g, vel.u0, vel.u0, X, Y, Z, ac, err), ac);
    double v1 = jl_mulb(itpl<1, 0>(g, vel.v0, vel.v0, X, Y, Z, ac, err), ac);
    double w1 = jl_mulb(itpl<2, 0>(g, vel.w0, vel.w0, X, Y, Z, ac, err), ac);
    double u2 = u1, v2 = v1, w2 = w1;
    double vx = X + jl_mulb(0.5 * u1 * dT, ac);
    double vy = Y + jl_mulb(0.5 * v1 * dT, ac);
    double vz = Z - jl_mulb(0.5 * w1 * dT, ac);
    vx = jl_mulb(bc_pos(vx, NX, g.tx), ac); vy = jl_mulb(bc_pos(vy, NY, g.ty), ac); vz = jl_mulb(bc_pos(vz, NZ, g.tz), ac);
    // stage 2 at vel½
    u1 = jl_mulb(itpl<0, 1>(g, vel.u0, vel.u1, vx, vy, vz, ac, err), ac);
    v1 = jl_mulb(itpl<1, 1>(g, vel.v0, vel.v1, vx, vy, vz, ac, err), ac);
    w1 = jl_mulb(itpl<2, 1>(g, vel.w0, vel.w1, vx, vy, vz, ac, err), ac);
    u2 = u2 + u1 * 2.0; v2 = v2 + v1 * 2.0; w2 = w2 + w1 * 2.0;
    vx = X + jl_mulb(0.5 * u1 * dT, ac);
    vy = Y + jl_mulb(0.5 * v1 * dT, ac);
    vz = Z - jl_mulb(0.5 * w1 * dT, ac);
    vx = jl_mulb(bc_pos(vx, NX, g.tx), ac); vy = jl_mulb(bc_pos(vy, NY, g.ty), ac); vz = jl_mulb(bc_pos(vz, NZ, g.tz), ac);
    // stage 3 at vel½
    u1 = jl_mulb(itpl<0, 1>(g, vel.u0, vel.u1, vx, vy, vz, ac, err), ac);
    v1 = jl_mulb(itpl<1, 1>(g, vel.v0, vel.v1, vx, vy, vz, ac, err), ac);
    w1 = jl_mulb(itpl<2, 1>(g, vel.w0, vel.w1, vx, vy, vz, ac, err), ac);
    u2 = u2 + u1 * 2.0; v2 = v2 + v1 * 2.0; w2 = w2 + w1 * 2.0;
    vx = X + jl_mulb(1.0 * u1 * dT, ac);
    vy = Y + jl_mulb(1.0 * v1 * dT, ac);
    vz = Z - jl_mulb(1.0 * w1 * dT, ac);
    vx = jl_mulb(bc_pos(vx, NX, g.tx), ac); vy = jl_mulb(bc_pos(vy, NY, g.ty), ac); vz = jl_mulb(bc_pos(vz, NZ, g.tz), ac);
    // stage 4 at vel₁
    u1 = jl_mulb(itpl<0, 0>(g, vel.u1, vel.u1, vx, vy, vz, ac, err), ac);
    v1 = jl_mulb(itpl<1, 0>(g, vel.v1, vel.v1, vx, vy, vz, ac, err), ac);
    w1 = jl_mulb(itpl<2, 0>(g, vel.w1, vel.w1, vx, vy, vz, ac, err), ac);
    u2 = u2 + u1; v2 = v2 + v1; w2 = w2 + w1;
    u2 = u2 / 6.0; v2 = v2 / 6.0; w2 = w2 / 6.0;
    double x = X + jl_mulb(1.0 * u2 * dT, ac);
    double y = Y + jl_mulb(1.0 * v2 * dT, ac);
    double z = Z - jl_mulb(1.0 * w2 * dT, ac);
    x = jl_mulb(bc_pos(x, NX, g.tx), ac); y = jl_mulb(bc_pos(y, NY, g.ty), ac); z = jl_mulb(bc_pos(z, NZ, g.tz), ac);
    // diffusion: rnd ∈ [0,1) → (rnd - 0.5) * 2 → · √(κΔT) / Δ
    double r0, r1, r2;
    pi_draw3(seed, iter, (uint32_t)s, PI_DRAW_DIFFUSION, (uint32_t)slot, &r0, &r1, &r2);
    r0 = (r0 - 0.5) * 2.0; r1 = (r1 - 0.5) * 2.0; r2 = (r2 - 0.5) * 2.0;
    r0 = r0 * sqrt(kappa_h * dT) / g.dx;
    r1 = r1 * sqrt(kappa_h * dT) / g.dy;
    r2 = r2 * sqrt(kappa_v * dT) / dzC1(g, kdz);
    x = x + jl_mulb(r0, ac); y = y + jl_mulb(r1, ac); z = z + jl_mulb(r2, ac);
    x = jl_mulb(bc_pos(x, NX, g.tx), ac); y = jl_mulb(bc_pos(y, NY, g.ty), ac); z = jl_mulb(bc_pos(z, NZ, g.tz), ac);
    P.x[slot] = x; P.y[slot] = y; P.z[slot] = z;
    // find_inds!
    int xi = clamp_idx(jl_trunc(jl_mulb(x + 1.0, ac)) + g.Hx, 1, g.Gx, err);
    int yi = clamp_idx(jl_trunc(jl_mulb(y + 1.0, ac)) + g.Hy, 1, g.Gy, err);
    int zi = clamp_idx(jl_trunc(jl_mulb(z + 1.0, ac)) + g.Hz, 1, g.Gz, err);
    P.cell[slot] = pack_cell(g, xi, yi, zi);
    int c = gidx(g, xi, yi, zi);
    key[gid] = (uint32_t)c;
    atomicAdd(&cnt[c], 1u);
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
        double atten = (chl / vol(g, kk) * kc + kw) * dzF1(g, kk);
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

// Applies last step's grazing/mortality decisions, writes the loss contributions of the
// individuals lost, the division/free flags for the slot scan and the graz/mort/dvid diags.
__global__ void k_decide(DGrid g, SpcDev P, pi_quota_params p, long long C, int s,
                         const int32_t* __restrict__ pos, double* __restrict__ loss,
                         uint8_t* __restrict__ evk, unsigned long long* __restrict__ flag64,
                         double* __restrict__ d_graz, double* __restrict__ d_mort,
                         double* __restrict__ d_dvid, uint32_t* err) {
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
            double Bm = P.Bm[slot], Cq = P.Cq[slot], Nq = P.Nq[slot], Pq = P.Pq[slot];
            double* L = loss + e * 6;
            L[0] = jl_mulb((Bm + Cq) * fC, 1) * 1.0;                  // DOC
            L[1] = jl_mulb((Bm * p.R_NC + Nq) * fN, 1) * 1.0;         // DON
            L[2] = jl_mulb((Bm * p.R_PC + Pq) * fP, 1) * 1.0;         // DOP
            L[3] = jl_mulb((Bm + Cq) * (1.0 - fC), 1) * 1.0;          // POC
            L[4] = jl_mulb((Bm * p.R_NC + Nq) * (1.0 - fN), 1) * 1.0; // PON
            L[5] = jl_mulb((Bm * p.R_PC + Pq) * (1.0 - fP), 1) * 1.0; // POP
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
                        uint32_t* ndiv, uint32_t* err, int64_t* err_iter, int64_t iter) {
    long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    unsigned long long tot = rank64[C - 1] + flag64[C - 1];
    unsigned long long tdiv = tot >> 32, tfree = tot & 0xffffffffull;
    if (tdiv > tfree) {
        if (slot == 0) { *ndiv = 0; *err_iter = iter; }
        __threadfence();
        // every thread sees the same totals; one flag write is enough but all are harmless
        if (slot == 0) set_err(err, PI_DEVERR_CAPACITY);
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
__global__ void k_daughters(SpcDev P, const int32_t* __restrict__ divlist,
                            const int32_t* __restrict__ freelist, const uint32_t* ndiv,
                            const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    uint32_t n = *ndiv;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        long long p = divlist[k], d = freelist[k];
        const double h = (2.0 - 1.0) / 2.0;
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
                             double* __restrict__ d_num, const uint32_t* err) {
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
    // diags_proc!(num, ac, ac) at the slot's (possibly stale) cell
    atomicAdd(&d_num[c], 1.0);
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

// x sweep: calc_Gcˣ + fill_halo_Gcs + multi_dim_x on tracer_temp = tracer.
__global__ void k_sweep_x(DGrid g, const double* __restrict__ tr, double* __restrict__ tta,
                          const double* __restrict__ u, double dT, const uint32_t* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1 + g.Hx;
    int j = blockIdx.y + 1 + g.Hy;
    int k = blockIdx.z + 1 + g.Hz;
    if (i > g.Nx + g.Hx) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    const long long G = g.G;
    int q = gidx(g, i, j, k);
    double ax = g.dy * dzF1(g, k);
    double volk = vol(g, k);
    double ui = u[q], up = u[q + 1];
    int last = (i == g.Nx + g.Hx);
    int lm2 = lmask(g, i - 2, j, k), lm1 = lmask(g, i - 1, j, k), l0 = lmask(g, i, j, k);
    int lp1 = lmask(g, i + 1, j, k), lp2 = last ? 0 : lmask(g, i + 2, j, k);
    int qw = gidx(g, g.Hx + 1, j, k);
    double ftr = jl_mulb(jl_mulb(ax * up - ax * ui, lp1), l0);
    for (int n = 0; n < PI_NTRACERS; ++n) {
        const double* c = tr + n * G;
        double cm2 = c[q - 2], cm1 = c[q - 1], c0 = c[q], cp1 = c[q + 1];
        double Fi = dst3_flux_xy(cm2, cm1, c0, cp1, lm2, lm1, l0, lp1, ui, ax, g.dx, dT);
        double Fp;
        if (!last) {
            Fp = dst3_flux_xy(cm1, c0, cp1, c[q + 2], lm1, l0, lp1, lp2, up, ax, g.dx, dT);
        } else if (g.tx == PI_PERIODIC) {
            Fp = dst3_flux_xy(c[qw - 2], c[qw - 1], c[qw], c[qw + 1],
                              lmask(g, g.Hx - 1, j, k), lmask(g, g.Hx, j, k), lmask(g, g.Hx + 1, j, k),
                              lmask(g, g.Hx + 2, j, k), u[qw], ax, g.dx, dT);
        } else {
            Fp = 0.0;
        }
        double dG = jl_mulb(jl_mulb(Fp - Fi, lp1), l0);
        tta[n * G + q] = c0 - dT / volk * (dG - c0 * ftr);
    }
}

// y sweep on tracer_temp after x; original tracer c in the update term.
__global__ void k_sweep_y(DGrid g, const double* __restrict__ tr, const double* __restrict__ tta,
                          double* __restrict__ ttb, const double* __restrict__ v, double dT,
                          const uint32_t* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1 + g.Hx;
    int j = blockIdx.y + 1 + g.Hy;
    int k = blockIdx.z + 1 + g.Hz;
    if (i > g.Nx + g.Hx) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    const long long G = g.G;
    int q = gidx(g, i, j, k);
    int last = (j == g.Ny + g.Hy);
    double ay = g.dx * dzF1(g, k);
    double volk = vol(g, k);
    double vj = v[q], vp = v[q + g.Gx];
    int jm2 = wrap_axis(j - 2, g.Ny, g.Hy, g.ty), jm1 = wrap_axis(j - 1, g.Ny, g.Hy, g.ty);
    int jp1 = wrap_axis(j + 1, g.Ny, g.Hy, g.ty), jp2 = wrap_axis(j + 2, g.Ny, g.Hy, g.ty);
    int lm2 = lmask(g, i, j - 2, k), lm1 = lmask(g, i, j - 1, k), l0 = lmask(g, i, j, k);
    int lp1 = lmask(g, i, j + 1, k), lp2 = last ? 0 : lmask(g, i, j + 2, k);
    double ftr = jl_mulb(jl_mulb(ay * vp - ay * vj, lp1), l0);
    int qm2 = gidx(g, i, jm2, k), qm1 = gidx(g, i, jm1, k), qp1 = gidx(g, i, jp1, k), qp2 = gidx(g, i, jp2, k);
    int js = g.Hy + 1;
    int qs = gidx(g, i, js, k);
    int qsm2 = gidx(g, i, wrap_axis(js - 2, g.Ny, g.Hy, g.ty), k);
    int qsm1 = gidx(g, i, wrap_axis(js - 1, g.Ny, g.Hy, g.ty), k);
    int qsp1 = gidx(g, i, wrap_axis(js + 1, g.Ny, g.Hy, g.ty), k);
    for (int n = 0; n < PI_NTRACERS; ++n) {
        const double* c = tta + n * G;
        double cm2 = c[qm2], cm1 = c[qm1], c0 = c[q], cp1 = c[qp1];
        double Fj = dst3_flux_xy(cm2, cm1, c0, cp1, lm2, lm1, l0, lp1, vj, ay, g.dy, dT);
        double Fp;
        if (!last) {
            Fp = dst3_flux_xy(cm1, c0, cp1, c[qp2], lm1, l0, lp1, lp2, vp, ay, g.dy, dT);
        } else if (g.ty == PI_PERIODIC) {
            Fp = dst3_flux_xy(c[qsm2], c[qsm1], c[qs], c[qsp1],
                              lmask(g, i, js - 2, k), lmask(g, i, js - 1, k), lmask(g, i, js, k),
                              lmask(g, i, js + 1, k), v[qs], ay, g.dy, dT);
        } else {
            Fp = 0.0;
        }
        double dG = jl_mulb(jl_mulb(Fp - Fj, lp1), l0);
        double cc = tr[n * G + q];
        ttb[n * G + q] = c0 - dT / volk * (dG - cc * ftr);
    }
}

struct ZFinalArgs {
    DGrid g;
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
    return b.v[(a - 1) + (long long)b.n1 * ((c - 1) + (long long)b.n2 * (it - 1))];
}

// z sweep + calc_tracer_tendency + diffusion + sinking + forcing + flux BCs + apply_tendency.
// One thread per water column (i, j), walking k downward so each z face flux is computed once.
__global__ void k_sweep_z_final(ZFinalArgs a) {
    const DGrid& g = a.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1 + g.Hx;
    int j = blockIdx.y + 1 + g.Hy;
    if (i > g.Nx + g.Hx) return;
    if (*a.err & PI_DEVERR_CAPACITY) return;
    const long long G = g.G;
    const double dT = a.dT;
    const pi_bgc_params& b = a.b;
    const double az = g.dx * g.dy;
    const int k0 = g.Hz + 1, k1 = g.Nz + g.Hz;
    double Ftop[PI_NTRACERS];
    // flux at the top face of cell k0
    {
        int k = k0;
        double wk = a.w[gidx(g, i, j, k)];
        int lm2 = lmask(g, i, j, k - 2), lm1 = lmask(g, i, j, k - 1), l0 = lmask(g, i, j, k), lp1 = lmask(g, i, j, k + 1);
        int km2 = gidx(g, i, j, wrap_axis(k - 2, g.Nz, g.Hz, PI_BOUNDED));
        int km1 = gidx(g, i, j, wrap_axis(k - 1, g.Nz, g.Hz, PI_BOUNDED));
        int kc = gidx(g, i, j, k);
        int kp1 = gidx(g, i, j, wrap_axis(k + 1, g.Nz, g.Hz, PI_BOUNDED));
        for (int n = 0; n < PI_NTRACERS; ++n) {
            const double* c = a.ttb + n * G;
            Ftop[n] = dst3_flux_z(c[km2], c[km1], c[kc], c[kp1], lm2, lm1, l0, lp1, wk, az, dzC1(g, k), dT);
        }
    }
    for (int k = k0; k <= k1; ++k) {
        int q = gidx(g, i, j, k);
        double volk = vol(g, k);
        double wk = a.w[q], wp = a.w[q + g.Gx * g.Gy];
        int l0 = lmask(g, i, j, k), lp1 = lmask(g, i, j, k + 1);
        double ftr = jl_mulb(jl_mulb(az * wk - az * wp, lp1), l0);
        double Gc[PI_NTRACERS];
        {
            int last = (k == k1);
            int lm1 = l0, lp2 = last ? 0 : lmask(g, i, j, k + 2);
            int kc = q;
            int kp1 = gidx(g, i, j, wrap_axis(k + 1, g.Nz, g.Hz, PI_BOUNDED));
            int kp2 = gidx(g, i, j, wrap_axis(k + 2, g.Nz, g.Hz, PI_BOUNDED));
            int km1 = gidx(g, i, j, wrap_axis(k - 1, g.Nz, g.Hz, PI_BOUNDED));
            for (int n = 0; n < PI_NTRACERS; ++n) {
                const double* c = a.ttb + n * G;
                double Fb;
                if (!last) {
                    // face k+1: c[k-1], c[k], c[k+1], c[k+2]
                    Fb = dst3_flux_z(c[km1], c[kc], c[kp1], c[kp2], lmask(g, i, j, k - 1), lm1, lp1, lp2,
                                     wp, az, dzC1(g, k + 1), dT);
                } else {
                    Fb = 0.0;   // fill_halo_bottom_Gc! (Bounded)
                }
                double dG = jl_mulb(jl_mulb(Ftop[n] - Fb, lp1), l0);
                double cc = a.tr[n * G + q];
                double ct = c[kc] - dT / volk * (dG - cc * ftr);
                Gc[n] = ct - cc;                         // calc_tracer_tendency!
                Ftop[n] = Fb;
            }
        }
        // tracer_diffusion! (κ∇², tracer_diffusion.jl:1-21) on the original tracer
        if (a.diffuse) {
            double kx = b.kappa_h, ky = b.kappa_h, kz = b.kappa_v;
            double axk = g.dy * dzF1(g, k), ayk = g.dx * dzF1(g, k);
            int li = lmask(g, i, j, k);
            for (int n = 0; n < PI_NTRACERS; ++n) {
                const double* c = a.tr + n * G;
                auto dx0 = [&](int ii) { return jl_mulb(jl_mulb(c[gidx(g, ii, j, k)] - c[gidx(g, ii - 1, j, k)], lmask(g, ii, j, k)), lmask(g, ii - 1, j, k)); };
                auto dy0 = [&](int jj) { return jl_mulb(jl_mulb(c[gidx(g, i, jj, k)] - c[gidx(g, i, jj - 1, k)], lmask(g, i, jj, k)), lmask(g, i, jj - 1, k)); };
                auto dz0 = [&](int kk) { return jl_mulb(jl_mulb(c[gidx(g, i, j, kk - 1)] - c[gidx(g, i, j, kk)], lmask(g, i, j, kk)), lmask(g, i, j, kk - 1)); };
                double fx1 = kx * axk * (dx0(i + 1) / g.dx), fx0 = kx * axk * (dx0(i) / g.dx);
                double fy1 = ky * ayk * (dy0(j + 1) / g.dy), fy0 = ky * ayk * (dy0(j) / g.dy);
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
            const int names[3] = { PI_PFe_inorg, PI_Dust, PI_PFe_bio };
            for (int m = 0; m < 3; ++m) {
                int n = names[m];
                double ws = m < 2 ? b.w_sink_inorg : b.w_sink_org;
                const double* c = a.tr + n * G;
                double fup = (k - 1 <= g.Hz || k - 1 >= g.Nz + g.Hz) ? 0.0 : ws * c[q - g.Gx * g.Gy];
                double fdn = (k >= g.Nz + g.Hz) ? 0.0 : ws * c[q];
                Gc[n] = Gc[n] + (fup - fdn) / dzC1(g, k - g.Hz) * dT;
            }
        }
        // tracer_forcing! (tracer_forcings.jl:2-50) on max(0, tracer)
        {
            double T[PI_NTRACERS];
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
            double axk = g.dy * dzF1(g, k), ayk = g.dx * dzF1(g, k);
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
        double plk[PI_NTRACERS];
        for (int n = 0; n < PI_NTRACERS; ++n) plk[n] = 0.0;
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
                            const double* L = a.loss + (long long)r * 6;
                            plk[PI_DOC] += L[0]; plk[PI_DON] += L[1]; plk[PI_DOP] += L[2];
                            plk[PI_POC] += L[3]; plk[PI_PON] += L[4]; plk[PI_POP] += L[5];
                        }
                for (uint32_t r = p; r < e; ++r) {
                    const double* K = a.contrib + (long long)r * 5;
                    plk[PI_DIC] += K[0]; plk[PI_DOC] += K[1]; plk[PI_NH4] += K[2];
                    plk[PI_NO3] += K[3]; plk[PI_PO4] += K[4];
                }
                p = e;
            }
        }
        for (int n = 0; n < PI_NTRACERS; ++n)            // apply_tendency!
            a.tr_next[n * G + q] = a.tr[n * G + q] + (Gc[n] + plk[n] / volk);
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
