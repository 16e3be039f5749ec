// FP32 form: kernels. Every launch covers all members of a batch; blocks and warps find their
// member through work tables built when the batch is created.
//
// The formulas are those of the FP64 kernels (and of the reference lines they cite) evaluated in
// Float32, with three changes of representation:
//  - a position is an interior cell (ci, cj, ck) plus an in-cell offset in [0, 1): find_inds! is
//    the cell itself, interpolation weights come straight from the offsets, and the precision of a
//    position does not degrade with the size of the grid;
//  - particle→grid sums (Chl for light, consumption, grazing and mortality losses) are 64-bit
//    fixed-point integers added with atomics; integer addition commutes, so the sums do not depend
//    on the order in which individuals are visited and no sort is needed for determinism; pop and
//    the diagnostic counts are exact integer counts;
//  - Sz is not stored: it is Bm / (Cquota Nsuper), as update_cellsize_kernel! sets it;
//  - individuals are stored in a physical order grouped by cell (kept by a periodic counting sort)
//    behind their logical slot numbers: draws are keyed by the logical slot and the division
//    bookkeeping runs on bitmaps over logical slots, so the order changes no result.
// FP64 is used for the fixed-point conversions, the mass budgets and the DST3FL limiter ratio
// where the centred gradient is within a few FP32 ulps of zero.
#pragma once

#include <cstddef>

#include "fp32_internal.h"

namespace p32 {

#define THMAX_F 1.0e20f
#define EPS20_F 1.0e-20f

struct Tab32 {
    const MemberDev* md;
    int nsp;
    const int2* tiles;        // {segment = member*nsp + species, first slot}, F32_TILE slots each
    int ntiles;
    const int* seg_tile0;     // first tile of each segment (nseg + 1 entries)
    const int4* icol; int nicol;  // column warps {m, i0, j, 0}
};

__device__ __forceinline__ int gid3(const MemberDev& m, int i, int j, int k) {   // 1-based, member-local
    return (i - 1) + m.Gx * ((j - 1) + m.Gy * (k - 1));
}
__device__ __forceinline__ int lm32(const MemberDev& m, const uint8_t* __restrict__ lm, int i, int j, int k) {
    return m.all_water ? 1 : (int)lm[m.cell_off + gid3(m, i, j, k)];
}
__device__ __forceinline__ float mulbf(float x, int b) { return b ? x : copysignf(0.0f, x); }
__device__ __forceinline__ void seterr(uint32_t* err, uint32_t bit) { atomicOr(err, bit); }
__device__ __forceinline__ bool stopped(const uint32_t* err) {
    return (*(volatile const uint32_t*)err & F32_ERR_CAPACITY) != 0;
}
__device__ __forceinline__ void seg_of(const Tab32& T, int seg, int& m, int& s) { m = seg / T.nsp; s = seg - m * T.nsp; }

// ------------------------------------------------------------------------------------------
// cells and positions
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void unpack_int(const MemberDev& m, int32_t code, int& ci, int& cj, int& ck) {
    f32_unpack(code, m.cbx, m.cby, ci, cj, ck);
}
__device__ __forceinline__ int32_t pack_int(const MemberDev& m, int ci, int cj, int ck) {
    return f32_pack(ci, cj, ck, m.cbx, m.cby);
}
__device__ __forceinline__ int32_t pack_halo(const MemberDev& m, int xi, int yi, int zi) {
    return f32_pack(xi, yi, zi, m.hbx, m.hby);
}
__device__ __forceinline__ void unpack_halo(const MemberDev& m, int32_t c, int& xi, int& yi, int& zi) {
    f32_unpack(c, m.hbx, m.hby, xi, yi, zi);
}
// halo-inclusive member-local cell of an interior position cell (find_inds!, Individuals/utils.jl:2-7)
__device__ __forceinline__ int q_of(const MemberDev& m, int ci, int cj, int ck) {
    return gid3(m, ci + 1 + m.Hx, cj + 1 + m.Hy, ck + 1 + m.Hz);
}
__device__ __forceinline__ bool interior_q(const MemberDev& m, int q) {
    const int i = q % m.Gx + 1, r = q / m.Gx, j = r % m.Gy + 1, k = r / m.Gy + 1;
    return i > m.Hx && i <= m.Nx + m.Hx && j > m.Hy && j <= m.Ny + m.Hy && k > m.Hz && k <= m.Nz + m.Hz;
}

struct Ax1 { int c; float o; };

// particle_boundary_condition (particle_advection_kernels.jl:2-11) on x = c + o
__device__ __forceinline__ void bc_axis(Ax1& a, int N, int topo) {
    const bool above = a.c > N || (a.c == N && a.o > 0.0f);
    const bool below = a.c < 0;
    if (topo == PI_PERIODIC) {
        if (above) a.c -= N;
        else if (below) a.c += N;
    } else if (above || below) {              // x → 2N − x or x → −x
        const int pivot = above ? 2 * N : 0;
        if (a.o > 0.0f) { a.c = pivot - a.c - 1; a.o = 1.0f - a.o; } else { a.c = pivot - a.c; }
        if (a.o >= 1.0f) { a.c += 1; a.o = 0.0f; }
    }
}
__device__ __forceinline__ void move(Ax1& a, float d, int N, int topo) {
    const float o = a.o + d;
    const float n = floorf(o);
    a.c += (int)n;
    a.o = o - n;
    if (a.o >= 1.0f) { a.c += 1; a.o = 0.0f; }
    bc_axis(a, N, topo);
}
// move() to an RK stage position, which is only sampled: a position left outside [0, N] by a
// displacement above one domain length (CFL far above 1) is noted in `bad` and held at the edge,
// so every corner index of the interpolation stays inside the halo-padded grid (H >= 2)
__device__ __forceinline__ void move_stage(Ax1& a, float d, int N, int topo, bool& bad) {
    move(a, d, N, topo);
    if (a.c < 0 || a.c > N) { bad = true; a.c = a.c < 0 ? 0 : N; a.o = 0.0f; }
}

// index and weight along one axis for a face-centred (own axis) or cell-centred field
// (interpolation.jl:3-83: x + 1 or x + 0.5 split into trunc and mod)
__device__ __forceinline__ void axis_iw(const Ax1& a, int H, bool face, int& idx, float& w) {
    if (face) { idx = a.c + 1 + H; w = a.o; return; }
    const bool lo = a.o < 0.5f;
    idx = a.c + H + (lo ? 0 : 1);
    w = lo ? a.o + 0.5f : a.o - 0.5f;
}
// clamp into [lo, hi], noting an index outside in `bad` (reported once per individual)
__device__ __forceinline__ int clampb(int v, int lo, int hi, bool& bad) {
    const int c = min(max(v, lo), hi);
    bad |= c != v;
    return c;
}

// One velocity component around a position, as the coefficients of its trilinear interpolant in
// grid cells per second: v(xd, yd, zd) = c0 + xd·cx + yd·cy + zd·cz + xd·yd·cxy + xd·zd·cxz +
// yd·zd·cyz + xd·yd·zd·cxyz, formed from the 8 corner values (each divided by its ΔxC, ΔyC or ΔzC,
// interpolation.jl:23-50) when they are loaded. The four RK stages of a step sample points a small
// fraction of a cell apart, usually from the same field (vel₀ = vel½ = vel₁ between velocity
// refreshes), so a stage reuses the coefficients of the previous one when the field and the base
// corner are the same: only the loads and the setup are saved.
struct Corners { int fid; int q; float c0, cx, cy, cz, cxy, cxz, cyz, cxyz; };   // fid: 0 vel₀, 1 vel½, 2 vel₁

// Member constants of the particle kernels, held in registers.
struct PGeom {
    int Nx, Ny, Nz, Hx, Hy, Hz, Gx, Gy, Gz, tx, ty, tz, dz_off;
    float rdx, rdy;
    int fh, f1;     // field ids of vel½ and vel₁ (fields that are the same arrays share an id)
};
__device__ __forceinline__ bool same3(const float* const* a, const float* const* b) {
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}
__device__ __forceinline__ PGeom pgeom(const MemberDev& m, const MemberForcing& f) {
    PGeom g;
    g.fh = same3(f.velh, f.vel0) ? 0 : 1;
    g.f1 = same3(f.vel1, f.velh) ? g.fh : same3(f.vel1, f.vel0) ? 0 : 2;
    g.Nx = m.Nx; g.Ny = m.Ny; g.Nz = m.Nz; g.Hx = m.Hx; g.Hy = m.Hy; g.Hz = m.Hz;
    g.Gx = m.Gx; g.Gy = m.Gy; g.Gz = m.Gz; g.tx = m.tx; g.ty = m.ty; g.tz = m.tz; g.dz_off = m.dz_off;
    g.rdx = m.rdx; g.rdy = m.rdy;
    return g;
}

// trilinear interpolation of one velocity component (member-local field pointer), in grid cells
// per second
// The 8 corner values come from the component's own halo-padded field: in the cell-sorted
// storage order the lanes of a warp sit in neighbouring cells, so the corner loads of a warp
// share sectors and the fields (12 bytes per cell) stay in L2.
// Every position passed here lies in [0, N] on each axis (uploads are validated, stored positions
// are clamped, stage positions pass through move_stage), so with H >= 2 the base corner (i, j, k)
// satisfies 1 <= i <= Gx - 1 (likewise j, k) and needs no clamp.
template <int COMP>
__device__ __forceinline__ float itpl32(const PGeom& m, const float* __restrict__ fld, int fid,
                                        const float* __restrict__ rdzC, const Ax1& X, const Ax1& Y,
                                        const Ax1& Z, Corners& cc) {
    int i, j, k;
    float xd, yd, zd;
    axis_iw(X, m.Hx, COMP == 0, i, xd);
    axis_iw(Y, m.Hy, COMP == 1, j, yd);
    axis_iw(Z, m.Hz, COMP == 2, k, zd);
    const int q = (i - 1) + m.Gx * ((j - 1) + m.Gy * (k - 1));
    if (cc.fid != fid || cc.q != q) {
        const float* __restrict__ p = fld + q;                 // (i, j, k); level k+1 one slab on
        const int sy = m.Gx, sz = m.Gx * m.Gy;
        cc.fid = fid; cc.q = q;
        // corners v_abc at (i + a, j + b, k + c), in cells per second
        float s0 = m.rdx, s1 = m.rdx;
        if (COMP == 1) { s0 = m.rdy; s1 = m.rdy; }
        if (COMP == 2) { s0 = __ldg(rdzC + m.dz_off + k - 1); s1 = __ldg(rdzC + m.dz_off + k); }
        const float v000 = __ldg(p) * s0, v010 = __ldg(p + sy) * s0, v100 = __ldg(p + 1) * s0, v110 = __ldg(p + 1 + sy) * s0;
        const float v001 = __ldg(p + sz) * s1, v011 = __ldg(p + sz + sy) * s1, v101 = __ldg(p + sz + 1) * s1,
                    v111 = __ldg(p + sz + 1 + sy) * s1;
        cc.c0 = v000;
        cc.cx = v100 - v000; cc.cy = v010 - v000; cc.cz = v001 - v000;
        cc.cxy = (v110 - v100) - (v010 - v000);
        cc.cxz = (v101 - v100) - (v001 - v000);
        cc.cyz = (v011 - v010) - (v001 - v000);
        cc.cxyz = ((v111 - v110) - (v101 - v100)) - ((v011 - v010) - (v001 - v000));
    }
    const float ty = fmaf(zd, cc.cxyz, cc.cxy);
    const float tx = fmaf(zd, cc.cxz, fmaf(yd, ty, cc.cx));
    const float tz = fmaf(zd, cc.cyz, cc.cy);
    return fmaf(zd, cc.cz, fmaf(yd, tz, fmaf(xd, tx, cc.c0)));
}

// the draws of the FP64 form (same keys, same numbers; lattice values are exact in float)
__device__ __forceinline__ void draw3f(uint64_t seed, uint32_t iter, uint32_t sp, uint32_t purpose,
                                       uint32_t slot, float& r0, float& r1, float& r2) {
    uint32_t ctr[4] = { slot, iter, (sp & 0xFFFFu) | (purpose << 16), 0x706c6b74u };
    uint32_t key[2] = { (uint32_t)seed, (uint32_t)(seed >> 32) };
    uint32_t o[4];
    pi_philox4x32_10(ctr, key, o);
    r0 = (float)(o[0] >> 8) * 0x1p-24f;
    r1 = (float)(o[1] >> 8) * 0x1p-24f;
    r2 = (float)(o[2] >> 8) * 0x1p-24f;
}

__device__ __forceinline__ unsigned long long to_fixed(float v, double inv_unit) {
    return (unsigned long long)__double2ll_rn((double)v * inv_unit);
}
__device__ __forceinline__ void add_fixed(unsigned long long* a, float v, double inv_unit) {
    const unsigned long long x = to_fixed(v, inv_unit);
    if (x) atomicAdd(a, x);
}

// Warp-segmented sums for the particle → grid scatters. In the cell-sorted storage order the
// individuals of one cell sit in adjacent slots, so the lanes of a warp form runs of equal cell
// keys; each run's first lane adds the run's total with one integer atomic instead of one atomic
// per individual. A warp whose runs are short (more than 16 runs in 32 lanes) adds per lane: the
// shuffles of the segmented sums would cost more than the atomics they save. Sums are integers
// (counts, fixed-point masses), so the result is the same either way. All 32 lanes call these
// with converged control flow; a key of -1 takes no part.
struct WarpRuns {
    bool head;      // this lane adds: the first lane of its run, or every lane when not aggregating
    bool agg;       // the warp adds per run (warp-uniform)
    int end;        // last lane of this lane's run
};
__device__ __forceinline__ WarpRuns warp_runs(long long key) {
    const int lane = threadIdx.x & 31;
    const long long prev = __shfl_up_sync(0xffffffffu, key, 1);
    WarpRuns R;
    const bool head = lane == 0 || prev != key;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const unsigned after = lane == 31 ? 0u : heads & ~((2u << lane) - 1u);
    R.end = after ? __ffs(after) - 2 : 31;
    R.agg = __popc(heads) <= 16;
    R.head = R.agg ? head : true;
    return R;
}
// the total of v over the lanes from this lane to the end of its run (the run's total at its head)
template <typename T>
__device__ __forceinline__ T run_sum(T v, const WarpRuns& R) {
    if (!R.agg) return v;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o <= R.end) v += y;
    }
    return v;
}

// ------------------------------------------------------------------------------------------
// step prologue: forcing of the step, vel½
// ------------------------------------------------------------------------------------------

// update!'s forcing selection (Simulation/update.jl:14-26) for members with device-resident
// series, from model.t before the step (or the step index of the call with time_offset), and the
// choice of the vel½ buffer. Grid: (x blocks, members); block x = 0 binds the fields, every block
// copies its share of the surface PAR snapshot.
__device__ __forceinline__ long long snap_index(double tm, double tc, int use_call, double dT_s, long long n,
                                                uint32_t* err, bool flag) {
    long long t = (long long)floor((use_call ? tc : tm) / dT_s);
    if (t < 0 || t >= n) { if (flag) seterr(err, F32_ERR_FORCING); t = t < 0 ? 0 : n - 1; }
    return t;
}

__global__ void k32_bind(int nm, const MemberDev* __restrict__ md, const MemberSeries* __restrict__ S,
                         MemberForcing* __restrict__ F, const StepState* __restrict__ st, double dT,
                         float* __restrict__ PARF, uint32_t* err) {
    const int m = blockIdx.y;
    if (m >= nm || stopped(err)) return;
    const MemberSeries& s = S[m];
    const MemberDev& M = md[m];
    const double tm = st->t, tc = (double)st->call_step * dT;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    if (lead) {
        MemberForcing f = F[m];
        if (s.has_series) {
            if (s.has_vel) {
                const long long tv = snap_index(tm, tc, s.time_offset & 1, s.dT_vel, s.nvel, err, true);
                for (int c = 0; c < 3; ++c) f.vel1[c] = s.vel + (tv * 3 + c) * M.G;
            }
            f.temp = s.temp + snap_index(tm, tc, s.time_offset & 4, s.dT_temp, s.ntemp, err, true) * M.G;
        }
        for (int c = 0; c < 3; ++c) f.velh[c] = (f.vel0[c] == f.vel1[c]) ? f.vel1[c] : s.velh_buf[c];
        F[m] = f;
    }
    if (!s.has_series) return;
    const long long tp = snap_index(tm, tc, s.time_offset & 2, s.dT_PAR, s.npar, err, lead);
    const long long n = (long long)M.Nx * M.Ny;
    const float* src = s.parf + tp * n;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        PARF[M.col_off + q] = src[q];
}

// vel½ = (vel₀ + vel₁) * 0.5 (time_step.jl:17-19) for members whose two fields differ.
// Grid: (x blocks, members).
__global__ void k32_velhalf(const MemberDev* __restrict__ md, const MemberForcing* __restrict__ F,
                            const uint32_t* err) {
    const int m = blockIdx.y;
    if (stopped(err)) return;
    const MemberForcing& f = F[m];
    if (f.velh[0] == f.vel1[0]) return;
    const long long G = md[m].G;
    float* h0 = (float*)f.velh[0];
    float* h1 = (float*)f.velh[1];
    float* h2 = (float*)f.velh[2];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < G; q += (long long)gridDim.x * blockDim.x) {
        h0[q] = (f.vel0[0][q] + f.vel1[0][q]) * 0.5f;
        h1[q] = (f.vel0[1][q] + f.vel1[1][q]) * 0.5f;
        h2[q] = (f.vel0[2][q] + f.vel1[2][q]) * 0.5f;
    }
}

// ------------------------------------------------------------------------------------------
// (a)+(e) particles: RK4 + diffusion + find_inds!, pop and Chl into the per-cell sums, then the
// grazing/mortality decisions of the previous step (inactivate!, calc_loss!, diagnostics) and the
// division/free counts of each tile of slots for the compaction.
// ------------------------------------------------------------------------------------------
struct MoveArgs {
    Tab32 T;
    IndDev32 P;
    const SpeciesDev32* sp;        // [member * nsp + species]
    const BgcDev32* bgc;           // [member]
    const MemberForcing* F;
    const float* rdzC;             // 1 / ΔzC
    const StepState* st;
    float dT;
    long long Gtot;
    int* pop;                      // Gtot: all species
    int* pop_sp;                   // nsp × Gtot when grazing is not shared, else null
    unsigned long long* chl_acc;   // Gtot
    unsigned long long* acc;       // ACC_N × Gtot
    uint32_t* dcnt;                // nsp × 4 × Gtot: num, graz, mort, dvid
    uint32_t* err;
};

// bit of logical slot L of species s of member m in a logical-slot bitmap
__device__ __forceinline__ void slot_bit(const MemberDev& m, int s, int L, long long& w, uint32_t& bit) {
    w = m.woff + (long long)s * m.wps + (L >> 5);
    bit = 1u << (L & 31);
}

// The slot state k32_move reads first, loaded one slot ahead of its use (the offsets and Chl of an
// inactive slot are read and unused).
struct MState { int32_t code; float ox, oy, oz, chl; uint8_t fl, stt; };
__device__ __forceinline__ MState move_state(const IndDev32& P, long long g, bool valid) {
    MState S{-1, 0.0f, 0.0f, 0.0f, 0.0f, 0, 0};
    if (valid) {
        S.fl = P.flags[g]; S.stt = P.stat[g]; S.code = P.cell[g];
        S.ox = P.ox[g]; S.oy = P.oy[g]; S.oz = P.oz[g]; S.chl = P.Chl[g];
    }
    return S;
}

// What k32_move adds to the grid for one slot: the cell (-1: nothing), a packed count
// (pop | grazed << 8 | dead << 16 | dividing << 24; a warp's run sums stay below 256 per field) and
// the Chl sum in fixed point (interior cells only).
struct MoveOut { long long cq; uint32_t cnt; unsigned long long chl; };

__device__ __forceinline__ MoveOut move_one(const MoveArgs& a, const MemberDev& m, const PGeom& pg, int mi, int s,
                                            long long g, uint32_t iter, const MState& S) {
    const IndDev32& P = a.P;
    MoveOut out{-1, 0u, 0ull};
    const uint8_t fl = S.fl, stt = S.stt;
    const int32_t code = S.code;
    const float ox = S.ox, oy = S.oy, oz = S.oz;
    const float chl = S.chl;
    if (!(fl & F32_AC)) {
        // every stage multiplies by ac: the position becomes (0, 0, 0) and the cell (Hx, Hy, Hz)
        if (code != -1) {
            P.cell[g] = -1;
            P.ox[g] = 0.0f; P.oy[g] = 0.0f; P.oz[g] = 0.0f;
        }
        if (stt) P.stat[g] = 0;
        return out;
    }
    uint32_t* err = a.err;
    int ci, cj, ck;
    unpack_int(m, code, ci, cj, ck);
    // ΔzC at the find_inds! zi of the previous step, plus Hz (particle_diffusion.jl:26-28)
    int zi = ck + 1 + pg.Hz;
    if (stt & F32_ST_STALE) { int a0, a1; unpack_halo(m, P.scell[g], a0, a1, zi); }
    bool bad = false;
    const int kdz = clampb(zi + pg.Hz, 1, pg.Gz, bad);
    const MemberForcing& f = a.F[mi];
    const Ax1 X0{ci, ox}, Y0{cj, oy}, Z0{ck, oz};
    const float dT = a.dT, hdT = 0.5f * dT;
    const float* __restrict__ rdzC = a.rdzC;
    Corners cu{-1, -1}, cv{-1, -1}, cw{-1, -1};
    const int fh = pg.fh, f1 = pg.f1;
    float u1 = itpl32<0>(pg, f.vel0[0], 0, rdzC, X0, Y0, Z0, cu);
    float v1 = itpl32<1>(pg, f.vel0[1], 0, rdzC, X0, Y0, Z0, cv);
    float w1 = itpl32<2>(pg, f.vel0[2], 0, rdzC, X0, Y0, Z0, cw);
    float u2 = u1, v2 = v1, w2 = w1;
    Ax1 X = X0, Y = Y0, Z = Z0;
    move_stage(X, u1 * hdT, pg.Nx, pg.tx, bad); move_stage(Y, v1 * hdT, pg.Ny, pg.ty, bad); move_stage(Z, -(w1 * hdT), pg.Nz, pg.tz, bad);
    u1 = itpl32<0>(pg, f.velh[0], fh, rdzC, X, Y, Z, cu); v1 = itpl32<1>(pg, f.velh[1], fh, rdzC, X, Y, Z, cv);
    w1 = itpl32<2>(pg, f.velh[2], fh, rdzC, X, Y, Z, cw);
    u2 += u1 * 2.0f; v2 += v1 * 2.0f; w2 += w1 * 2.0f;
    X = X0; Y = Y0; Z = Z0;
    move_stage(X, u1 * hdT, pg.Nx, pg.tx, bad); move_stage(Y, v1 * hdT, pg.Ny, pg.ty, bad); move_stage(Z, -(w1 * hdT), pg.Nz, pg.tz, bad);
    u1 = itpl32<0>(pg, f.velh[0], fh, rdzC, X, Y, Z, cu); v1 = itpl32<1>(pg, f.velh[1], fh, rdzC, X, Y, Z, cv);
    w1 = itpl32<2>(pg, f.velh[2], fh, rdzC, X, Y, Z, cw);
    u2 += u1 * 2.0f; v2 += v1 * 2.0f; w2 += w1 * 2.0f;
    X = X0; Y = Y0; Z = Z0;
    move_stage(X, u1 * dT, pg.Nx, pg.tx, bad); move_stage(Y, v1 * dT, pg.Ny, pg.ty, bad); move_stage(Z, -(w1 * dT), pg.Nz, pg.tz, bad);
    u1 = itpl32<0>(pg, f.vel1[0], f1, rdzC, X, Y, Z, cu); v1 = itpl32<1>(pg, f.vel1[1], f1, rdzC, X, Y, Z, cv);
    w1 = itpl32<2>(pg, f.vel1[2], f1, rdzC, X, Y, Z, cw);
    const float sixth = 1.0f / 6.0f;
    u2 = (u2 + u1) * sixth; v2 = (v2 + v1) * sixth; w2 = (w2 + w1) * sixth;
    X = X0; Y = Y0; Z = Z0;
    move(X, u2 * dT, pg.Nx, pg.tx); move(Y, v2 * dT, pg.Ny, pg.ty); move(Z, -(w2 * dT), pg.Nz, pg.tz);
    // random-walk diffusion (particle_diffusion.jl:16-33); a zero κ moves nothing
    const BgcDev32& b = a.bgc[mi];
    if (b.kappa_hP != 0.0f || b.kappa_vP != 0.0f) {
        float r0, r1, r2;
        draw3f(m.seed, iter, (uint32_t)s, PI_DRAW_DIFFUSION, (uint32_t)P.lslot[g], r0, r1, r2);
        move(X, (r0 - 0.5f) * 2.0f * sqrtf(b.kappa_hP * dT) * pg.rdx, pg.Nx, pg.tx);
        move(Y, (r1 - 0.5f) * 2.0f * sqrtf(b.kappa_hP * dT) * pg.rdy, pg.Ny, pg.ty);
        move(Z, (r2 - 0.5f) * 2.0f * sqrtf(b.kappa_vP * dT) * __ldg(rdzC + pg.dz_off + kdz - 1), pg.Nz, pg.tz);
    }
    if (X.c < 0 || X.c > pg.Nx) { bad = true; X.c = X.c < 0 ? 0 : pg.Nx; X.o = 0.0f; }
    if (Y.c < 0 || Y.c > pg.Ny) { bad = true; Y.c = Y.c < 0 ? 0 : pg.Ny; Y.o = 0.0f; }
    if (Z.c < 0 || Z.c > pg.Nz) { bad = true; Z.c = Z.c < 0 ? 0 : pg.Nz; Z.o = 0.0f; }
    if (bad) seterr(err, F32_ERR_DOMAIN);
    // everything that reads the member record is formed before the stores below
    const int32_t code_new = pack_int(m, X.c, Y.c, Z.c);
    const long long cq = m.cell_off + q_of(m, X.c, Y.c, Z.c);
    const bool inside = X.c < pg.Nx && Y.c < pg.Ny && Z.c < pg.Nz;
    const double chl_inv = m.chl_inv, fx_inv = m.fx_inv;
    P.ox[g] = X.o; P.oy[g] = Y.o; P.oz[g] = Z.o;
    P.cell[g] = code_new;
    const long long G = a.Gtot;
    // previous step's decisions (plankton_update.jl:5-16, division_death.jl:2-25)
    const int gz = (fl & F32_GRAZ) != 0, mt = (fl & F32_MORT) != 0, dv = (fl & F32_DVID) != 0;
    const int ac1 = !gz, ac2 = ac1 && !mt, dv2 = dv && ac2;
    // pop, the Chl sum and the graz/mort/dvid diagnostics counts, added by scatter_move
    out.cq = cq;
    out.cnt = 1u | (gz ? 1u << 8 : 0u) | (ac1 && mt ? 1u << 16 : 0u) | (dv2 ? 1u << 24 : 0u);
    out.chl = inside ? to_fixed(chl, chl_inv) : 0ull;
    const int kind = gz ? 1 : (ac1 && mt) ? 2 : 0;
    if (kind && inside) {
        const SpeciesDev32& p = a.sp[mi * a.T.nsp + s];
        const float fC = kind == 1 ? p.grazFracC : p.mortFracC;
        const float fN = kind == 1 ? p.grazFracN : p.mortFracN;
        const float fP = kind == 1 ? p.grazFracP : p.mortFracP;
        const float Bm = P.Bm[g], Cq = P.Cq[g], Nq = P.Nq[g], Pq = P.Pq[g];
        const double u = fx_inv;
        add_fixed(&a.acc[ACC_DOC * G + cq], (Bm + Cq) * fC, u);
        add_fixed(&a.acc[ACC_DON * G + cq], (Bm * p.R_NC + Nq) * fN, u);
        add_fixed(&a.acc[ACC_DOP * G + cq], (Bm * p.R_PC + Pq) * fP, u);
        add_fixed(&a.acc[ACC_POC * G + cq], (Bm + Cq) * (1.0f - fC), u);
        add_fixed(&a.acc[ACC_PON * G + cq], (Bm * p.R_NC + Nq) * (1.0f - fN), u);
        add_fixed(&a.acc[ACC_POP * G + cq], (Bm * p.R_PC + Pq) * (1.0f - fP), u);
    }
    P.flags[g] = (uint8_t)((ac2 ? F32_AC : 0) | (dv2 ? F32_DVID : 0));
    P.stat[g] = F32_ST_AC0;
    // division bookkeeping on logical slots: dividers of this step, slots freed by this step's
    // grazing and mortality (free slots stay marked until a daughter takes them)
    if (dv2 || !ac2) {
        long long w;
        uint32_t bit;
        slot_bit(m, s, P.lslot[g], w, bit);
        atomicOr(dv2 ? &P.dvbits[w] : &P.freebits[w], bit);
    }
    return out;
}

// k32_move's grid sums of one warp (segment s of one member): one atomic per run of a cell
__device__ __forceinline__ void scatter_move(const MoveArgs& a, int s, const MoveOut& o) {
    if (__all_sync(0xffffffffu, o.cq < 0)) return;      // a warp of inactive slots adds nothing
    const WarpRuns R = warp_runs(o.cq);
    const uint32_t c = run_sum(o.cnt, R);
    const unsigned long long chl = run_sum(o.chl, R);
    if (R.head && o.cq >= 0) {
        const long long G = a.Gtot, cq = o.cq;
        const int np = (int)(c & 0xffu);
        atomicAdd(&a.pop[cq], np);
        if (a.pop_sp) atomicAdd(&a.pop_sp[(long long)s * G + cq], np);
        if (chl) atomicAdd(&a.chl_acc[cq], chl);
        uint32_t* dc = a.dcnt + (long long)s * 4 * G + cq;
        if (c >> 8 & 0xffu) atomicAdd(dc + 1 * G, c >> 8 & 0xffu);
        if (c >> 16 & 0xffu) atomicAdd(dc + 2 * G, c >> 16 & 0xffu);
        if (c >> 24) atomicAdd(dc + 3 * G, c >> 24);
    }
}

// MINB: blocks of 256 threads per SM the registers are fitted for (2: 128 registers, 3: 80, 4: 64);
// the autotuner picks the variant.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k32_move(MoveArgs a) {
    if (stopped(a.err)) return;
    __shared__ PGeom sg;
    const int bs = blockDim.x, ppt = F32_TILE / bs;
    const uint32_t iter = (uint32_t)(a.st->iteration + 1);
    for (int t = blockIdx.x; t < a.T.ntiles; t += gridDim.x) {
        const int2 tl = a.T.tiles[t];
        int mi, s;
        seg_of(a.T, tl.x, mi, s);
        const MemberDev& m = a.T.md[mi];
        if (threadIdx.x == 0) sg = pgeom(m, a.F[mi]);
        __syncthreads();
        const long long base = m.slot_off + (long long)s * m.C;
        long long slot = (long long)tl.y + threadIdx.x;
        MState nx = move_state(a.P, base + slot, slot < m.C);
        for (int p = 0; p < ppt; ++p, slot += bs) {
            const MState cur = nx;
            if (p + 1 < ppt) nx = move_state(a.P, base + slot + bs, slot + bs < m.C);
            MoveOut o{-1, 0u, 0ull};
            if (slot < m.C) o = move_one(a, m, sg, mi, s, base + slot, iter, cur);
            scatter_move(a, s, o);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------
// PAR down each column (calc_par!, Individuals/utils.jl:55-63); consumes the Chl sums
// ------------------------------------------------------------------------------------------
//
// For every interior cell holding individuals it also packs the environment physiology gathers
// (find_NPT!, utils.jl:14-25: NH4, NO3, PO4, DOC, par, temperature, pop) into one 32-byte record,
// so an individual reads one sector instead of seven.
#define PAR_CH 8      // levels whose loads are issued together (the column walk is a latency chain)
__global__ void k32_par(Tab32 T, const float* __restrict__ dzF, const BgcDev32* __restrict__ bgc,
                        unsigned long long* __restrict__ chl_acc, float* __restrict__ PARF,
                        float* __restrict__ par, float* __restrict__ diag_par, const float* __restrict__ tr,
                        long long Gtot, const MemberForcing* __restrict__ F, const int* __restrict__ pop,
                        float4* __restrict__ env, const uint32_t* err) {
    if (stopped(err)) return;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < T.nicol; w += nw) {
        const int4 it = T.icol[w];
        const MemberDev& m = T.md[it.x];
        const int i = it.y + lane, j = it.z;     // 1-based interior column
        if (i > m.Nx) continue;
        const float kc = bgc[it.x].kc, kw = bgc[it.x].kw;
        const long long fcol = m.col_off + (i - 1) + (long long)m.Nx * (j - 1);
        float parf = PARF[fcol];
        const long long c1 = m.cell_off + gid3(m, i + m.Hx, j + m.Hy, 1 + m.Hz);
        const long long slab = (long long)m.Gx * m.Gy;
        const float* __restrict__ temp = F[it.x].temp;
        const float areaf = m.dx * m.dy;
        for (int k0 = 1; k0 <= m.Nz; k0 += PAR_CH) {
            // the loads of PAR_CH levels first (only PARF carries down the column)
            long long v[PAR_CH];
            int pp[PAR_CH];
            float dp[PAR_CH], dz[PAR_CH];
#pragma unroll
            for (int e = 0; e < PAR_CH; ++e) {
                const int k = k0 + e;
                const long long c = c1 + (k - 1) * slab;
                const bool in = k <= m.Nz;
                v[e] = in ? (long long)chl_acc[c] : 0;
                pp[e] = in ? pop[c] : 0;
                dp[e] = in ? diag_par[c] : 0.0f;
                dz[e] = in ? dzF[m.dz_off + k + m.Hz - 1] : 1.0f;
            }
            float pvs[PAR_CH];
#pragma unroll
            for (int e = 0; e < PAR_CH; ++e) {
                const int k = k0 + e;
                if (k > m.Nz) { pvs[e] = 0.0f; continue; }
                const long long c = c1 + (k - 1) * slab;
                if (v[e]) chl_acc[c] = 0ull;
                const float chl = (float)((double)v[e] * m.chl_unit);
                const float volk = areaf * dz[e];
                const float atten = (chl / volk * kc + kw) * dz[e];
                const float ex = expf(-atten);
                const float pv = parf * (1.0f - ex) / atten;
                par[c] = pv;
                parf = parf * ex;
                diag_par[c] = dp[e] + pv;
                pvs[e] = pv;
            }
            // environment records of the occupied cells of these levels
#pragma unroll
            for (int e = 0; e < PAR_CH; ++e) {
                const int k = k0 + e;
                if (k > m.Nz || pp[e] <= 0) continue;
                const long long c = c1 + (k - 1) * slab;
                env[2 * c] = make_float4(tr[PI_NH4 * Gtot + c], tr[PI_NO3 * Gtot + c], tr[PI_PO4 * Gtot + c],
                                         tr[PI_DOC * Gtot + c]);
                env[2 * c + 1] = make_float4(pvs[e], temp[c - m.cell_off], (float)pp[e], 0.0f);
            }
        }
        PARF[fcol] = parf;
    }
}

// ------------------------------------------------------------------------------------------
// (e) division: k-th divider (logical slot order) → k-th free logical slot (findall(!ac),
// ascending), per segment (get_tind!, Individuals/utils.jl:76-86), with the capacity check
// (plankton_update.jl:18-22). Dividers and free slots are bits of two bitmaps over logical slots;
// a tile of F32_TILE logical slots is 32 words, one per lane of a warp.
// ------------------------------------------------------------------------------------------

// (dividers << 32) | free slots of every tile, from the bitmaps. One warp per tile.
__global__ void k32_count_tiles(Tab32 T, IndDev32 P, unsigned long long* __restrict__ tile_cnt, const uint32_t* err) {
    if (stopped(err)) return;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T.ntiles; t += nw) {
        const int2 tl = T.tiles[t];
        int mi, s;
        seg_of(T, tl.x, mi, s);
        const MemberDev& m = T.md[mi];
        const long long w = m.woff + (long long)s * m.wps + (tl.y >> 5) + lane;
        const unsigned nd = __reduce_add_sync(0xffffffffu, (unsigned)__popc(P.dvbits[w]));
        const unsigned nf = __reduce_add_sync(0xffffffffu, (unsigned)__popc(P.freebits[w]));
        if (lane == 0) tile_cnt[t] = ((unsigned long long)nd << 32) | nf;
    }
}

// ---- exclusive prefix sums of 64-bit counts (block-wide, 1024 threads) ----------------------
// inclusive scan over the lanes of a warp
__device__ __forceinline__ unsigned long long warp_inscan64(unsigned long long x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}
// Exclusive scan of v over the block (blockDim.x == 1024); returns the thread's prefix and the
// block total in *total. sh holds 33 values.
__device__ __forceinline__ unsigned long long block_exscan64(unsigned long long v, unsigned long long* sh,
                                                             unsigned long long* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned long long inc = warp_inscan64(v);
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        const unsigned long long w = sh[lane];
        const unsigned long long wi = warp_inscan64(w);
        sh[lane] = wi - w;
        if (lane == 31) sh[32] = wi;
    }
    __syncthreads();
    const unsigned long long out = sh[wid] + inc - v;
    *total = sh[32];
    __syncthreads();
    return out;
}

// Exclusive scan of the tile counts within each (member, species) segment: one block of 1024
// threads per segment.
__global__ void __launch_bounds__(1024) k32_scan_tiles(Tab32 T, const unsigned long long* __restrict__ tile_cnt,
                                                       unsigned long long* __restrict__ tile_off, int nseg,
                                                       const uint32_t* err) {
    if (stopped(err)) return;
    __shared__ unsigned long long sh[33];
    for (int seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
        const int t0 = T.seg_tile0[seg], t1 = T.seg_tile0[seg + 1];
        unsigned long long run = 0;
        for (int base = t0; base < t1; base += 1024) {
            const int t = base + threadIdx.x;
            const unsigned long long v = t < t1 ? tile_cnt[t] : 0ull;
            unsigned long long tot;
            const unsigned long long ex = block_exscan64(v, sh, &tot);
            if (t < t1) tile_off[t] = run + ex;
            run += tot;
        }
    }
}

// Exclusive scan of n 64-bit values in three passes (chunks of 1024 × PER values): chunk sums,
// a scan of the chunk sums in one block, then each chunk's scan from its offset.
#define SCAN_PER 8
__global__ void __launch_bounds__(1024) k32_scan_sums(const unsigned long long* __restrict__ in, long long n,
                                                      unsigned long long* __restrict__ sums) {
    __shared__ unsigned long long sh[33];
    const long long base = (long long)blockIdx.x * 1024 * SCAN_PER;
    unsigned long long v = 0;
    for (int e = 0; e < SCAN_PER; ++e) {
        const long long q = base + (long long)e * 1024 + threadIdx.x;
        if (q < n) v += in[q];
    }
    unsigned long long tot;
    block_exscan64(v, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}
__global__ void __launch_bounds__(1024) k32_scan_chunks(unsigned long long* __restrict__ sums, long long nchunks) {
    __shared__ unsigned long long sh[33];
    unsigned long long run = 0;
    for (long long b = 0; b < nchunks; b += 1024) {
        const long long q = b + threadIdx.x;
        const unsigned long long v = q < nchunks ? sums[q] : 0ull;
        unsigned long long tot;
        const unsigned long long ex = block_exscan64(v, sh, &tot);
        if (q < nchunks) sums[q] = run + ex;
        run += tot;
    }
}
__global__ void __launch_bounds__(1024) k32_scan_apply(const unsigned long long* __restrict__ in, long long n,
                                                       const unsigned long long* __restrict__ sums,
                                                       unsigned long long* __restrict__ out) {
    __shared__ unsigned long long sh[33];
    const long long base = (long long)blockIdx.x * 1024 * SCAN_PER;
    // each thread takes PER consecutive values so that the chunk is scanned in order
    const long long q0 = base + (long long)threadIdx.x * SCAN_PER;
    unsigned long long loc[SCAN_PER], v = 0;
#pragma unroll
    for (int e = 0; e < SCAN_PER; ++e) { loc[e] = q0 + e < n ? in[q0 + e] : 0ull; v += loc[e]; }
    unsigned long long tot;
    unsigned long long run = sums[blockIdx.x] + block_exscan64(v, sh, &tot);
#pragma unroll
    for (int e = 0; e < SCAN_PER; ++e) {
        if (q0 + e < n) out[q0 + e] = run;
        run += loc[e];
    }
}

// exclusive prefix sum over the lanes of a warp
__device__ __forceinline__ unsigned warp_exscan(unsigned v) {
    const int lane = threadIdx.x & 31;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x - v;
}

// Lists of the dividers and of the free slots they take, in logical order. One warp per tile;
// tiles with neither dividers nor needed free slots do nothing. The divider bits are cleared once
// listed.
__global__ void k32_assign(Tab32 T, IndDev32 P, const unsigned long long* __restrict__ tile_cnt,
                           const unsigned long long* __restrict__ tile_off, int* __restrict__ divlist,
                           int* __restrict__ freelist, uint32_t* __restrict__ ndiv, StepState* st,
                           uint32_t* err) {
    if (stopped(err)) return;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T.ntiles; t += nw) {
        const int2 tl = T.tiles[t];
        const int seg = tl.x;
        int mi, s;
        seg_of(T, seg, mi, s);
        const MemberDev& m = T.md[mi];
        const long long base = m.slot_off + (long long)s * m.C;
        const int t0 = T.seg_tile0[seg], t1 = T.seg_tile0[seg + 1];
        const unsigned long long b0 = tile_off[t0];
        const unsigned long long tot = tile_off[t1 - 1] + tile_cnt[t1 - 1] - b0;
        const unsigned int tdiv = (unsigned int)(tot >> 32), tfree = (unsigned int)(tot & 0xffffffffull);
        if (tdiv > tfree) {
            if (t == t0 && lane == 0) {
                ndiv[seg] = 0;
                if (!(atomicOr(err, F32_ERR_CAPACITY) & F32_ERR_CAPACITY)) {
                    st->err_iter = st->iteration + 1;
                    st->err_member = mi;
                }
            }
            continue;
        }
        if (t == t0 && lane == 0) ndiv[seg] = tdiv;
        const unsigned long long before = tile_off[t] - b0;
        const unsigned int dbefore = (unsigned int)(before >> 32), fbefore = (unsigned int)(before & 0xffffffffull);
        const unsigned long long c = tile_cnt[t];
        const bool wd = (c >> 32) != 0, wf = (c & 0xffffffffull) != 0 && fbefore < tdiv;
        if (!wd && !wf) continue;                                   // uniform over the warp
        const long long w = m.woff + (long long)s * m.wps + (tl.y >> 5) + lane;
        uint32_t dw = wd ? P.dvbits[w] : 0u, fw = wf ? P.freebits[w] : 0u;
        unsigned rd = dbefore + warp_exscan((unsigned)__popc(dw));
        unsigned rf = fbefore + warp_exscan((unsigned)__popc(fw));
        const int L0 = tl.y + lane * 32;
        while (dw) {
            const int bpos = __ffs(dw) - 1;
            dw &= dw - 1u;
            divlist[base + rd++] = L0 + bpos;
        }
        while (fw && rf < tdiv) {
            const int bpos = __ffs(fw) - 1;
            fw &= fw - 1u;
            freelist[base + rf++] = L0 + bpos;
        }
        if (wd) P.dvbits[w] = 0u;
    }
}

// copy_daughter_individuals! and divide_to_half! (division_death.jl:28-63). The lists hold logical
// slots; phys gives where each is stored. Grid: (x, segments).
__global__ void k32_daughters(Tab32 T, IndDev32 P, const int* __restrict__ divlist,
                              const int* __restrict__ freelist, const uint32_t* __restrict__ ndiv,
                              uint32_t* err) {
    if (stopped(err)) return;
    const int seg = blockIdx.y;
    int mi, s;
    seg_of(T, seg, mi, s);
    const MemberDev& m = T.md[mi];
    const long long base = m.slot_off + (long long)s * m.C;
    const uint32_t n = ndiv[seg];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int pl = divlist[base + k], dl = freelist[base + k];
        if (k >= (uint32_t)m.C || pl < 0 || pl >= m.C || dl < 0 || dl >= m.C) { seterr(err, F32_ERR_LISTS); continue; }
        const int pp = P.phys[base + pl], dp = P.phys[base + dl];
        if (pp < 0 || pp >= m.C || dp < 0 || dp >= m.C) { seterr(err, F32_ERR_LISTS); continue; }
        const long long p = base + pp, d = base + dp;
        // the daughter's slot keeps the cell find_inds! gave it this step
        const int32_t cd = P.cell[d];
        int32_t sc;
        if (cd < 0) sc = pack_halo(m, m.Hx, m.Hy, m.Hz);
        else { int a0, a1, a2; unpack_int(m, cd, a0, a1, a2); sc = pack_halo(m, a0 + 1 + m.Hx, a1 + 1 + m.Hy, a2 + 1 + m.Hz); }
        P.scell[d] = sc;
        P.cell[d] = P.cell[p];
        P.ox[d] = P.ox[p]; P.oy[d] = P.oy[p]; P.oz[d] = P.oz[p];
        const float Bm = P.Bm[p] * 0.5f, Cq = P.Cq[p] * 0.5f, Nq = P.Nq[p] * 0.5f, Pq = P.Pq[p] * 0.5f;
        const float Chl = P.Chl[p] * 0.5f, gen = P.gen[p] + 1.0f;
        P.Bm[d] = Bm; P.Cq[d] = Cq; P.Nq[d] = Nq; P.Pq[d] = Pq; P.Chl[d] = Chl; P.gen[d] = gen;
        P.age[d] = P.age[d] * 0.0f;
        P.Bm[p] = Bm; P.Cq[p] = Cq; P.Nq[p] = Nq; P.Pq[p] = Pq; P.Chl[p] = Chl; P.gen[p] = gen;
        P.age[p] = P.age[p] * 0.0f;
        P.flags[d] = F32_AC | F32_DVID;
        P.stat[d] = (uint8_t)((P.stat[d] & F32_ST_AC0) | F32_ST_STALE);
        long long w;
        uint32_t bit;
        slot_bit(m, s, dl, w, bit);
        atomicAnd(&P.freebits[w], ~bit);
    }
}

// ------------------------------------------------------------------------------------------
// (b) QuotaMode physiology in Float32 (plankton_growth.jl:2-24, growth_kernels.jl:2-166,
//     division_death_probability.jl:7-107, find_NPT!, calc_consume!, diags num)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float shape_dec_f(float x, float xmax, float k, int pw) {
    const float fx = fmaxf(0.0f, fminf(1.0f, 1.0f - x / xmax));
    const float p = pw == 2 ? fx * fx : (fx * fx) * (fx * fx);
    return p / (k + p);
}
__device__ __forceinline__ float shape_inc_f(float x, float xmax, float k, int pw) {
    return 1.0f - shape_dec_f(x, xmax, k, pw);
}
__device__ __forceinline__ float tempFunc_f(float T, const SpeciesDev32& p) {
    const float k = fmaxf(0.0f, expf(-p.Ea / (8.3145f * (T + 273.15f))));
    return fminf(1.0f, k / p.OGT_rate);
}
__device__ __forceinline__ float tempFunc_PS_f(float T, const SpeciesDev32& p) {
    const float regT = shape_dec_f(T - p.Topt, p.Tmax - p.Topt, 4.0e-2f, 4);
    const float k = fmaxf(0.0f, expf(-p.Ea / (8.3145f * (T + 273.15f))) * regT);
    return fminf(1.0f, k / p.OGT_rate);
}
// Julia isless on floats without signed zeros: NaN orders last
__device__ __forceinline__ bool jl_lessf(float x, float y) { return x < y || (y != y && x == x); }

struct PhysArgs {
    Tab32 T;
    IndDev32 P;
    const SpeciesDev32* sp;
    const MemberForcing* F;
    const StepState* st;
    float dT;
    long long Gtot;
    const float* tr;
    const float* par;
    const int* pop;
    const int* pop_sp;
    const float4* env;          // packed environment of occupied interior cells
    unsigned long long* acc;
    uint32_t* dcnt;
    const uint32_t* err;
    const SpeciesDec64* dec64;  // [member * nsp + species]
    unsigned long long* guard;  // [0] decisions recomputed in Float64, [1] of those, decisions changed
    unsigned long long* dproc;  // optional process diagnostics, fixed point: (species * PI_NPROC + q) * Gtot
    uint32_t pmask;             // enabled processes (PI_PROC_* bits)
};

// Fixed-point units of the process diagnostics: rates (mmol s⁻¹) in the mass unit per minute,
// Bm, Cq, Nq and Pq in the mass unit, Chl in the Chl unit (so a sum over any set of individuals is
// exact in 64 bits and independent of the order).
__host__ __device__ inline double proc_unit(const MemberDev& m, int q) {
    return q < PI_PROC_Bm ? m.fx_unit / 60.0 : q < PI_PROC_Chl ? m.fx_unit : m.chl_unit;
}

// Guard band of the decisions (get_probability!, division_death_probability.jl:95-107): a draw
// within this relative distance of p·ΔT in Float32 takes the decision from p recomputed in Float64
// from the individual's Float32 state, which removes the rounding of the probability formulas
// (a few Float32 ulps) from the comparison.
#define F32_GUARD_REL 1.0e-5f

__device__ __forceinline__ double shape_dec_d(double x, double xmax, double k, int pw) {
    const double fx = fmax(0.0, fmin(1.0, 1.0 - x / xmax));
    const double p = pw == 2 ? fx * fx : (fx * fx) * (fx * fx);
    return p / (k + p);
}
__device__ __forceinline__ bool near_threshold(float r, float t) {
    return fabsf(r - t) <= F32_GUARD_REL * fabsf(t);
}

// flags, status, cell and logical slot of a slot, loaded one slot ahead of its physiology, and,
// for an active slot, its quotas and age and, when it was binned this step into an interior cell
// (not a stale cell), the environment record of that cell: phys_one then waits on no load.
struct PHead {
    int32_t code, ls;
    uint8_t fl, stt;
    int env;                    // e0, e1 hold the environment record
    float Bm, Cq, Nq, Pq, Chl, age;
    float4 e0, e1;
};
// The first level of a slot's loads (flags, status, cell, logical slot): the loads of phys_head
// depend on them, so k32_physiology issues these two slots ahead and phys_head one slot ahead.
struct PPre { int32_t code, ls; uint8_t fl, stt; };
__device__ __forceinline__ PPre phys_pre(const IndDev32& P, long long g, bool valid) {
    PPre r{-1, 0, 0, 0};
    if (valid) { r.fl = P.flags[g]; r.stt = P.stat[g]; r.code = P.cell[g]; r.ls = P.lslot[g]; }
    return r;
}
__device__ __forceinline__ PHead phys_head(const IndDev32& P, long long g, const PPre& pre, const MemberDev& m,
                                           const float4* __restrict__ envr) {
    PHead h{-1, 0, 0, 0, 0, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, {}, {}};
    {
        h.fl = pre.fl; h.stt = pre.stt; h.code = pre.code; h.ls = pre.ls;
        if (h.fl & F32_AC) {
            h.Bm = P.Bm[g]; h.Cq = P.Cq[g]; h.Nq = P.Nq[g]; h.Pq = P.Pq[g]; h.Chl = P.Chl[g]; h.age = P.age[g];
            if ((h.stt & F32_ST_AC0) && !(h.stt & F32_ST_STALE)) {
                int ci, cj, ck;
                unpack_int(m, h.code, ci, cj, ck);
                if (ci < m.Nx && cj < m.Ny && ck < m.Nz) {
                    const long long cq = m.cell_off + q_of(m, ci, cj, ck);
                    h.e0 = envr[2 * cq]; h.e1 = envr[2 * cq + 1];
                    h.env = 1;
                }
            }
        }
    }
    return h;
}

// What k32_physiology adds to the grid for one slot: the cell (-1: nothing; the diagnostics count
// num is added there) and the consumption of DIC, DOC, NH4, NO3, PO4 in fixed point (zero unless
// the individual was binned this step into an interior cell).
struct PhysOut { long long cq; unsigned long long v[5]; };

__device__ __forceinline__ PhysOut phys_one(const PhysArgs& a, const MemberDev& m, int mi, int s,
                                            long long g, uint32_t iter, double tnow, const PHead& hd) {
    const IndDev32& P = a.P;
    PhysOut out{-1, {0ull, 0ull, 0ull, 0ull, 0ull}};
    // the quotas are loaded with the environment
    const uint8_t fl = hd.fl, stt = hd.stt;
    const int32_t code = hd.code;
    if (!(fl & F32_AC)) return out;
    const int ac0 = stt & F32_ST_AC0;
    int q;
    bool inside;
    if (stt & F32_ST_STALE) {
        int xi, yi, zi;
        unpack_halo(m, P.scell[g], xi, yi, zi);
        q = gid3(m, xi, yi, zi);
        inside = interior_q(m, q);
    } else {
        int ci, cj, ck;
        unpack_int(m, code, ci, cj, ck);
        q = q_of(m, ci, cj, ck);
        inside = ci < m.Nx && cj < m.Ny && ck < m.Nz;
    }
    const long long cq = m.cell_off + q;
    const long long G = a.Gtot;
    const SpeciesDev32& p = a.sp[mi * a.T.nsp + s];
    const float dT = a.dT;
    float NH4 = 0.0f, NO3 = 0.0f, PO4 = 0.0f, DOC = 0.0f, parv = 0.0f, Tm = 0.0f, popv = 0.0f;
    if (ac0 && inside) {
        const float4 e0 = hd.env ? hd.e0 : a.env[2 * cq], e1 = hd.env ? hd.e1 : a.env[2 * cq + 1];
        NH4 = fmaxf(0.0f, e0.x); NO3 = fmaxf(0.0f, e0.y); PO4 = fmaxf(0.0f, e0.z); DOC = fmaxf(0.0f, e0.w);
        parv = e1.x; Tm = e1.y;
        popv = a.pop_sp ? (float)a.pop_sp[(long long)s * G + cq] : e1.z;
    } else if (ac0) {
        // a cell on the halo face (a position exactly at x = Nx): read the fields themselves
        NH4 = fmaxf(0.0f, a.tr[PI_NH4 * G + cq]); NO3 = fmaxf(0.0f, a.tr[PI_NO3 * G + cq]);
        PO4 = fmaxf(0.0f, a.tr[PI_PO4 * G + cq]); DOC = fmaxf(0.0f, a.tr[PI_DOC * G + cq]);
        parv = a.par[cq];
        Tm = a.F[mi].temp[q];
        popv = (float)(a.pop_sp ? a.pop_sp[(long long)s * G + cq] : a.pop[cq]);
    }
    float Bm = hd.Bm, Cq = hd.Cq, Nq = hd.Nq, Pq = hd.Pq, Chl = hd.Chl;
    const double fx_inv = m.fx_inv;         // read before the stores below
    const float tf = tempFunc_f(Tm, p);
    // calc_inorganic_uptake_kernel! (:48-56)
    const float aI = parv * p.alpha * p.Phi;
    const float PCm = p.PCmax * tempFunc_PS_f(Tm, p);
    const float PS = PCm * (1.0f - expf(-aI / fmaxf(1.0e-30f, PCm) * Chl / fmaxf(1.0e-30f, Bm))) * Bm;
    const float Qn = (Nq + Bm * p.R_NC) / fmaxf(1.0e-30f, Bm + Cq);
    const float Qp = (Pq + Bm * p.R_PC) / fmaxf(1.0e-30f, Bm + Cq);
    const float regQN = shape_dec_f(Qn, p.Nqmax, 1.0e-4f, 4), regQP = shape_dec_f(Qp, p.Pqmax, 1.0e-4f, 4);
    const float ipop = fmaxf(1.0f, popv);
    const float VNH4 = fminf(p.VNH4max * regQN * NH4 / fmaxf(1.0e-30f, NH4 + p.KsatNH4) * tf * Bm, NH4 / dT / ipop);
    const float VNO3 = fminf(p.VNO3max * regQN * NO3 / fmaxf(1.0e-30f, NO3 + p.KsatNO3) * tf * Bm, NO3 / dT / ipop);
    const float VPO4 = fminf(p.VPO4max * regQP * PO4 / fmaxf(1.0e-30f, PO4 + p.KsatPO4) * tf * Bm, PO4 / dT / ipop);
    // update_quotas_1_kernel! (:64-69)
    Cq += PS * dT; Pq += VPO4 * dT; Nq += (VNH4 + VNO3) * dT;
    // calc_organic_uptake_kernel! (:78-84)
    const float Qc = Cq / fmaxf(1.0e-30f, Bm + Cq);
    const float regQ = shape_dec_f(Qc, p.Cqmax, 1.0e-4f, 4);
    float VDOC = fminf(p.VDOCmax * regQ * DOC / fmaxf(1.0e-30f, DOC + p.KsatDOC) * tf * Bm, DOC / dT / ipop);
    VDOC = mulbf(VDOC, jl_lessf(1.0e-2f, PS / (VDOC + PS)));
    // calc_ρChl_kernel! (:92-97)
    const float rChl = mulbf(PS / fmaxf(1.0e-30f, Bm) * p.Chl2N / fmaxf(1.0e-30f, parv * p.alpha * p.Phi * Chl / Bm),
                             jl_lessf(1.0e-1f, parv));
    // calc_respir_kernel! (:105-108)
    const float resp = p.respir * Bm * tf;
    // update_quotas_2_kernel! (:117-124)
    Cq = Cq + (VDOC - resp) * dT;
    const float def = fmaxf(0.0f, 0.0f - Cq);
    Bm = Bm - def; Nq = Nq + def * p.R_NC; Pq = Pq + def * p.R_PC; Cq = Cq + def;
    // calc_BS_kernel! (:132-138)
    const float mn = fminf(fminf(Cq, Nq / p.R_NC), Pq / p.R_PC);
    const float BS = mn * p.k_mtb, exu = fmaxf(0.0f, Cq - mn) * p.k_mtb;
    // update_biomass_kernel! (:146-154)
    Bm += dT * BS; Cq -= dT * (BS + exu); Nq -= dT * BS * p.R_NC; Pq -= dT * BS * p.R_PC;
    Chl += dT * BS * p.R_NC * rChl;
    const float age = hd.age + dT / 3600.0f;
    // update_cellsize_kernel! (:163-166) and the probabilities (division_death_probability.jl:7-68)
    const float Sz = Bm / (p.Cquota * p.Nsuper);
    const float graz = popv * p.grz_P;
    const float mort = p.mort_P * shape_dec_f(Sz, p.mort_reg, 1.0e-5f, 4);
    float dv;
    if (p.dvid_type == 1) dv = p.dvid_P * shape_inc_f(Sz, p.dvid_reg, 2.0e-3f, 2);
    else {
        const float h = (float)(fmod(tnow, 86400.0) / 3600.0);
        if (p.dvid_type == 2) dv = p.dvid_P * shape_inc_f(h, p.dvid_reg, 1.0e-5f, 4);
        else dv = p.dvid_P * shape_inc_f(Sz, p.dvid_reg, 1.0e-3f, 4) * shape_inc_f(h, p.dvid_reg2, 1.0e-5f, 4);
    }
    // get_probability! (:95-107)
    float r0, r1, r2;
    draw3f(m.seed, iter, (uint32_t)s, PI_DRAW_DECISION, (uint32_t)hd.ls, r0, r1, r2);
    int dg = jl_lessf(r0, graz * dT), dm = jl_lessf(r1, mort * dT), dd = jl_lessf(r2, dv * dT);
    if (near_threshold(r0, graz * dT) || near_threshold(r1, mort * dT) || near_threshold(r2, dv * dT)) {
        // the same probabilities in Float64 from the Float32 state (the constants are the Float32
        // literals of the reference's formulas)
        const SpeciesDec64& q = a.dec64[mi * a.T.nsp + s];
        const double dTd = (double)dT, Sz64 = (double)Bm / q.CqNs;
        const double g64 = (double)popv * q.grz_P;
        const double m64 = q.mort_P * shape_dec_d(Sz64, q.mort_reg, (double)1.0e-5f, 4);
        double d64;
        if (q.dvid_type == 1) d64 = q.dvid_P * (1.0 - shape_dec_d(Sz64, q.dvid_reg, (double)2.0e-3f, 2));
        else {
            const double h = fmod(tnow, 86400.0) / 3600.0;
            if (q.dvid_type == 2) d64 = q.dvid_P * (1.0 - shape_dec_d(h, q.dvid_reg, (double)1.0e-5f, 4));
            else d64 = q.dvid_P * (1.0 - shape_dec_d(Sz64, q.dvid_reg, (double)1.0e-3f, 4)) *
                       (1.0 - shape_dec_d(h, q.dvid_reg2, (double)1.0e-5f, 4));
        }
        const int dg2 = (double)r0 < g64 * dTd, dm2 = (double)r1 < m64 * dTd, dd2 = (double)r2 < d64 * dTd;
        atomicAdd(&a.guard[0], 1ull);
        if (dg2 != dg || dm2 != dm || dd2 != dd) atomicAdd(&a.guard[1], 1ull);
        dg = dg2; dm = dm2; dd = dd2;
    }
    P.Bm[g] = Bm; P.Cq[g] = Cq; P.Nq[g] = Nq; P.Pq[g] = Pq; P.Chl[g] = Chl; P.age[g] = age;
    P.flags[g] = (uint8_t)(F32_AC | (dg ? F32_GRAZ : 0) | (dm ? F32_MORT : 0) | (dd ? F32_DVID : 0));
    // calc_consume_kernel! (consume_loss.jl:2-9): only individuals binned this step reach the grid
    out.cq = cq;                // diags num at the (possibly stale) cell
    if (ac0 && inside) {
        const double u = fx_inv;
        out.v[0] = to_fixed((resp - PS) * dT, u);
        out.v[1] = to_fixed((exu - VDOC) * dT, u);
        out.v[2] = to_fixed(-VNH4 * dT, u);
        out.v[3] = to_fixed(-VNO3 * dT, u);
        out.v[4] = to_fixed(-VPO4 * dT, u);
    }
    // diags_spcs! (Diagnostics/diagnostics_kernels.jl:14-33) at the same cell
    if (a.pmask) {
        const float v[PI_NPROC] = { PS, BS, VDOC, VNH4, VNO3, VPO4, resp, exu, Bm, Cq, Nq, Pq, Chl };
        for (int q = 0; q < PI_NPROC; ++q)
            if (a.pmask >> q & 1u) add_fixed(&a.dproc[((long long)s * PI_NPROC + q) * G + cq], v[q], 1.0 / proc_unit(m, q));
    }
    return out;
}

// k32_physiology's grid sums of one warp (segment s of one member): one atomic per run of a cell
__device__ __forceinline__ void scatter_phys(const PhysArgs& a, int s, const PhysOut& o) {
    if (__all_sync(0xffffffffu, o.cq < 0)) return;      // a warp of inactive slots adds nothing
    const WarpRuns R = warp_runs(o.cq);
    const int n = (int)run_sum(o.cq >= 0 ? 1u : 0u, R);
    unsigned long long v[5];
#pragma unroll
    for (int e = 0; e < 5; ++e) v[e] = run_sum(o.v[e], R);
    if (R.head && o.cq >= 0) {
        const long long G = a.Gtot, cq = o.cq;
        atomicAdd(&a.dcnt[(long long)s * 4 * G + cq], (uint32_t)n);
        const int slot_of[5] = { ACC_DIC, ACC_DOC, ACC_NH4, ACC_NO3, ACC_PO4 };
#pragma unroll
        for (int e = 0; e < 5; ++e)
            if (v[e]) atomicAdd(&a.acc[(long long)slot_of[e] * G + cq], v[e]);
    }
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) k32_physiology(PhysArgs a) {
    if (stopped(a.err)) return;
    const int bs = blockDim.x, ppt = F32_TILE / bs;
    const uint32_t iter = (uint32_t)(a.st->iteration + 1);
    const double tnow = (double)(a.st->iteration + 1) * (double)a.dT;
    for (int t = blockIdx.x; t < a.T.ntiles; t += gridDim.x) {
        const int2 tl = a.T.tiles[t];
        int mi, s;
        seg_of(a.T, tl.x, mi, s);
        const MemberDev& m = a.T.md[mi];
        const long long base = m.slot_off + (long long)s * m.C;
        long long slot = (long long)tl.y + threadIdx.x;
        PHead hd = phys_head(a.P, base + slot, phys_pre(a.P, base + slot, slot < m.C), m, a.env);
        PPre pre = phys_pre(a.P, base + slot + bs, 1 < ppt && slot + bs < m.C);
        for (int p = 0; p < ppt; ++p, slot += bs) {
            const PHead cur = hd;
            if (p + 1 < ppt) {
                hd = phys_head(a.P, base + slot + bs, pre, m, a.env);
                pre = phys_pre(a.P, base + slot + 2 * bs, p + 2 < ppt && slot + 2 * bs < m.C);
            }
            PhysOut o{-1, {0ull, 0ull, 0ull, 0ull, 0ull}};
            if (slot < m.C) o = phys_one(a, m, mi, s, base + slot, iter, tnow, cur);
            scatter_phys(a, s, o);
        }
    }
}

// ------------------------------------------------------------------------------------------
// (d) tracer update in Float32: the three DST3FL sweeps (DST3FL.jl:1-73, multi_dim_adv.jl:1-135)
//     and the rest of tracer_update! (tracer_update.jl:22-43) in two kernels: k32_xy (x and y
//     sweeps of a level tile staged in shared memory) and k32_ztail (z sweep walking columns, then
//     diffusion, sinking, forcing, boundary fluxes, particle terms and apply_tendency!). Both
//     handle all 14 tracers per thread, so face coefficients and indices are formed once per face.
//
// The flux limiter is evaluated without forming θ: for the upwind side,
//   ψ(δ/δ⁰)·δ⁰ = max(0, min(δ⁰, d₀δ⁰ + d₁δ, Rδ)) for δ⁰ ≥ 0 and min(0, max(δ⁰, d₀δ⁰ + d₁δ, Rδ))
//   for δ⁰ < 0, R = (1 − cfl)/(cfl + 1e-20),
// which equals ψ(θ)·δ⁰ (the θmax cap never changes ψ) and needs no division by δ⁰, so gradients
// near zero are exact. The downwind term of the reference multiplies a zero transport and is
// dropped.
// ------------------------------------------------------------------------------------------
//
// Every product and sum of the tracer update is written with an explicit rounding intrinsic
// (__fmul_rn, __fadd_rn, __fsub_rn, and __fmaf_rn where a fused multiply-add is chosen), so the
// compiler contracts nothing on its own: the kernels that evaluate these formulas (k32_xy and
// k32_ztail, and the fused k32_tracer) give the same bits in whatever code they are inlined into.
struct FCu { float tr, d0c, d1c, R; };

__device__ __forceinline__ FCu fcu(float vel, float area, float rdxc, float dT) {
    FCu f;
    const float cfl = fabsf(__fmul_rn(__fmul_rn(vel, dT), rdxc));
    f.tr = __fmul_rn(area, vel);
    f.d0c = __fmul_rn(__fmul_rn(__fsub_rn(2.0f, cfl), __fsub_rn(1.0f, cfl)), 1.0f / 6.0f);
    f.d1c = __fmul_rn(__fmaf_rn(-cfl, cfl, 1.0f), 1.0f / 6.0f);
    f.R = __fdividef(__fsub_rn(1.0f, cfl), __fadd_rn(cfl, EPS20_F));
    return f;
}
__device__ __forceinline__ float psid0(float d0, float dn, const FCu& f) {
    const float a = __fmaf_rn(f.d0c, d0, __fmul_rn(f.d1c, dn)), b = __fmul_rn(f.R, dn);
    return d0 >= 0.0f ? fmaxf(0.0f, fminf(fminf(d0, a), b)) : fminf(0.0f, fmaxf(fmaxf(d0, a), b));
}
// one sweep's update v − dtv·(ΔF − c·ftr) (multi_dim_adv.jl:111-135)
__device__ __forceinline__ float upd_sweep(float v, float dtv, float dF, float c, float ftr) {
    return __fmaf_rn(-dtv, __fmaf_rn(-c, ftr, dF), v);
}
// a·x1 − a·x0: the transport difference of a cell's two faces
__device__ __forceinline__ float tdiff(float a, float x1, float x0) { return __fmaf_rn(a, x1, -__fmul_rn(a, x0)); }
// tracer_forcing! of a nutrient tracer on max(0, ·): G + (aS·T + aO·T_partner)
__device__ __forceinline__ float add_forcing(float G, float aS, float own, float aO, float partner) {
    return __fadd_rn(G, __fmaf_rn(aS, fmaxf(0.0f, own), __fmul_rn(aO, fmaxf(0.0f, partner))));
}
// tracer_sinking!: G + (ws·T_above − ws·T)·ΔT/ΔzC
__device__ __forceinline__ float add_sinking(float G, float fup, float fdn, float sk) {
    return __fmaf_rn(__fsub_rn(fup, fdn), sk, G);
}
// the new tracer value T + (G + particle term) (apply_tendency!)
__device__ __forceinline__ float tendency(float c, float G, float plk) { return __fadd_rn(c, __fadd_rn(G, plk)); }
// landmask product of a difference (δ·mask_a·mask_b); LM = false: every cell is water
template <bool LM>
__device__ __forceinline__ float mk(float x, int ma, int mb) { return LM ? mulbf(mulbf(x, ma), mb) : x; }

// adv_flux_x / adv_flux_y at a face from c[f-2], c[f-1], c[f], c[f+1] and the landmask there; the
// upwind side is selected, not branched on (a zero transport gives a zero flux either way)
template <bool LM>
__device__ __forceinline__ float flux_h(const FCu& f, float cm2, float cm1, float c0, float cp1,
                                        int lm2, int lm1, int l0, int lp1) {
    const float d0 = mk<LM>(__fsub_rn(c0, cm1), l0, lm1);
    const bool pos = f.tr > 0.0f;
    const float dn = pos ? mk<LM>(__fsub_rn(cm1, cm2), lm1, lm2) : mk<LM>(__fsub_rn(cp1, c0), lp1, l0);
    const float ps = psid0(d0, dn, f);
    return __fmul_rn(f.tr, pos ? __fadd_rn(cm1, ps) : __fsub_rn(c0, ps));
}
// adv_flux_z at face k from c[k-2], c[k-1], c[k], c[k+1] (the index grows downward)
template <bool LM>
__device__ __forceinline__ float flux_v(const FCu& f, float cm2, float cm1, float c0, float cp1,
                                        int lm2, int lm1, int l0, int lp1) {
    const float d0 = mk<LM>(__fsub_rn(cm1, c0), l0, lm1);
    const bool pos = f.tr > 0.0f;
    const float dn = pos ? mk<LM>(__fsub_rn(c0, cp1), lp1, l0) : mk<LM>(__fsub_rn(cm2, cm1), lm1, lm2);
    const float ps = psid0(d0, dn, f);
    return __fmul_rn(f.tr, pos ? __fadd_rn(c0, ps) : __fsub_rn(cm1, ps));
}
__device__ __forceinline__ int wrap_ax(int a, int N, int H, int topo) {
    if (topo == PI_PERIODIC) { while (a < H + 1) a += N; while (a > N + H) a -= N; return a; }
    return a < H + 1 ? H + 1 : (a > N + H ? N + H : a);
}

__device__ __forceinline__ int acc_slot(int n) {
    switch (n) {
        case PI_DIC: return ACC_DIC; case PI_NH4: return ACC_NH4; case PI_NO3: return ACC_NO3;
        case PI_PO4: return ACC_PO4; case PI_DOC: return ACC_DOC; case PI_DON: return ACC_DON;
        case PI_DOP: return ACC_DOP; case PI_POC: return ACC_POC; case PI_PON: return ACC_PON;
        case PI_POP: return ACC_POP; default: return -1;
    }
}

__device__ __forceinline__ float getbc32(const FluxBC32& b, int a, int c, int64_t it) {
    if (b.kind == PI_BC_CONST) return b.v[0];
    if (b.kind == PI_BC_ARRAY2D) return b.v[(a - 1) + (long long)b.n1 * (c - 1)];
    const int64_t t = it < 1 ? 1 : (it > b.nt ? b.nt : it);   // the host rejects steps past nt
    return b.v[(a - 1) + (long long)b.n1 * ((c - 1) + (long long)b.n2 * (t - 1))];
}

// Pairs of FP32 values — the same cell of tracers 2p and 2p+1 — in one 64-bit register, for the
// packed FP32 instructions of sm_100 (add/sub/mul/fma .rn.f32x2). Each half is rounded exactly as the
// scalar __fadd_rn, __fsub_rn, __fmul_rn and __fmaf_rn, so the packed x-y tile gives the same bits
// as xy_tile while issuing one instruction for two tracers.
typedef unsigned long long fx2;
__device__ __forceinline__ fx2 fx2_of(float lo, float hi) {
    fx2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void fx2_split(fx2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ fx2 fx2_add(fx2 a, fx2 b) { fx2 d; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ fx2 fx2_sub(fx2 a, fx2 b) { fx2 d; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ fx2 fx2_mul(fx2 a, fx2 b) { fx2 d; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ fx2 fx2_fma(fx2 a, fx2 b, fx2 c) {
    fx2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ fx2 fx2_neg(fx2 a) { return a ^ 0x8000000080000000ull; }   // exact sign flips

// the face coefficients of one face for both halves
struct FCu2 { fx2 tr, d0c, d1c, R; bool pos; };
__device__ __forceinline__ FCu2 fcu2(const FCu& f) {
    FCu2 g;
    g.tr = fx2_of(f.tr, f.tr); g.d0c = fx2_of(f.d0c, f.d0c); g.d1c = fx2_of(f.d1c, f.d1c); g.R = fx2_of(f.R, f.R);
    g.pos = f.tr > 0.0f;
    return g;
}
// flux_h of an all-water face for two tracers: the upwind operands are selected first (the
// selected difference and the sum c0 − ψ = c0 + (−ψ) are the same IEEE operations), the limiter
// (min/max, no packed form) runs per half
__device__ __forceinline__ fx2 flux_h2(const FCu2& f, fx2 cm2, fx2 cm1, fx2 c0, fx2 cp1) {
    const fx2 d0 = fx2_sub(c0, cm1);
    const fx2 dn = f.pos ? fx2_sub(cm1, cm2) : fx2_sub(cp1, c0);
    const fx2 a = fx2_fma(f.d0c, d0, fx2_mul(f.d1c, dn)), b = fx2_mul(f.R, dn);
    float d0l, d0h, al, ah, bl, bh;
    fx2_split(d0, d0l, d0h); fx2_split(a, al, ah); fx2_split(b, bl, bh);
    const float pl = d0l >= 0.0f ? fmaxf(0.0f, fminf(fminf(d0l, al), bl)) : fminf(0.0f, fmaxf(fmaxf(d0l, al), bl));
    const float ph = d0h >= 0.0f ? fmaxf(0.0f, fminf(fminf(d0h, ah), bh)) : fminf(0.0f, fmaxf(fmaxf(d0h, ah), bh));
    const fx2 ps = fx2_of(pl, ph);
    return fx2_mul(f.tr, f.pos ? fx2_add(cm1, ps) : fx2_add(c0, fx2_neg(ps)));
}
// upd_sweep for two tracers: v − dtv·(ΔF − c·ftr)
__device__ __forceinline__ fx2 upd_sweep2(fx2 v, fx2 ndtv, fx2 dF, fx2 c, fx2 ftr) {
    return fx2_fma(ndtv, fx2_fma(fx2_neg(c), ftr, dF), v);
}

struct TrArgs {
    Tab32 T;
    const int4* items;          // k32_xy: {member, i0, j0, level}; k32_ztail: {member, i0, j, k0}
    int nitems;
    const uint8_t* lm;
    const float* dzF;
    const float* dzC;
    const float* rdzC;          // 1 / dzC
    const BgcDev32* bgc;
    const FluxBC32* bcs;
    const StepState* st;
    const MemberForcing* F;
    long long Gtot;
    const float* tr;            // tracers at the start of the step
    float* tb;                  // tracer_temp after the x and y sweeps
    float* tr_next;
    unsigned long long* acc;
    const int* pop;
    float dT;
    const uint32_t* err;
};

// x and y sweeps of all 14 tracers on one level of a tile of 28 columns × TY rows. Warp w holds
// row j0-2+w (TY+4 rows: the y sweep reads two rows on each side, outside the domain through the
// halo-fill map), lane l column i0-2+l (28 cells and two halo columns on each side, exchanged by
// shuffles). The face coefficients are computed once per face and shared by the 14 tracers.
// Shared memory [row][tracer][lane]: TA (after x), FY (y face fluxes), TRs (tracer of the rows
// the y sweep updates).
// The inputs of one item for this thread (its row and column): u and the 14 tracers of the x
// sweep, and the y velocities it reads later — v at its y face j0 + wid (x) and at the two faces
// of its row (y, z; in range whenever the row is updated). A block loops over items and loads the
// next item's inputs while it works on the current one.
__device__ __forceinline__ void xy_load(const TrArgs& a, int item, float& u, float* v, float3& vy) {
    const int4 it = a.items[item];
    const MemberDev& m = a.T.md[it.x];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int jj = wrap_ax(it.z - 2 + wid, m.Ny, m.Hy, m.ty);
    const int ic = min(it.y - 2 + lane, m.Gx);
    const int q = gid3(m, ic, jj, it.w);
    const MemberForcing& F = a.F[it.x];
    u = F.vel1[0][q];
    const float* __restrict__ src = a.tr + m.cell_off + q;
#pragma unroll
    for (int n = 0; n < PI_NTRACERS; ++n) v[n] = src[n * a.Gtot];
    const int f = it.z + wid;
    const int fs = f == m.Ny + m.Hy + 1 ? m.Hy + 1 : min(f, m.Ny + m.Hy);
    const int jr = min(f, m.Gy - 1);
    const float* __restrict__ vv = F.vel1[1];
    vy.x = vv[gid3(m, ic, fs, it.w)];
    const int qr = gid3(m, ic, jr, it.w);
    vy.y = vv[qr];
    vy.z = vv[qr + m.Gx];
}

template <int TY, bool LM>
__device__ __forceinline__ void xy_tile(const TrArgs& a, const MemberDev& m, const int4 it, float* sm,
                                        float& pu, float* pv, float3& pvy, int next) {
    float* TA = sm;                                        // (TY+4) × 14 × 32
    float* FY = TA + (TY + 4) * PI_NTRACERS * 32;          // (TY+1) × 14 × 32
    float* TRs = FY + (TY + 1) * PI_NTRACERS * 32;         // TY × 14 × 32
    auto at = [](float* base, int r, int n, int l) -> float& { return base[(r * PI_NTRACERS + n) * 32 + l]; };
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long G = a.Gtot;
    const float dT = a.dT;
    const int i0 = it.y, j0 = it.z, L = it.w;
    const long long off = m.cell_off;
    const float dz = a.dzF[m.dz_off + L - 1];
    const float az = __fmul_rn(m.dx, m.dy), dtv = __fdiv_rn(dT, __fmul_rn(az, dz));
    // ---- x sweep of row j0-2+wid
    {
        const int jj = wrap_ax(j0 - 2 + wid, m.Ny, m.Hy, m.ty);
        const int i = i0 - 2 + lane;
        const int ic = min(i, m.Gx);
        const float ax = __fmul_rn(m.dy, dz);
        const float uw = pu;
        const float ue = __shfl_down_sync(0xffffffffu, uw, 1);
        const FCu fc = fcu(uw, ax, __frcp_rn(m.dx), dT);
        int l0 = 1, lm1 = 1, lm2 = 1, lp1 = 1;
        if (LM) {
            l0 = lm32(m, a.lm, ic, jj, L);
            lm1 = __shfl_up_sync(0xffffffffu, l0, 1); lm2 = __shfl_up_sync(0xffffffffu, l0, 2);
            lp1 = __shfl_down_sync(0xffffffffu, l0, 1);
        }
        const bool east_zero = i == m.Nx + m.Hx && m.tx != PI_PERIODIC;   // fill_halo_east_Gc! (Bounded)
        const float ftr = mk<LM>(tdiff(ax, ue, uw), lp1, l0);
        const bool store_tr = wid >= 2 && wid < TY + 2;
#pragma unroll
        for (int n = 0; n < PI_NTRACERS; ++n) {
            const float v = pv[n];
            const float cm2 = __shfl_up_sync(0xffffffffu, v, 2), cm1 = __shfl_up_sync(0xffffffffu, v, 1);
            const float cp1 = __shfl_down_sync(0xffffffffu, v, 1);
            const float Fw = flux_h<LM>(fc, cm2, cm1, v, cp1, lm2, lm1, l0, lp1);
            float Fe = __shfl_down_sync(0xffffffffu, Fw, 1);
            if (east_zero) Fe = 0.0f;
            at(TA, wid, n, lane) = upd_sweep(v, dtv, mk<LM>(__fsub_rn(Fe, Fw), lp1, l0), v, ftr);
            if (store_tr) at(TRs, wid - 2, n, lane) = v;
        }
    }
    __syncthreads();
    // the registers of this item's x inputs are free: start the next item's loads
    const float3 vy = pvy;
    if (next < a.nitems) xy_load(a, next, pu, pv, pvy);
    // ---- y faces j0 + r, r = 0..TY
    const int i = i0 - 2 + lane;
    const bool col = lane >= 2 && lane < 30 && i <= m.Nx + m.Hx;
    const float ay = __fmul_rn(m.dx, dz);
    if (wid <= TY) {
        const int r = wid, f = j0 + r;
        const bool special = f == m.Ny + m.Hy + 1;
        const bool zero = !col || f > m.Ny + m.Hy + 1 || (special && m.ty != PI_PERIODIC);
        const int fs = special ? m.Hy + 1 : min(f, m.Ny + m.Hy);
        const int ic = min(i, m.Gx);
        const FCu fc = fcu(zero ? 0.0f : vy.x, ay, __frcp_rn(m.dy), dT);
        int L2 = 1, L1 = 1, L0 = 1, Lp = 1;
        if (LM) {
            L2 = lm32(m, a.lm, ic, fs - 2, L); L1 = lm32(m, a.lm, ic, fs - 1, L);
            L0 = lm32(m, a.lm, ic, fs, L); Lp = lm32(m, a.lm, ic, fs + 1, L);
        }
#pragma unroll
        for (int n = 0; n < PI_NTRACERS; ++n)
            at(FY, r, n, lane) = zero ? 0.0f : flux_h<LM>(fc, at(TA, r, n, lane), at(TA, r + 1, n, lane), at(TA, r + 2, n, lane),
                                                          at(TA, r + 3, n, lane), L2, L1, L0, Lp);
    }
    __syncthreads();
    // ---- y update of row j0 + wid
    if (wid < TY) {
        const int j = j0 + wid;
        if (col && j <= m.Ny + m.Hy) {
            const int q = gid3(m, i, j, L);
            const int c0m = LM ? lm32(m, a.lm, i, j, L) : 1, cpm = LM ? lm32(m, a.lm, i, j + 1, L) : 1;
            const float ftr = mk<LM>(tdiff(ay, vy.z, vy.y), cpm, c0m);
            float* dst = a.tb + off + q;
#pragma unroll
            for (int n = 0; n < PI_NTRACERS; ++n) {
                const float dG = mk<LM>(__fsub_rn(at(FY, wid + 1, n, lane), at(FY, wid, n, lane)), cpm, c0m);
                dst[n * G] = upd_sweep(at(TA, wid + 2, n, lane), dtv, dG, at(TRs, wid, n, lane), ftr);
            }
        }
    }
    __syncthreads();
}

// xy_tile for an all-water member with the 14 tracers handled as 7 packed pairs: the same tile,
// threads and operations, with shared memory laid out [row][pair][lane] of 64-bit pairs so that a
// lane reads or writes both tracers of a pair with one access.
template <int TY>
__device__ __forceinline__ void xy_tile_pk(const TrArgs& a, const MemberDev& m, const int4 it, float* sm,
                                           float& pu, float* pv, float3& pvy, int next) {
    constexpr int NP = PI_NTRACERS / 2;
    fx2* TA = reinterpret_cast<fx2*>(sm);                 // (TY+4) × 7 × 32
    fx2* FY = TA + (TY + 4) * NP * 32;                     // (TY+1) × 7 × 32
    fx2* TRs = FY + (TY + 1) * NP * 32;                    // TY × 7 × 32
    auto at = [](fx2* base, int r, int p, int l) -> fx2& { return base[(r * NP + p) * 32 + l]; };
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long G = a.Gtot;
    const float dT = a.dT;
    const int i0 = it.y, j0 = it.z, L = it.w;
    const long long off = m.cell_off;
    const float dz = a.dzF[m.dz_off + L - 1];
    const float az = __fmul_rn(m.dx, m.dy), dtv = __fdiv_rn(dT, __fmul_rn(az, dz));
    const fx2 ndtv = fx2_of(-dtv, -dtv);
    // ---- x sweep of row j0-2+wid
    {
        const int i = i0 - 2 + lane;
        const float ax = __fmul_rn(m.dy, dz);
        const float uw = pu;
        const float ue = __shfl_down_sync(0xffffffffu, uw, 1);
        const FCu2 fc = fcu2(fcu(uw, ax, __frcp_rn(m.dx), dT));
        const bool east_zero = i == m.Nx + m.Hx && m.tx != PI_PERIODIC;   // fill_halo_east_Gc! (Bounded)
        const float ftr1 = tdiff(ax, ue, uw);
        const fx2 ftr = fx2_of(ftr1, ftr1);
        const bool store_tr = wid >= 2 && wid < TY + 2;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const float v0 = pv[2 * p], v1 = pv[2 * p + 1];
            const fx2 v = fx2_of(v0, v1);
            const fx2 cm2 = fx2_of(__shfl_up_sync(0xffffffffu, v0, 2), __shfl_up_sync(0xffffffffu, v1, 2));
            const fx2 cm1 = fx2_of(__shfl_up_sync(0xffffffffu, v0, 1), __shfl_up_sync(0xffffffffu, v1, 1));
            const fx2 cp1 = fx2_of(__shfl_down_sync(0xffffffffu, v0, 1), __shfl_down_sync(0xffffffffu, v1, 1));
            const fx2 Fw = flux_h2(fc, cm2, cm1, v, cp1);
            float wl, wh;
            fx2_split(Fw, wl, wh);
            fx2 Fe = fx2_of(__shfl_down_sync(0xffffffffu, wl, 1), __shfl_down_sync(0xffffffffu, wh, 1));
            if (east_zero) Fe = 0ull;
            at(TA, wid, p, lane) = upd_sweep2(v, ndtv, fx2_sub(Fe, Fw), v, ftr);
            if (store_tr) at(TRs, wid - 2, p, lane) = v;
        }
    }
    __syncthreads();
    // the registers of this item's x inputs are free: start the next item's loads
    const float3 vy = pvy;
    if (next < a.nitems) xy_load(a, next, pu, pv, pvy);
    // ---- y faces j0 + r, r = 0..TY
    const int i = i0 - 2 + lane;
    const bool col = lane >= 2 && lane < 30 && i <= m.Nx + m.Hx;
    const float ay = __fmul_rn(m.dx, dz);
    if (wid <= TY) {
        const int r = wid, f = j0 + r;
        const bool special = f == m.Ny + m.Hy + 1;
        const bool zero = !col || f > m.Ny + m.Hy + 1 || (special && m.ty != PI_PERIODIC);
        const FCu2 fc = fcu2(fcu(zero ? 0.0f : vy.x, ay, __frcp_rn(m.dy), dT));
#pragma unroll
        for (int p = 0; p < NP; ++p)
            at(FY, r, p, lane) = zero ? 0ull : flux_h2(fc, at(TA, r, p, lane), at(TA, r + 1, p, lane), at(TA, r + 2, p, lane),
                                                      at(TA, r + 3, p, lane));
    }
    __syncthreads();
    // ---- y update of row j0 + wid
    if (wid < TY) {
        const int j = j0 + wid;
        if (col && j <= m.Ny + m.Hy) {
            const int q = gid3(m, i, j, L);
            const float ftr1 = tdiff(ay, vy.z, vy.y);
            const fx2 ftr = fx2_of(ftr1, ftr1);
            float* dst = a.tb + off + q;
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const fx2 dG = fx2_sub(at(FY, wid + 1, p, lane), at(FY, wid, p, lane));
                float lo, hi;
                fx2_split(upd_sweep2(at(TA, wid + 2, p, lane), ndtv, dG, at(TRs, wid, p, lane), ftr), lo, hi);
                dst[(2 * p) * G] = lo;
                dst[(2 * p + 1) * G] = hi;
            }
        }
    }
    __syncthreads();
}

template <int TY>
__global__ void __launch_bounds__(32 * (TY + 4)) k32_xy(TrArgs a) {
    if (stopped(a.err)) return;
    extern __shared__ float sm[];
    if ((int)blockIdx.x >= a.nitems) return;
    float pu, pv[PI_NTRACERS];
    float3 pvy;
    xy_load(a, blockIdx.x, pu, pv, pvy);
    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
        const int4 it = a.items[item];
        const MemberDev& m = a.T.md[it.x];
        const int next = item + gridDim.x;
        if (m.all_water) xy_tile_pk<TY>(a, m, it, sm, pu, pv, pvy, next);
        else xy_tile<TY, true>(a, m, it, sm, pu, pv, pvy, next);
    }
}

// z sweep and the rest of tracer_update! for LZ levels of 32 columns: warp y of the block takes
// tracer y and each lane walks its column keeping the 4-level stencil window of tracer_temp and
// the flux of the face above the current cell. What does not depend on the tracer is formed once
// per item in shared memory for the 14 tracer warps: the face coefficients, the vertical
// transport term of each cell, the cell counts and the per-level constants (ΔT/vol, ΔT/ΔzC and
// the fixed-point unit per volume). As the warps walk the same cells, the forcing terms' reads of
// the other tracers at a cell hit lines already loaded.
struct ZLev {
    float dtv;      // ΔT / (Δx Δy ΔzF[k])
    float sk;       // ΔT / ΔzC (tracer_sinking!)
    float dz;       // ΔzF[k]
    float dzn;      // ΔzF[k+1]
    double fxv;     // mmol per fixed-point unit / (Δx Δy ΔzF[k])
};

// tracer_forcing! (tracer_forcings.jl:2-50) of the three iron tracers on max(0, tracer), with the
// products of rate constants and ΔT formed once per walk
struct FeCoef { float kpoc, frac, kdiss, fefe, frac_poc, lig, lpoc, lmin, ldust; };
__device__ __forceinline__ FeCoef fe_coef(const BgcDev32& b, float dT) {
    FeCoef c;
    c.kpoc = b.kPOC * dT; c.frac = b.DFeFrac * dT; c.kdiss = b.kdiss * dT;
    c.fefe = b.DFeFrac * b.lambda_Fe * dT; c.frac_poc = b.DFeFrac * b.lambda_POC * dT;
    c.lig = b.ligand; c.lpoc = b.lambda_POC; c.lmin = b.lambda_min; c.ldust = b.lambda_dust;
    return c;
}
__device__ __forceinline__ float fe_forcing(int n, const FeCoef& c, float dfe, float poc, float dust, float pfeb, float pfei) {
    const float fe = __fmul_rn(__fmul_rn(fmaxf(__fsub_rn(dfe, c.lig), 0.0f), dfe), c.fefe);
    const float bio = __fmul_rn(pfeb, c.kpoc), diss = __fmul_rn(pfei, c.kdiss);
    if (n == PI_DFe) {
        const float scav = __fadd_rn(__fadd_rn(__fmul_rn(c.lpoc, poc), c.lmin), __fmul_rn(c.ldust, dust));
        return __fsub_rn(__fadd_rn(__fsub_rn(bio, __fmul_rn(__fmul_rn(scav, dfe), c.frac)), diss), fe);
    }
    if (n == PI_PFe_bio) return __fsub_rn(__fmul_rn(__fmul_rn(poc, dfe), c.frac_poc), bio);
    const float scav = __fadd_rn(c.lmin, __fmul_rn(c.ldust, dust));
    return __fadd_rn(__fadd_rn(-diss, __fmul_rn(__fmul_rn(scav, dfe), c.frac)), fe);
}

// Asynchronous global → shared copies (cp.async): a warp's z walk reads the inputs of each level
// from a ring of ZS levels filled ahead of it, so ZS - 1 levels of loads are in flight while it
// computes. A lane reads back only what it copied itself, which wait_group makes visible to it.
__device__ __forceinline__ void cpa4(unsigned sdst, const float* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" :: "r"(sdst), "l"(gsrc) : "memory");
}
// 8 bytes, or zeros without reading when `on` is false
__device__ __forceinline__ void cpa8(unsigned sdst, const unsigned long long* gsrc, bool on) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(sdst), "l"(gsrc), "r"(on ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory"); }
// shared loads ordered after the wait above (volatile asm keeps program order among them)
__device__ __forceinline__ float lds_f32(unsigned a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];\n" : "=f"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ unsigned long long lds_u64(unsigned a) {
    unsigned long long v;
    asm volatile("ld.shared.u64 %0, [%1];\n" : "=l"(v) : "r"(a));
    return v;
}

#define ZS 4                              // levels of a z walk ring (power of two)
// One warp's ring: own tracer c, tracer_temp t two levels below, the other tracers the forcing
// reads and the particle sum of the cell. A nutrient warp uses x[0] and acc; an iron warp reads
// DFe, POC, Dust, PFe_bio, PFe_inorg into x[0..3] and, for the fifth, the first 512 bytes of acc.
struct ZRing {
    float c[ZS][32];
    float t[ZS][32];
    float x[4][ZS][32];
    unsigned long long acc[ZS][32];
};
static_assert(ZS == 4 && offsetof(ZRing, t) == 512 && offsetof(ZRing, x) == 1024 && offsetof(ZRing, acc) == 3072 &&
              sizeof(ZRing) == 4096, "z walk ring layout");

// NUT: the ten nutrient tracers (linear forcing, particle sums); otherwise the three iron tracers
// and dust (iron forcing, sinking). GEN: diffusion or flux boundary conditions are switched on.
template <int LZ, bool LM, bool NUT, bool GEN>
__device__ __forceinline__ void z_walk(const TrArgs& a, const MemberDev& md, const int4 it, const float4* sFC,
                                       const float* sFtr, const int* sPop, const ZLev* sLev, ZRing& R) {
    const int lane = threadIdx.x, n = threadIdx.y;
    // member constants in registers: the stores of the walk could otherwise alias them
    const int Nx = md.Nx, Hx = md.Hx, Hz = md.Hz, Gx = md.Gx, Gy = md.Gy;
    const int i = it.y + lane, j = it.z, k0 = it.w;
    // levels of the walk where any of the 32 columns holds an individual: only those have
    // particle sums to read and zero (a warp-uniform test; the others skip the sum's copy)
    uint64_t occm = 0;
    if (NUT) {
#pragma unroll 4
        for (int l = 0; l < LZ; ++l)
            if (__ballot_sync(0xffffffffu, sPop[l * 32 + lane] > 0)) occm |= 1ull << l;
    }
    if (i > Nx + Hx) return;
    const long long G = a.Gtot, off = md.cell_off;
    const float dT = a.dT;
    const int slab = Gx * Gy;
    const int top = Hz + 1, bot = md.Nz + Hz;
    const int kend = min(k0 + LZ - 1, bot);
    const int qcol = (i - 1) + Gx * (j - 1);             // level 1 of the column, member-local
    const BgcDev32& b = a.bgc[it.x];
    const bool sinks = !NUT && n != PI_DFe;
    const float ws = n == PI_PFe_bio ? b.w_sink_org : b.w_sink_inorg;
    // tracer_forcing! of the ten nutrient tracers: aS·T(n) + aO·T(x0) (aO = 0 where there is no
    // second tracer); of the iron tracers: T of DFe, POC, Dust, PFe_bio, PFe_inorg, each the own
    // tracer (-1) or one of the four others x0..x3
    float aS = 0.0f, aO = 0.0f;
    int xo[5] = { n, PI_POC, PI_Dust, PI_PFe_bio, PI_PFe_inorg };
    if (NUT) {
        switch (n) {
            case PI_DIC: xo[0] = PI_DOC; aO = b.kDOC * dT; break;
            case PI_DOC: aS = -b.kDOC * dT; xo[0] = PI_POC; aO = b.kPOC * dT; break;
            case PI_POC: aS = -b.kPOC * dT; break;
            case PI_NH4: aS = -b.Nit * dT; xo[0] = PI_DON; aO = b.kDON * dT; break;
            case PI_NO3: xo[0] = PI_NH4; aO = b.Nit * dT; break;
            case PI_DON: aS = -b.kDON * dT; xo[0] = PI_PON; aO = b.kPON * dT; break;
            case PI_PON: aS = -b.kPON * dT; break;
            case PI_PO4: xo[0] = PI_DOP; aO = b.kDOP * dT; break;
            case PI_DOP: aS = -b.kDOP * dT; xo[0] = PI_POP; aO = b.kPOP * dT; break;
            case PI_POP: aS = -b.kPOP * dT; break;
            default: break;
        }
    } else {
        xo[0] = PI_DFe;
    }
    const FeCoef fc = fe_coef(b, dT);
    // POC, PON and POP force on themselves only: their partner term reads the own value (aO = 0)
    const bool partner = !NUT || xo[0] != n;
    const float* __restrict__ t = a.tb + n * G + off;
    const float* __restrict__ c = a.tr + n * G + off;
    const float* __restrict__ trm = a.tr + off;           // all tracers of the member
    float* __restrict__ out = a.tr_next + n * G + off;
    unsigned long long* __restrict__ acc = a.acc + (NUT ? acc_slot(n) : 0) * G + off;
    const uint8_t* __restrict__ lmc = a.lm + off + qcol;
    auto tl = [&](int kk) { return qcol + (min(max(kk, top), bot) - 1) * slab; };
    auto lmk = [&](int kk) -> int { return LM ? (int)lmc[(kk - 1) * slab] : 1; };
    auto fcz = [&](int l) { const float4 v = sFC[l * 32 + lane]; FCu r; r.tr = v.x; r.d0c = v.y; r.d1c = v.z; r.R = v.w; return r; };
    // ring addresses of this lane (shared space): stage sl of c at rc + 128 sl, t at rc + 512 +
    // 128 sl, x[e] at rc + 1024 + 512 e + 128 sl, the particle sum at ra + 256 sl, the fifth
    // iron tracer at rx4 + 128 sl
    const unsigned rc = (unsigned)__cvta_generic_to_shared(&R.c[0][lane]);
    const unsigned ra = (unsigned)__cvta_generic_to_shared(&R.acc[0][lane]);
    const unsigned rx4 = (unsigned)__cvta_generic_to_shared(&R.acc[0][0]) + 4u * lane;   // iron x[4]: 128 B stages
    const float* __restrict__ x0p = trm + xo[0] * G;
    const float* __restrict__ x1p = trm + xo[1] * G;
    const float* __restrict__ x2p = trm + xo[2] * G;
    const float* __restrict__ x3p = trm + xo[3] * G;
    const float* __restrict__ x4p = trm + xo[4] * G;
    // ring fill of level kk (nothing past the last level: an empty group keeps the wait count)
    auto issue = [&](int kk) {
        if (kk <= kend) {                                     // warp-uniform
            const unsigned so = (unsigned)((kk - k0) & (ZS - 1)) * 128u;
            const int qq = qcol + (kk - 1) * slab;
            cpa4(rc + so, c + qq);
            cpa4(rc + 512u + so, t + tl(kk + 2));
            if (NUT) {
                if (partner) cpa4(rc + 1024u + so, x0p + qq);
                if (occm >> (kk - k0) & 1ull) cpa8(ra + 2u * so, acc + qq, sPop[(kk - k0) * 32 + lane] > 0);
            } else if (n != PI_Dust) {
                cpa4(rc + 1024u + so, x0p + qq);
                cpa4(rc + 1536u + so, x1p + qq);
                cpa4(rc + 2048u + so, x2p + qq);
                cpa4(rc + 2560u + so, x3p + qq);
                cpa4(rx4 + so, x4p + qq);
            }
        }
        cpa_commit();
    };
#pragma unroll
    for (int e = 0; e < ZS - 1; ++e) issue(k0 + e);
    // stencil windows: w (tracer_temp) and mm (land mask) at levels k-1 .. k+2 of the current cell k
    float w0 = t[tl(k0 - 2)], w1 = t[tl(k0 - 1)], w2 = t[tl(k0)], w3 = t[tl(k0 + 1)];
    int mm0 = lmk(k0 - 2), mm1 = lmk(k0 - 1), mm2 = lmk(k0), mm3 = lmk(k0 + 1);
    float Ft = flux_v<LM>(fcz(0), w0, w1, w2, w3, mm0, mm1, mm2, mm3);
    int q = qcol + (k0 - 1) * slab;
    float sink_prev = (sinks && k0 - 1 > Hz) ? c[q - slab] : 0.0f;
    for (int k = k0; k <= kend; ++k, q += slab) {
        const int l = k - k0;
        const unsigned so = (unsigned)(l & (ZS - 1)) * 128u;
        issue(k + ZS - 1);
        cpa_wait<ZS - 1>();
        const float cc = lds_f32(rc + so);
        w0 = w1; w1 = w2; w2 = w3; w3 = lds_f32(rc + 512u + so);
        if (LM) { mm0 = mm1; mm1 = mm2; mm2 = mm3; mm3 = lmk(k + 2); }
        const int l1 = mm1, l0 = mm2;                       // land mask of cell k and k+1
        const float Fb = flux_v<LM>(fcz(l + 1), w0, w1, w2, w3, mm0, mm1, mm2, mm3);   // zero at the bottom
        const ZLev L = sLev[l];
        float Gc = __fsub_rn(upd_sweep(w1, L.dtv, mk<LM>(__fsub_rn(Ft, Fb), l0, l1), cc, sFtr[l * 32 + lane]), cc);
        Ft = Fb;
        if (GEN) {
            // tracer_diffusion! (tracer_diffusion.jl:1-21)
            if (b.kappa_h != 0.0f || b.kappa_v != 0.0f) {
                const float dz = L.dz, az = md.dx * md.dy, volk = az * dz;
                const float axk = md.dy * dz, ayk = md.dx * dz;
                auto lmq = [&](int dq) -> int { return LM ? (int)lmc[(k - 1) * slab + dq] : 1; };
                auto dif = [&](int dq, int dp) { return mulbf(mulbf(c[q + dq] - c[q + dp], lmq(dq)), lmq(dp)); };
                const float fx1 = b.kappa_h * axk * (dif(1, 0) / md.dx), fx0 = b.kappa_h * axk * (dif(0, -1) / md.dx);
                const float fy1 = b.kappa_h * ayk * (dif(Gx, 0) / md.dy), fy0 = b.kappa_h * ayk * (dif(0, -Gx) / md.dy);
                const float fz0 = b.kappa_v * az * (dif(-slab, 0) / dz), fz1 = b.kappa_v * az * (dif(0, slab) / L.dzn);
                const float ax_ = mulbf(mulbf(fx1 - fx0, lmq(1)), l1);
                const float ay_ = mulbf(mulbf(fy1 - fy0, lmq(Gx)), l1);
                const float az_ = mulbf(mulbf(fz0 - fz1, l0), l1);
                Gc += 1.0f / volk * (ax_ + ay_ + az_) * dT;
            }
        }
        if (NUT) {
            // tracer_forcing! (tracer_forcings.jl:2-50) on max(0, tracer)
            Gc = add_forcing(Gc, aS, cc, aO, partner ? lds_f32(rc + 1024u + so) : cc);
        } else {
            // tracer_sinking! (tracer_sinking.jl:1-42)
            if (sinks) {
                const float fup = (k - 1 <= Hz) ? 0.0f : __fmul_rn(ws, sink_prev);
                const float fdn = (k >= bot) ? 0.0f : __fmul_rn(ws, cc);
                Gc = add_sinking(Gc, fup, fdn, L.sk);
                sink_prev = cc;
            }
            if (n != PI_Dust) {
                const float dfe = fmaxf(0.0f, lds_f32(rc + 1024u + so)), poc = fmaxf(0.0f, lds_f32(rc + 1536u + so));
                const float dust = fmaxf(0.0f, lds_f32(rc + 2048u + so)), pfeb = fmaxf(0.0f, lds_f32(rc + 2560u + so));
                const float pfei = fmaxf(0.0f, lds_f32(rx4 + so));
                Gc += fe_forcing(n, fc, dfe, poc, dust, pfeb, pfei);
            }
        }
        if (GEN && md.any_bc) {
            // apply_bcs! (apply_bcs.jl:4-98)
            const int64_t itn = a.st->iteration + 1;
            const FluxBC32* B = a.bcs + md.bc_off + n * 6;
            const int ii = i - Hx, jj = j - md.Hy, kk = k - Hz;
            const float dz = L.dz, az = md.dx * md.dy, volk = az * dz;
            const float axk = md.dy * dz, ayk = md.dx * dz;
            if (B[PI_WEST].kind && i == 1 + Hx) Gc += getbc32(B[PI_WEST], jj, kk, itn) * dT * axk / volk;
            if (B[PI_EAST].kind && i == Nx + Hx) Gc -= getbc32(B[PI_EAST], jj, kk, itn) * dT * axk / volk;
            if (B[PI_SOUTH].kind && j == 1 + md.Hy) Gc += getbc32(B[PI_SOUTH], ii, kk, itn) * dT * ayk / volk;
            if (B[PI_NORTH].kind && j == md.Ny + md.Hy) Gc -= getbc32(B[PI_NORTH], ii, kk, itn) * dT * ayk / volk;
            if (B[PI_BOTTOM].kind && k == bot) Gc += getbc32(B[PI_BOTTOM], ii, jj, itn) * dT * az / volk;
            if (B[PI_TOP].kind && k == top) Gc -= getbc32(B[PI_TOP], ii, jj, itn) * dT * az / volk;
        }
        // particle terms from the fixed-point sums (zeroed as they are consumed), apply_tendency!
        // (tracer_update.jl:6-13)
        float plk = 0.0f;
        if (NUT && (occm >> l & 1ull)) {
            const long long vv = (long long)lds_u64(ra + 2u * so);   // zero where the cell holds no individual
            if (vv) { acc[q] = 0ull; plk = (float)((double)vv * L.fxv); }
        }
        out[q] = tendency(cc, Gc, plk);
    }
    cpa_wait<0>();
}

template <int LZ, bool LM>
__device__ __forceinline__ void z_walk_any(const TrArgs& a, const MemberDev& m, const int4 it, const float4* sFC,
                                           const float* sFtr, const int* sPop, const ZLev* sLev, ZRing& R) {
    const BgcDev32& b = a.bgc[it.x];
    const bool gen = m.any_bc || b.kappa_h != 0.0f || b.kappa_v != 0.0f;
    const bool nut = acc_slot(threadIdx.y) >= 0;
    if (nut) {
        if (gen) z_walk<LZ, LM, true, true>(a, m, it, sFC, sFtr, sPop, sLev, R);
        else z_walk<LZ, LM, true, false>(a, m, it, sFC, sFtr, sPop, sLev, R);
    } else {
        if (gen) z_walk<LZ, LM, false, true>(a, m, it, sFC, sFtr, sPop, sLev, R);
        else z_walk<LZ, LM, false, false>(a, m, it, sFC, sFtr, sPop, sLev, R);
    }
}

// dynamic shared memory of k32_ztail: one ring per tracer warp, then the per-item arrays (face
// coefficients, transport terms, cell counts, per-level constants) of a walk of lz levels
inline size_t ztail_smem(int lz) {
    return sizeof(ZRing) * PI_NTRACERS + (size_t)(lz + 1) * 32 * sizeof(float4) + (size_t)lz * 32 * (sizeof(float) + sizeof(int))
         + (size_t)lz * sizeof(ZLev);
}

template <int LZ>
__global__ void __launch_bounds__(32 * PI_NTRACERS, 2) k32_ztail(TrArgs a) {
    if (stopped(a.err)) return;
    extern __shared__ __align__(16) unsigned char zsm[];
    ZRing* ring = reinterpret_cast<ZRing*>(zsm);
    float4* sFC = reinterpret_cast<float4*>(zsm + sizeof(ZRing) * PI_NTRACERS);   // faces k0 .. k0+LZ of the 32 columns
    float* sFtr = reinterpret_cast<float*>(sFC + (LZ + 1) * 32);       // vertical transport term of the cells k0 .. k0+LZ-1
    int* sPop = reinterpret_cast<int*>(sFtr + LZ * 32);                 // individuals in those cells
    ZLev* sLev = reinterpret_cast<ZLev*>(sPop + LZ * 32);               // per-level constants
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int w = blockIdx.x; w < a.nitems; w += gridDim.x) {
        const int4 it = a.items[w];
        const MemberDev& m = a.T.md[it.x];
        const int k0 = it.w, bot = m.Nz + m.Hz;
        const float* wv = a.F[it.x].vel1[2];
        const float az = __fmul_rn(m.dx, m.dy);
        for (int e = tid; e < (LZ + 1) * 32; e += 32 * PI_NTRACERS) {
            const int f = k0 + e / 32, i = it.y + (e & 31);
            const bool col = i <= m.Nx + m.Hx;
            float4 fc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (col && f <= bot) {                            // fill_halo_bottom_Gc!: zero flux at the bottom
                const int q = gid3(m, i, it.z, f);
                const float wt = wv[q];
                const FCu c = fcu(wt, az, a.rdzC[m.dz_off + f - 1], a.dT);
                fc = make_float4(c.tr, c.d0c, c.d1c, c.R);
                if (e < LZ * 32) {                            // cell f: w at its top and bottom faces
                    const float ftr = tdiff(az, wt, wv[q + m.Gx * m.Gy]);
                    sFtr[e] = m.all_water ? ftr : mulbf(mulbf(ftr, lm32(m, a.lm, i, it.z, f + 1)), lm32(m, a.lm, i, it.z, f));
                    sPop[e] = a.pop[m.cell_off + q];
                }
            } else if (e < LZ * 32) {
                sFtr[e] = 0.0f;
                sPop[e] = 0;
            }
            sFC[e] = fc;
        }
        if (tid < LZ) {
            const int k = k0 + tid;
            ZLev L = {0.0f, 0.0f, 1.0f, 1.0f, 0.0};
            if (k <= bot) {
                const float dz = a.dzF[m.dz_off + k - 1], volk = __fmul_rn(az, dz);
                L.dtv = __fdiv_rn(a.dT, volk);
                L.sk = __fdiv_rn(a.dT, a.dzC[m.dz_off + k - m.Hz - 1]);
                L.dz = dz;
                L.dzn = a.dzF[m.dz_off + k];
                L.fxv = m.fx_unit / (double)volk;
            }
            sLev[tid] = L;
        }
        __syncthreads();
        if (m.all_water) z_walk_any<LZ, false>(a, m, it, sFC, sFtr, sPop, sLev, ring[threadIdx.y]);
        else z_walk_any<LZ, true>(a, m, it, sFC, sFtr, sPop, sLev, ring[threadIdx.y]);
        __syncthreads();
    }
}

// fill_halo_tracer! (halo_regions.jl:2-62): one thread per line along the axis over all members'
// lines; sources are read before writes. line_off[m] = first line of member m.
template <int AXIS>
__global__ void k32_halo(const MemberDev* __restrict__ md, const long long* __restrict__ line_off, int nm,
                         long long Gtot, float* __restrict__ f, int nfields, const uint32_t* err) {
    if (err && stopped(err)) return;
    const long long nlines = line_off[nm];
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nlines; l += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nm - 1;
        while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (line_off[mid] <= l) lo = mid; else hi = mid - 1; }
        const MemberDev& m = md[lo];
        const long long ll = l - line_off[lo];
        const int na = AXIS == 0 ? m.Gy : m.Gx;
        const int a1 = (int)(ll % na) + 1, b1 = (int)(ll / na) + 1;
        const int N = AXIS == 0 ? m.Nx : AXIS == 1 ? m.Ny : m.Nz;
        const int H = AXIS == 0 ? m.Hx : AXIS == 1 ? m.Hy : m.Hz;
        const int topo = AXIS == 0 ? m.tx : AXIS == 1 ? m.ty : m.tz;
        for (int n = 0; n < nfields; ++n) {
            float* c = f + n * Gtot + m.cell_off;
            auto at = [&](int t) -> float& {
                if (AXIS == 0) return c[gid3(m, t, a1, b1)];
                if (AXIS == 1) return c[gid3(m, a1, t, b1)];
                return c[gid3(m, a1, b1, t)];
            };
            float wv[8], ev[8];
            for (int h = 1; h <= H; ++h) {
                wv[h - 1] = topo == PI_PERIODIC ? at(N + h) : at(H + 1);
                ev[h - 1] = topo == PI_PERIODIC ? at(H + h) : at(N + H);
            }
            for (int h = 1; h <= H; ++h) { at(h) = wv[h - 1]; at(N + H + h) = ev[h - 1]; }
        }
    }
}

// fill_halo_tracer! in one pass when every axis of every member has N >= H: each halo cell then takes
// the value of the interior cell reached by applying the rule of each axis (periodic: ±N; Bounded:
// the nearest interior cell), which is what the three sequential passes above produce. Grid:
// (x blocks, members); every thread walks halo cells of its member, all fields.
__device__ __forceinline__ int halo_src(int a, int N, int H, int topo) {
    if (a > H && a <= N + H) return a;
    if (topo == PI_PERIODIC) return a <= H ? a + N : a - N;
    return a <= H ? H + 1 : N + H;
}
// halo cells of a member: the 2Hz halo levels, then the 2Hy halo rows of the interior levels,
// then the 2Hx halo columns of the interior rows
__global__ void k32_halo_direct(const MemberDev* __restrict__ md, long long Gtot, float* __restrict__ f,
                                int nfields, const uint32_t* err) {
    if (err && stopped(err)) return;
    const MemberDev& m = md[blockIdx.y];
    const int Gx = m.Gx, Gy = m.Gy, Nx = m.Nx, Ny = m.Ny, Nz = m.Nz, Hx = m.Hx, Hy = m.Hy, Hz = m.Hz;
    const int tx = m.tx, ty = m.ty;
    const int nz = 2 * Hz * Gx * Gy, ny = 2 * Nz * Hy * Gx, n = nz + ny + 2 * Nz * Ny * Hx;   // below 2^31
    float* __restrict__ c = f + m.cell_off;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        int i, j, k;
        if (t < nz) {
            const int kk = t / (Gx * Gy), r = t - kk * (Gx * Gy);
            k = kk < Hz ? kk + 1 : Nz + kk + 1;
            j = r / Gx + 1; i = r - (j - 1) * Gx + 1;
        } else if (t < nz + ny) {
            const int u = t - nz, kk = u / (2 * Hy * Gx), r = u - kk * (2 * Hy * Gx), jj = r / Gx;
            k = Hz + 1 + kk;
            j = jj < Hy ? jj + 1 : Ny + jj + 1;
            i = r - jj * Gx + 1;
        } else {
            const int u = t - nz - ny, kk = u / (2 * Hx * Ny), r = u - kk * (2 * Hx * Ny), jj = r / (2 * Hx);
            const int ii = r - jj * 2 * Hx;
            k = Hz + 1 + kk; j = Hy + 1 + jj;
            i = ii < Hx ? ii + 1 : Nx + ii + 1;
        }
        const int q = (i - 1) + Gx * ((j - 1) + Gy * (k - 1));
        const int si = halo_src(i, Nx, Hx, tx), sj = halo_src(j, Ny, Hy, ty), sk = halo_src(k, Nz, Hz, PI_BOUNDED);
        const int src = (si - 1) + Gx * ((sj - 1) + Gy * (sk - 1));
        for (int n2 = 0; n2 < nfields; ++n2) c[n2 * Gtot + q] = c[n2 * Gtot + src];
    }
}

// vel₀ .= vel₁ (time_step.jl:174-176), model.iteration += 1, model.t = iteration·ΔT. After a
// capacity error nothing advances.
__global__ void k32_end_step(int nm, MemberForcing* __restrict__ F, StepState* st, double dT, const uint32_t* err) {
    if (stopped(err)) return;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < nm) {
        for (int c = 0; c < 3; ++c) F[m].vel0[c] = F[m].vel1[c];
    }
    if (m == 0) { st->iteration += 1; st->t = (double)st->iteration * dT; st->call_step += 1; }
}

// After a capacity error the tracers keep their values: the buffer that becomes current is a copy.
__global__ void k32_copy_if_err(float* __restrict__ dst, const float* __restrict__ src, long long n, const uint32_t* err) {
    if (!stopped(err)) return;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = src[q];
}

// ------------------------------------------------------------------------------------------
// uploads, counts, budgets
// ------------------------------------------------------------------------------------------

// Interior array (reference layout, x fastest, Float64 or Float32) into a member's halo-padded
// FP32 field.
template <typename S>
__global__ void k32_scatter_interior(MemberDev m, float* __restrict__ dst, const S* __restrict__ src,
                                     int nx, int ny, int nz) {
    const long long n = (long long)nx * ny * nz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx);
        const long long r = q / nx;
        const int j = (int)(r % ny), k = (int)(r / ny);
        dst[gid3(m, i + 1 + m.Hx, j + 1 + m.Hy, k + 1 + m.Hz)] = (float)src[q];
    }
}

// Velocity halo rule along one axis (halo_regions.jl:64-99) on one member-local field.
template <int AXIS>
__global__ void k32_halo_vel(MemberDev m, float* __restrict__ c, int face_axis) {
    const int na = AXIS == 0 ? m.Gy : m.Gx, nb = AXIS == 2 ? m.Gy : m.Gz;
    const long long nl = (long long)na * nb;
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += (long long)gridDim.x * blockDim.x) {
        const int a1 = (int)(l % na) + 1, b1 = (int)(l / na) + 1;
        const int N = AXIS == 0 ? m.Nx : AXIS == 1 ? m.Ny : m.Nz;
        const int H = AXIS == 0 ? m.Hx : AXIS == 1 ? m.Hy : m.Hz;
        const int topo = AXIS == 0 ? m.tx : AXIS == 1 ? m.ty : m.tz;
        auto at = [&](int t) -> float& {
            if (AXIS == 0) return c[gid3(m, t, a1, b1)];
            if (AXIS == 1) return c[gid3(m, a1, t, b1)];
            return c[gid3(m, a1, b1, t)];
        };
        float wv[8], ev[8];
        const int velrule = (face_axis == AXIS) && topo == PI_BOUNDED;
        for (int h = 1; h <= H; ++h) {
            wv[h - 1] = topo == PI_PERIODIC ? at(N + h) : at(H + 1);
            ev[h - 1] = topo == PI_PERIODIC ? at(H + h) : at(N + H);
        }
        const float face = velrule ? at(N + H + 1) : 0.0f;
        for (int h = 1; h <= H; ++h) at(h) = wv[h - 1];
        if (velrule) { for (int h = N + H + 2; h <= N + 2 * H; ++h) at(h) = face; }
        else { for (int h = 1; h <= H; ++h) at(N + H + h) = ev[h - 1]; }
    }
}

// A setter's new own velocity (vel₁) and/or temperature of a member, bound on the device in
// stream order (after the steps already queued).
__global__ void k32_bind_own(MemberForcing* __restrict__ F, int m, const float* u, const float* v, const float* w,
                             const float* temp) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    MemberForcing& f = F[m];
    if (u) { f.vel1[0] = u; f.vel1[1] = v; f.vel1[2] = w; }
    if (temp) f.temp = temp;
}

template <typename S>
__global__ void k32_to_f32(float* __restrict__ dst, const S* __restrict__ src, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (float)src[q];
}

__global__ void k32_d2f(float* __restrict__ dst, const double* __restrict__ src, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (float)src[q];
}
__global__ void k32_f2d(double* __restrict__ dst, const float* __restrict__ src, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (double)src[q];
}
__global__ void k32_u2d(double* __restrict__ dst, const uint32_t* __restrict__ src, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (double)src[q];
}

// Index of the first non-finite value of a[0, n) (atomicMin into *first, which starts at ~0).
__global__ void k32_first_nonfinite(const float* __restrict__ a, long long n, unsigned long long* first) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        if (!isfinite(a[q])) atomicMin(first, (unsigned long long)q);
}

// First logical slot of a segment whose active individual has a non-finite attribute.
__global__ void k32_first_nonfinite_inds(IndDev32 P, long long base, long long C, unsigned long long* first) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < C; q += (long long)gridDim.x * blockDim.x) {
        const long long g = base + q;
        if (!(P.flags[g] & F32_AC)) continue;
        const float v[10] = { P.ox[g], P.oy[g], P.oz[g], P.Bm[g], P.Cq[g], P.Nq[g], P.Pq[g], P.Chl[g], P.age[g], P.gen[g] };
        bool bad = false;
        for (int k = 0; k < 10; ++k) bad |= !isfinite(v[k]);
        if (bad) atomicMin(first, (unsigned long long)P.lslot[g]);
    }
}

// diags.tracer[name] .+= tracer (time_step.jl:168-172) for the enabled tracers, halos included.
__global__ void k32_diag_tracers(float* __restrict__ d, const float* __restrict__ tr, uint32_t mask, long long Gtot,
                                 const uint32_t* err) {
    if (stopped(err)) return;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < (long long)PI_NTRACERS * Gtot;
         q += (long long)gridDim.x * blockDim.x)
        if (mask >> (q / Gtot) & 1u) d[q] = d[q] + tr[q];
}

// fixed-point sums to Float64 values
__global__ void k32_fx2d(double* __restrict__ dst, const unsigned long long* __restrict__ src, long long n, double unit) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (double)(long long)src[q] * unit;
}

// Active individuals of a slot range (calc_active_individuals, models.jl:157-164).
__global__ void k32_count_active(const uint8_t* __restrict__ flags, long long n, unsigned long long* out) {
    unsigned long long c = 0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        c += (flags[q] & F32_AC) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// FP64 mass budgets of one member: interior Σ c·vol of the C, N and P tracers (DIC+DOC+POC,
// NH4+NO3+DON+PON, PO4+DOP+POP) and the individuals' C, N, P. Block partials (fixed order).
__global__ void k32_budget_cells(MemberDev m, const float* __restrict__ tr, const float* __restrict__ dzF,
                                 long long Gtot, double* __restrict__ partial) {
    __shared__ double sh[3][256];
    double c = 0.0, n = 0.0, p = 0.0;
    const long long V = (long long)m.Nx * m.Ny * m.Nz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < V; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % m.Nx) + 1 + m.Hx;
        const long long r = q / m.Nx;
        const int j = (int)(r % m.Ny) + 1 + m.Hy, k = (int)(r / m.Ny) + 1 + m.Hz;
        const long long cq = m.cell_off + gid3(m, i, j, k);
        const double vol = (double)m.dx * (double)m.dy * (double)dzF[m.dz_off + k - 1];
        c += vol * ((double)tr[PI_DIC * Gtot + cq] + (double)tr[PI_DOC * Gtot + cq] + (double)tr[PI_POC * Gtot + cq]);
        n += vol * ((double)tr[PI_NH4 * Gtot + cq] + (double)tr[PI_NO3 * Gtot + cq] + (double)tr[PI_DON * Gtot + cq] + (double)tr[PI_PON * Gtot + cq]);
        p += vol * ((double)tr[PI_PO4 * Gtot + cq] + (double)tr[PI_DOP * Gtot + cq] + (double)tr[PI_POP * Gtot + cq]);
    }
    sh[0][threadIdx.x] = c; sh[1][threadIdx.x] = n; sh[2][threadIdx.x] = p;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) for (int r = 0; r < 3; ++r) sh[r][threadIdx.x] += sh[r][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) for (int r = 0; r < 3; ++r) partial[blockIdx.x * 3 + r] = sh[r][0];
}

__global__ void k32_budget_inds(MemberDev m, int nsp, const SpeciesDev32* __restrict__ sp, IndDev32 P,
                                double* __restrict__ partial) {
    __shared__ double sh[3][256];
    double c = 0.0, n = 0.0, p = 0.0;
    const long long S = (long long)nsp * m.C;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < S; q += (long long)gridDim.x * blockDim.x) {
        // logical slot order, so the sum does not depend on the storage order
        const long long g = m.slot_off + (q / m.C) * m.C + P.phys[m.slot_off + q];
        if (!(P.flags[g] & F32_AC)) continue;
        const SpeciesDev32& s = sp[q / m.C];
        const double Bm = P.Bm[g];
        c += Bm + (double)P.Cq[g];
        n += Bm * (double)s.R_NC + (double)P.Nq[g];
        p += Bm * (double)s.R_PC + (double)P.Pq[g];
    }
    sh[0][threadIdx.x] = c; sh[1][threadIdx.x] = n; sh[2][threadIdx.x] = p;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) for (int r = 0; r < 3; ++r) sh[r][threadIdx.x] += sh[r][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) for (int r = 0; r < 3; ++r) partial[blockIdx.x * 3 + r] = sh[r][0];
}

// ------------------------------------------------------------------------------------------
// storage order: counting sort of every segment by cell (a periodic pass between steps)
// ------------------------------------------------------------------------------------------

// Sort bin of a stored slot: its interior cell in x-fastest order; an inactive slot goes to one of
// the bins after the cells, one per tile of F32_TILE stored positions (so inactive slots keep
// their relative order and no bin collects a whole segment).
__device__ __forceinline__ long long sort_bin(const MemberDev& m, int s, uint8_t fl, int32_t code, long long slot) {
    const long long V = (long long)m.Nx * m.Ny * m.Nz;
    const long long per = V + (m.wps >> 5);
    long long b;
    if ((fl & F32_AC) && code >= 0) {
        int ci, cj, ck;
        unpack_int(m, code, ci, cj, ck);
        b = min(ci, m.Nx - 1) + (long long)m.Nx * (min(cj, m.Ny - 1) + (long long)m.Ny * min(ck, m.Nz - 1));
    } else {
        b = V + slot / F32_TILE;
    }
    return m.bin_off + (long long)s * per + b;
}

// Warp-aggregated increment of bin counters: lanes with the same bin add once; each lane gets the
// counter value before its own increment (the lanes of a bin take consecutive values). All 32
// lanes call it; lanes with valid = false take no part.
__device__ __forceinline__ unsigned long long bin_claim(unsigned long long* ctr, long long bin, bool valid) {
    const int lane = threadIdx.x & 31;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    const unsigned long long key = valid ? (unsigned long long)bin : ~0ull;
    const unsigned peers = __match_any_sync(0xffffffffu, key) & vmask;
    const int leader = valid ? __ffs(peers) - 1 : lane;
    unsigned long long base = 0;
    if (valid && lane == leader) base = atomicAdd(&ctr[bin], (unsigned long long)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + (unsigned long long)__popc(peers & ((1u << lane) - 1u));
}

// population of every bin (bins zeroed beforehand); blockDim.x divides F32_TILE
__global__ void k32_sort_count(Tab32 T, IndDev32 P, unsigned long long* __restrict__ bins) {
    for (int t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
        const int2 tl = T.tiles[t];
        int mi, s;
        seg_of(T, tl.x, mi, s);
        const MemberDev& m = T.md[mi];
        const long long base = m.slot_off + (long long)s * m.C;
        for (int p = 0; p < F32_TILE / (int)blockDim.x; ++p) {
            const long long slot = (long long)tl.y + p * blockDim.x + threadIdx.x;
            const bool valid = slot < m.C;
            const long long g = base + (valid ? slot : 0);
            const long long bin = valid ? sort_bin(m, s, P.flags[g], P.cell[g], slot) : 0;
            bin_claim(bins, bin, valid);
        }
    }
}

// Moves every slot from P to Q at the next position of its bin (offs: the exclusive scan of the
// bin populations over the whole batch, which starts each segment's bins at the segment's first
// slot) and records where each logical slot went. The order inside a bin is that of the atomics;
// nothing computed from the individuals depends on it.
__global__ void k32_sort_scatter(Tab32 T, IndDev32 P, IndDev32 Q, unsigned long long* __restrict__ offs) {
    for (int t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
        const int2 tl = T.tiles[t];
        int mi, s;
        seg_of(T, tl.x, mi, s);
        const MemberDev& m = T.md[mi];
        const long long base = m.slot_off + (long long)s * m.C;
        for (int p = 0; p < F32_TILE / (int)blockDim.x; ++p) {
            const long long slot = (long long)tl.y + p * blockDim.x + threadIdx.x;
            const bool valid = slot < m.C;
            const long long g = base + (valid ? slot : 0);
            const uint8_t fl = P.flags[g];
            const int32_t code = P.cell[g];
            const long long np = (long long)bin_claim(offs, valid ? sort_bin(m, s, fl, code, slot) : 0, valid);
            if (!valid) continue;
            Q.cell[np] = code; Q.scell[np] = P.scell[g];
            Q.ox[np] = P.ox[g]; Q.oy[np] = P.oy[g]; Q.oz[np] = P.oz[g];
            Q.Bm[np] = P.Bm[g]; Q.Cq[np] = P.Cq[g]; Q.Nq[np] = P.Nq[g]; Q.Pq[np] = P.Pq[g];
            Q.Chl[np] = P.Chl[g]; Q.age[np] = P.age[g]; Q.gen[np] = P.gen[g];
            Q.flags[np] = fl; Q.stat[np] = P.stat[g];
            const int L = P.lslot[g];
            Q.lslot[np] = L;
            P.phys[base + L] = (int)(np - base);
        }
    }
}

// Storage order equal to the logical order over a slot range (after an upload): lslot and phys
// are the identity, relative to the segment's first slot.
__global__ void k32_identity_order(IndDev32 P, long long base, long long C) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < C; q += (long long)gridDim.x * blockDim.x) {
        P.lslot[base + q] = (int)q;
        P.phys[base + q] = (int)q;
    }
}

}  // namespace p32
