// FP32 form: the whole tracer update (tracer_update.jl:22-43 without diffusion and flux boundary
// conditions) in one kernel, k32_tracer.
//
// A block owns a tile of 31 × 8 columns and a run of levels of one member, for one group of seven
// tracers, and walks down the levels. At each level L it
//   1. receives the level's tracers (tile plus two columns and two rows on each side) in shared
//      memory, staged two levels ahead by TMA tensor copies (cp.async.bulk.tensor, one box of
//      40 columns × 12 rows per tracer) or, for grids whose row pitch is not a multiple of 16
//      bytes, by per-thread cp.async copies that signal the same mbarrier;
//   2. runs the DST3FL x sweep on the 12 staged rows and the y sweep on the 8 tile rows
//      (multi_dim_adv.jl:1-135): tracer_temp of level L stays in registers;
//   3. finishes cell L-2 of its column: the z sweep from a 4-level register window of tracer_temp,
//      then sinking, forcing, particle sums and apply_tendency!, and writes the result into the
//      cell and into the halo cells the halo rule copies it to (fill_halo_tracer!).
// tracer_temp never goes to memory: per cell the kernel reads the tracers once (plus halo re-reads
// that hit L2), the velocities, the particle sums of occupied cells, and writes the result.
//
// The x sweep of the two rows on each side of the tile runs on the staged halo rows of the tracer,
// which equal the rows the halo rule maps them to once the tracer's halos are filled (every step
// ends with fill_halo_tracer!). The first step after a tracer upload runs the two-kernel path
// (k32_xy + k32_ztail + halo fill), which maps those rows explicitly. Every formula is evaluated
// as in those kernels, so both paths produce the same bits.
#pragma once

#include "kernels_fp32.cuh"

namespace p32 {

#define TRK_TY 8                  // tile rows (one warp each)
#define TRK_TX 31                 // tile columns finished per block (32 x faces)
#define TRK_R (TRK_TY + 4)        // staged rows
#define TRK_W 40                  // staged columns per row (TMA box width, 160 bytes)
#define TRK_NB 3                  // level buffers of the staging ring
#define TRK_NG 7                  // tracers per group
#define TRK_THREADS (32 * TRK_TY)
#define TRK_MAXLEV 66             // per-level constants held: up to 64 levels per block + 2

// The two tracer groups: every forcing partner of a tracer is in its group, except POC for the
// iron tracers of group 1, which is read as an extra value.
__host__ __device__ constexpr int trk_tracer(int grp, int q) {
    return grp == 0 ? (q == 0 ? PI_DIC : q == 1 ? PI_NH4 : q == 2 ? PI_NO3 : q == 3 ? PI_DOC
                                       : q == 4 ? PI_DON : q == 5 ? PI_POC : PI_PON)
                    : (q == 0 ? PI_PO4 : q == 1 ? PI_DFe : q == 2 ? PI_DOP : q == 3 ? PI_PFe_inorg
                                       : q == 4 ? PI_POP : q == 5 ? PI_PFe_bio : PI_Dust);
}
// position in the group of tracer n (or -1)
__host__ __device__ constexpr int trk_slot(int grp, int n) {
    for (int q = 0; q < TRK_NG; ++q) if (trk_tracer(grp, q) == n) return q;
    return -1;
}

inline size_t tracer_smem_bytes() {
    return (size_t)TRK_NB * TRK_NG * TRK_R * TRK_W * sizeof(float)      // staging ring
         + (size_t)TRK_R * TRK_NG * 32 * sizeof(float)                  // x-swept rows
         + (size_t)(TRK_TY + 1) * TRK_NG * 32 * sizeof(float)           // y face fluxes
         + (size_t)TRK_MAXLEV * sizeof(ZLev)                            // per-level constants
         + (size_t)TRK_NB * sizeof(unsigned long long);                 // mbarriers
}

// ---- mbarrier and bulk-copy primitives (inline PTX) ---------------------------------------
__device__ __forceinline__ void mbar_init(unsigned addr, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(addr), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned addr, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" :: "r"(addr), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned addr, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(addr), "r"(parity) : "memory");
    return ok != 0;
}
// the cp.async copies this thread issued arrive on the mbarrier when they complete
__device__ __forceinline__ void cpa_mbar_arrive(unsigned addr) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" :: "r"(addr) : "memory");
}
// 4 bytes, or zeros without reading when `on` is false
__device__ __forceinline__ void cpa4z(unsigned sdst, const float* gsrc, bool on) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" :: "r"(sdst), "l"(gsrc), "r"(on ? 4 : 0) : "memory");
}
// One box of a 4-D tensor map (x, y, z, tracer) into shared memory, completing on an mbarrier.
__device__ __forceinline__ void tma_load_4d(unsigned sdst, const void* map, int x, int y, int z, int t, unsigned mbar) {
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                 :: "r"(sdst), "l"(map), "r"(x), "r"(y), "r"(z), "r"(t), "r"(mbar) : "memory");
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
    return t;
}
// Bounded wait on an mbarrier phase (one second at most by default); false when it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned addr, unsigned parity, unsigned long long limit_ns = 1000000000ull) {
    if (mbar_try_wait(addr, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    do {
        if (mbar_try_wait(addr, parity)) return true;
    } while (globaltimer_ns() - t0 < limit_ns);
    return false;
}

// Self-test of the bounded wait: one thread waits on an mbarrier that nothing arrives on, with the
// given limit, and records whether it gave up (1) and how long it waited.
__global__ void k32_wait_selftest(unsigned long long limit_ns, int* gave_up, unsigned long long* waited_ns) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const unsigned a = (unsigned)__cvta_generic_to_shared(&bar);
    mbar_init(a, 1u);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    const unsigned long long t0 = globaltimer_ns();
    const bool ok = mbar_wait(a, 0u, limit_ns);
    *waited_ns = globaltimer_ns() - t0;
    *gave_up = ok ? 0 : 1;
}

// The cells an interior cell a (1-based, along one axis of N >= H cells with H halo points) stands
// for after the halo fill: itself (t = 0), then its periodic images in the halo, or the halo points
// a Bounded edge cell is copied to.
__device__ __forceinline__ int halo_count(int a, int N, int H, int topo) {
    if (topo == PI_PERIODIC) return 1 + (a - H <= H ? 1 : 0) + (a - H > N - H ? 1 : 0);
    return 1 + (a == H + 1 ? H : 0) + (a == N + H ? H : 0);
}
__device__ __forceinline__ int halo_image(int a, int N, int H, int topo, int t) {
    if (t == 0) return a;
    if (topo == PI_PERIODIC) return (t == 1 && a - H <= H) ? a + N : a - N;
    if (a == H + 1 && t <= H) return t;
    return N + H + t - (a == H + 1 ? H : 0);
}

struct TrkArgs {
    TrArgs a;
    const unsigned char* maps;   // CUtensorMap (128 bytes) per member for the current tracer buffer
    int lz;                      // levels finished per block (at most 64)
};

// Stages level L (1-based) of the block's tracers into ring buffer `buf`.
__device__ __forceinline__ void trk_issue(const TrkArgs& A, const MemberDev& md, const void* map, bool tma, int grp,
                                          float* ring, unsigned mbar0, int L, int buf, int x0, int y0) {
    float* dst = ring + (size_t)buf * TRK_NG * TRK_R * TRK_W;
    const unsigned sdst = (unsigned)__cvta_generic_to_shared(dst);
    const unsigned mbar = mbar0 + 8u * buf;
    if (tma) {
        if (threadIdx.x == 0) {
            // the buffer's earlier contents were read through the generic proxy
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            mbar_expect_tx(mbar, TRK_NG * TRK_R * TRK_W * 4);
#pragma unroll
            for (int q = 0; q < TRK_NG; ++q)
                tma_load_4d(sdst + q * (TRK_R * TRK_W * 4), map, x0, y0, L - 1, trk_tracer(grp, q), mbar);
        }
        return;
    }
    // per-thread copies of the same boxes; outside the grid: zeros, as the tensor copy fills them
    const float* src = A.a.tr + md.cell_off;
    const long long G = A.a.Gtot;
    const long long lev = (long long)(L - 1) * md.Gx * md.Gy;
    for (int e = threadIdx.x; e < TRK_NG * TRK_R * TRK_W; e += TRK_THREADS) {
        const int q = e / (TRK_R * TRK_W), r = (e / TRK_W) % TRK_R, c = e % TRK_W;
        const int x = x0 + c, y = y0 + r;
        const bool in = x < md.Gx && y < md.Gy;
        const float* p = src + (long long)trk_tracer(grp, q) * G + lev + (in ? (long long)y * md.Gx + x : 0);
        cpa4z(sdst + 4u * e, p, in);
    }
    cpa_mbar_arrive(mbar);
}

template <int GRP, bool LM>
__device__ __forceinline__ void trk_body(const TrkArgs& A, const MemberDev& md, const int4 it, unsigned char* smem) {
    const TrArgs& a = A.a;
    float* ring = reinterpret_cast<float*>(smem);
    float* TA = ring + TRK_NB * TRK_NG * TRK_R * TRK_W;         // [row][tracer][lane]
    float* FY = TA + TRK_R * TRK_NG * 32;                        // [face][tracer][lane]
    ZLev* sLev = reinterpret_cast<ZLev*>(FY + (TRK_TY + 1) * TRK_NG * 32);
    unsigned long long* mbar = reinterpret_cast<unsigned long long*>(sLev + TRK_MAXLEV);
    const unsigned mbar0 = (unsigned)__cvta_generic_to_shared(mbar);

    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int Nx = md.Nx, Ny = md.Ny, Hx = md.Hx, Hy = md.Hy, Hz = md.Hz, Gx = md.Gx, Gy = md.Gy;
    const int top = Hz + 1, bot = md.Nz + Hz;
    const int i0 = it.y, j0 = it.z, k0 = it.w;
    const int k1 = min(k0 + A.lz - 1, bot);
    const int Ls = max(top, k0 - 2), Le = min(bot, k1 + 2);
    const int x0 = (i0 - 3) & ~3, xo = i0 - 3 - x0, y0 = j0 - 3;
    const long long G = a.Gtot, off = md.cell_off;
    const int slab = Gx * Gy;
    const float dT = a.dT;
    const float dx = md.dx, dy = md.dy, az = __fmul_rn(dx, dy);
    const bool tma = A.maps != nullptr && (Gx & 3) == 0;
    const void* map = tma ? (const void*)(A.maps + 128 * it.x) : nullptr;
    const MemberForcing& F = a.F[it.x];
    const float* __restrict__ uu = F.vel1[0];
    const float* __restrict__ vv = F.vel1[1];
    const float* __restrict__ ww = F.vel1[2];
    const uint8_t* __restrict__ lmm = a.lm + off;
    auto lmq = [&](int i, int j, int k) -> int { return LM ? (int)lmm[gid3(md, i, j, k)] : 1; };
    const BgcDev32& bg = a.bgc[it.x];

    if (threadIdx.x == 0)
        for (int b = 0; b < TRK_NB; ++b) mbar_init(mbar0 + 8u * b, tma ? 1u : (unsigned)TRK_THREADS);
    // per-level constants of the levels this block finishes (as k32_ztail forms them)
    for (int e = threadIdx.x; e <= k1 - Ls; e += TRK_THREADS) {
        const int k = Ls + e;
        ZLev Lv;
        const float dz = a.dzF[md.dz_off + k - 1], volk = __fmul_rn(az, dz);
        Lv.dtv = __fdiv_rn(a.dT, volk);
        Lv.sk = __fdiv_rn(a.dT, a.dzC[md.dz_off + k - Hz - 1]);
        Lv.dz = dz;
        Lv.dzn = a.dzF[md.dz_off + k];
        Lv.fxv = md.fx_unit / (double)volk;
        sLev[e] = Lv;
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    __syncthreads();
    for (int p = 0; p < TRK_NB && Ls + p <= Le; ++p) trk_issue(A, md, map, tma, GRP, ring, mbar0, Ls + p, p, x0, y0);

    // the thread's column (lanes 0..30 finish one each) and row
    const int i = i0 + lane, j = j0 + wid;
    const bool col = lane < TRK_TX && i <= Nx + Hx;
    const bool own = col && j <= Ny + Hy;
    const int ic = min(i, Gx);
    const FeCoef fc_fe = fe_coef(bg, dT);
    const float wso = bg.w_sink_org, wsi = bg.w_sink_inorg;

    float tw[TRK_NG][4];        // tracer_temp at levels L-3 .. L of the column
    float Ft[TRK_NG];           // z flux of the face above the current cell
    float ccp[TRK_NG];          // the tracer at the previous level (sinking)
    int mm0 = 1, mm1 = 1, mm2 = 1, mm3 = 1;
#pragma unroll
    for (int q = 0; q < TRK_NG; ++q) { Ft[q] = 0.0f; ccp[q] = 0.0f; tw[q][0] = tw[q][1] = tw[q][2] = tw[q][3] = 0.0f; }
    if (LM && own) {
        // land mask window [L-3, L-2, L-1, L] after the shift of iteration Ls
        mm1 = Ls - 3 >= 1 ? lmq(i, j, Ls - 3) : 1;
        mm2 = lmq(i, j, Ls - 2);
        mm3 = lmq(i, j, Ls - 1);
    }
    float wprev = 0.0f;          // w at the face above the current cell
    int pop_next = 0;
    bool ok = true;
    int waited = Ls - 1;         // last level whose staging this thread has waited for
    int issued = min(Le, Ls + TRK_NB - 1);

    for (int L = Ls; L <= k1 + 2; ++L) {
        const bool xy = L <= Le;
        const int k = L - 2;                          // the cell finished in this iteration
        const bool fin = own && k >= k0 && k <= k1;
        // loads for the end of the iteration: the tracers at cell k (and POC for the iron tracers)
        float cc[TRK_NG], poc = 0.0f;
        unsigned long long accv[TRK_NG];
        const int qk = (ic - 1) + Gx * ((min(j, Gy) - 1) + Gy * (max(k, 1) - 1));
        const bool kvalid = own && k >= top;
#pragma unroll
        for (int q = 0; q < TRK_NG; ++q) {
            cc[q] = kvalid ? a.tr[(long long)trk_tracer(GRP, q) * G + off + qk] : 0.0f;
            accv[q] = 0ull;
            const int as = acc_slot(trk_tracer(GRP, q));
            if (as >= 0 && fin && pop_next > 0) accv[q] = a.acc[(long long)as * G + off + qk];
        }
        if (GRP == 1 && kvalid) poc = a.tr[(long long)PI_POC * G + off + qk];
        const float wf = (own && L - 1 <= bot + 1 && L - 1 >= top) ? ww[qk + slab] : 0.0f;   // w at face L-1
        const int pop_cur = pop_next;
        pop_next = (own && k + 1 >= top && k + 1 <= bot) ? a.pop[off + qk + slab] : 0;

        // level L-1 done: its buffer, TA and FY are free; a wait that gave up stops the block
        if (__syncthreads_or(!ok)) break;
        if (L > Ls && L - 1 + TRK_NB <= Le) {
            trk_issue(A, md, map, tma, GRP, ring, mbar0, L - 1 + TRK_NB, (L - 1 - Ls) % TRK_NB, x0, y0);
            issued = L - 1 + TRK_NB;
        }
        float tbn[TRK_NG];
        if (xy) {
            const int b = (L - Ls) % TRK_NB;
            if (!mbar_wait(mbar0 + 8u * b, (unsigned)(((L - Ls) / TRK_NB) & 1))) ok = false;
            waited = L;
            const float* R = ring + (size_t)b * TRK_NG * TRK_R * TRK_W;
            const float dz = a.dzF[md.dz_off + L - 1];
            const float dtv = __fdiv_rn(dT, __fmul_rn(az, dz));
            // ---- x sweep of rows wid and wid + 8 (rows j0-2 .. j0+9)
            const float ax = __fmul_rn(dy, dz);
            for (int r = wid; r < TRK_R; r += TRK_TY) {
                const int jj = wrap_ax(j0 - 2 + r, Ny, Hy, md.ty);
                const float uw = uu[gid3(md, ic, jj, L)];
                const float ue = __shfl_down_sync(0xffffffffu, uw, 1);
                const FCu fc = fcu(uw, ax, __frcp_rn(dx), dT);
                int l0 = 1, lm1 = 1, lm2 = 1, lp1 = 1;
                if (LM) {
                    l0 = lmq(ic, jj, L); lm1 = lmq(max(i - 1, 1), jj, L); lm2 = lmq(max(i - 2, 1), jj, L);
                    lp1 = lmq(min(i + 1, Gx), jj, L);
                }
                const bool east_zero = i == Nx + Hx && md.tx != PI_PERIODIC;
                const float ftr = mk<LM>(tdiff(ax, ue, uw), lp1, l0);
#pragma unroll
                for (int q = 0; q < TRK_NG; ++q) {
                    const float* cr = R + (q * TRK_R + r) * TRK_W + xo + lane;
                    const float cm2 = cr[0], cm1 = cr[1], v = cr[2], cp1 = cr[3];
                    const float Fw = flux_h<LM>(fc, cm2, cm1, v, cp1, lm2, lm1, l0, lp1);
                    float Fe = __shfl_down_sync(0xffffffffu, Fw, 1);
                    if (east_zero) Fe = 0.0f;
                    TA[(r * TRK_NG + q) * 32 + lane] = upd_sweep(v, dtv, mk<LM>(__fsub_rn(Fe, Fw), lp1, l0), v, ftr);
                }
            }
            __syncthreads();
            // ---- y faces j0 + f, f = 0 .. 8 (warp w: face w + 1; warp 0 also face 0)
            const float ay = __fmul_rn(dx, dz);
            for (int f = (wid == 0 ? 0 : wid + 1); f <= wid + 1; ++f) {
                const int fj = j0 + f;
                const bool special = fj == Ny + Hy + 1;
                const bool zero = !col || fj > Ny + Hy + 1 || (special && md.ty != PI_PERIODIC);
                const int fs = special ? Hy + 1 : min(fj, Ny + Hy);
                const FCu fc = fcu(zero ? 0.0f : vv[gid3(md, ic, fs, L)], ay, __frcp_rn(dy), dT);
                int L2 = 1, L1 = 1, L0 = 1, Lp = 1;
                if (LM) { L2 = lmq(ic, fs - 2, L); L1 = lmq(ic, fs - 1, L); L0 = lmq(ic, fs, L); Lp = lmq(ic, fs + 1, L); }
#pragma unroll
                for (int q = 0; q < TRK_NG; ++q)
                    FY[(f * TRK_NG + q) * 32 + lane] =
                        zero ? 0.0f : flux_h<LM>(fc, TA[(f * TRK_NG + q) * 32 + lane], TA[((f + 1) * TRK_NG + q) * 32 + lane],
                                                 TA[((f + 2) * TRK_NG + q) * 32 + lane], TA[((f + 3) * TRK_NG + q) * 32 + lane],
                                                 L2, L1, L0, Lp);
            }
            __syncthreads();
            // ---- y update of row j0 + wid: tracer_temp of level L
            if (own) {
                const int qq = gid3(md, i, j, L);
                const int c0m = LM ? lmq(i, j, L) : 1, cpm = LM ? lmq(i, j + 1, L) : 1;
                const float ftr = mk<LM>(tdiff(ay, vv[qq + Gx], vv[qq]), cpm, c0m);
#pragma unroll
                for (int q = 0; q < TRK_NG; ++q) {
                    const float dG = mk<LM>(__fsub_rn(FY[((wid + 1) * TRK_NG + q) * 32 + lane], FY[(wid * TRK_NG + q) * 32 + lane]), cpm, c0m);
                    const float trs = R[(q * TRK_R + wid + 2) * TRK_W + xo + lane + 2];
                    tbn[q] = upd_sweep(TA[((wid + 2) * TRK_NG + q) * 32 + lane], dtv, dG, trs, ftr);
                }
            }
        }
        if (!own) continue;
        // ---- window: tracer_temp at L-3 .. L (clamped below the bottom and above the top)
#pragma unroll
        for (int q = 0; q < TRK_NG; ++q) {
            const float tn = xy ? tbn[q] : tw[q][3];
            if (L == top) { tw[q][0] = tw[q][1] = tw[q][2] = tw[q][3] = tn; }
            else { tw[q][0] = tw[q][1]; tw[q][1] = tw[q][2]; tw[q][2] = tw[q][3]; tw[q][3] = tn; }
        }
        if (LM) { mm0 = mm1; mm1 = mm2; mm2 = mm3; mm3 = lmq(i, j, L); }
        // z flux of face L-1 (zero below the bottom)
        FCu fz;
        fz.tr = 0.0f; fz.d0c = 0.0f; fz.d1c = 0.0f; fz.R = 0.0f;
        if (L - 1 <= bot && L - 1 >= top) fz = fcu(wf, az, a.rdzC[md.dz_off + L - 2], dT);
        float Fb[TRK_NG];
#pragma unroll
        for (int q = 0; q < TRK_NG; ++q) Fb[q] = flux_v<LM>(fz, tw[q][0], tw[q][1], tw[q][2], tw[q][3], mm0, mm1, mm2, mm3);
        if (fin) {
            const ZLev Z = sLev[k - Ls];
            const int l1 = mm1, l0 = mm2;                       // land mask of cell k and k+1
            const float ftr = LM ? mulbf(mulbf(tdiff(az, wprev, wf), mm2), mm1) : tdiff(az, wprev, wf);
            const float dfe = GRP == 1 ? fmaxf(0.0f, cc[trk_slot(1, PI_DFe)]) : 0.0f;
            const long long qo = off + qk;
            const int nix = halo_count(i, Nx, Hx, md.tx), njy = halo_count(j, Ny, Hy, md.ty);
            const int nkz = halo_count(k, md.Nz, Hz, PI_BOUNDED);
#pragma unroll
            for (int q = 0; q < TRK_NG; ++q) {
                const int n = trk_tracer(GRP, q);
                float Gc = __fsub_rn(upd_sweep(tw[q][1], Z.dtv, mk<LM>(__fsub_rn(Ft[q], Fb[q]), l0, l1), cc[q], ftr), cc[q]);
                const int as = acc_slot(n);
                if (as >= 0) {
                    // tracer_forcing! on max(0, tracer): aS·T(n) + aO·T(partner), the partner in the
                    // group (k32_ztail's coefficients)
                    float aS = 0.0f, aO = 0.0f;
                    int po = -1;
                    switch (n) {
                        case PI_DIC: po = trk_slot(GRP, PI_DOC); aO = bg.kDOC * dT; break;
                        case PI_DOC: aS = -bg.kDOC * dT; po = trk_slot(GRP, PI_POC); aO = bg.kPOC * dT; break;
                        case PI_POC: aS = -bg.kPOC * dT; break;
                        case PI_NH4: aS = -bg.Nit * dT; po = trk_slot(GRP, PI_DON); aO = bg.kDON * dT; break;
                        case PI_NO3: po = trk_slot(GRP, PI_NH4); aO = bg.Nit * dT; break;
                        case PI_DON: aS = -bg.kDON * dT; po = trk_slot(GRP, PI_PON); aO = bg.kPON * dT; break;
                        case PI_PON: aS = -bg.kPON * dT; break;
                        case PI_PO4: po = trk_slot(GRP, PI_DOP); aO = bg.kDOP * dT; break;
                        case PI_DOP: aS = -bg.kDOP * dT; po = trk_slot(GRP, PI_POP); aO = bg.kPOP * dT; break;
                        case PI_POP: aS = -bg.kPOP * dT; break;
                        default: break;
                    }
                    Gc = add_forcing(Gc, aS, cc[q], aO, po >= 0 ? cc[po] : 0.0f);
                } else {
                    // tracer_sinking! and the iron forcing
                    if (n != PI_DFe) {
                        const float ws = n == PI_PFe_bio ? wso : wsi;
                        const float fup = (k - 1 <= Hz) ? 0.0f : __fmul_rn(ws, ccp[q]);
                        const float fdn = (k >= bot) ? 0.0f : __fmul_rn(ws, cc[q]);
                        Gc = add_sinking(Gc, fup, fdn, Z.sk);
                    }
                    if (n != PI_Dust) {
                        const float pfi = fmaxf(0.0f, cc[trk_slot(1, PI_PFe_inorg)]);
                        const float pfb = fmaxf(0.0f, cc[trk_slot(1, PI_PFe_bio)]);
                        const float dst = fmaxf(0.0f, cc[trk_slot(1, PI_Dust)]);
                        Gc += fe_forcing(n, fc_fe, dfe, fmaxf(0.0f, poc), dst, pfb, pfi);
                    }
                }
                float plk = 0.0f;
                if (as >= 0 && pop_cur > 0) {
                    const long long vvv = (long long)accv[q];
                    if (vvv) { a.acc[(long long)as * G + qo] = 0ull; plk = (float)((double)vvv * Z.fxv); }
                }
                a.tr_next[(long long)n * G + qo] = tendency(cc[q], Gc, plk);
            }
            if (nix * njy * nkz > 1) {
                // a cell on the edge of the domain: copy its new values into its halo images
#pragma unroll 1
                for (int q = 0; q < TRK_NG; ++q) {
                    float* dst = a.tr_next + (long long)trk_tracer(GRP, q) * G + off;
                    const float outv = dst[qk];
                    for (int c = 0; c < nkz; ++c)
                        for (int bq = 0; bq < njy; ++bq)
                            for (int aq = 0; aq < nix; ++aq)
                                if (aq | bq | c)
                                    dst[gid3(md, halo_image(i, Nx, Hx, md.tx, aq), halo_image(j, Ny, Hy, md.ty, bq),
                                             halo_image(k, md.Nz, Hz, PI_BOUNDED, c))] = outv;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < TRK_NG; ++q) { Ft[q] = Fb[q]; ccp[q] = cc[q]; }
        wprev = wf;
    }
    if (!ok) {
        // wait (bounded) for the copies still in flight into this block's shared memory
        for (int L = waited + 1; L <= issued; ++L) mbar_wait(mbar0 + 8u * ((L - Ls) % TRK_NB), (unsigned)(((L - Ls) / TRK_NB) & 1));
        seterr(const_cast<uint32_t*>(a.err), F32_ERR_TIMEOUT);
    }
}

// Grid: (items, 2 tracer groups). Items {member, i0, j0, k0}: tiles of 31 × 8 columns and runs of
// `lz` levels.
__global__ void __launch_bounds__(TRK_THREADS, 2) k32_tracer(TrkArgs A) {
    if (stopped(A.a.err)) return;
    extern __shared__ __align__(128) unsigned char tsm[];
    const int4 it = A.a.items[blockIdx.x];
    const MemberDev& md = A.a.T.md[it.x];
    if (blockIdx.y == 0) {
        if (md.all_water) trk_body<0, false>(A, md, it, tsm); else trk_body<0, true>(A, md, it, tsm);
    } else {
        if (md.all_water) trk_body<1, false>(A, md, it, tsm); else trk_body<1, true>(A, md, it, tsm);
    }
}

}  // namespace p32
