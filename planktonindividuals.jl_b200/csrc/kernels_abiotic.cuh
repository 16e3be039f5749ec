// Abiotic particles in the FP64 plain form (src/Individuals/Abiotic/): creation from particle flux
// boundary conditions, the particle step, the interaction with phytoplankton and the release.
//
// The reference's interaction compares every active phytoplankton with every active particle
// (particle_interaction.jl:24-40) and merges through a candidate table written by racing
// threads. Two particles only interact when their find_inds! cells are equal, so here both kinds
// are binned by cell (a stable radix sort keyed by cell, slots ascending inside a cell) and one
// thread walks each cell that holds particles: its particles in ascending slot against the cell's
// phytoplankton in ascending slot. That is the table and the merges a single-threaded run of the
// reference kernels leaves, found in O(particles + phytoplankton + pairs per cell).
#pragma once

#include "kernels_fp64.cuh"

namespace pib {

// 1 where the slot is free (findall(isequal(false), abiotic.ac)).
__global__ void k_abio_free_flags(AbioDev A, long long C, uint32_t* __restrict__ fl) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < C) fl[k] = A.ac[k] ? 0u : 1u;
}

// free slot list in ascending order from the flags and their exclusive prefix
__global__ void k_abio_free_list(const uint32_t* __restrict__ fl, const uint32_t* __restrict__ fr, long long C,
                                 int32_t* __restrict__ freelist) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < C && fl[k]) freelist[fr[k]] = (int32_t)k;
}

// One face of calc_particle_bcs! (particle_interaction.jl:142-229): tr_temp of the face's cells =
// isless(rnd_3d·sz_min·Nsuper, getbc(bc, a, b, iteration)·ΔT·area), area Az on top/bottom, Ax on
// east/west, Ay on north/south. rnd_3d is one draw per cell and step of abiotic species sa.
template <bool LL, int FACE>
__global__ void k_abio_bc_face(DGrid g, FluxBCDev bc, double sz_min, double Nsuper, double dT, uint64_t seed,
                               int64_t iteration, int sa, uint32_t* __restrict__ flag, const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    const int n1 = (FACE == PI_EAST || FACE == PI_WEST) ? g.Ny : g.Nx;
    const int n2 = (FACE == PI_TOP || FACE == PI_BOTTOM) ? g.Ny : g.Nz;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n1 * n2) return;
    const int a = (int)(e % n1) + 1, b = (int)(e / n1) + 1;
    int ii, jj, kk;
    double area;
    if (FACE == PI_TOP || FACE == PI_BOTTOM) {
        ii = a + g.Hx; jj = b + g.Hy; kk = FACE == PI_TOP ? 1 + g.Hz : g.Nz + g.Hz;
        area = Azm<LL>(g, ii, jj);
    } else if (FACE == PI_EAST || FACE == PI_WEST) {
        ii = FACE == PI_EAST ? g.Nx + g.Hx : 1 + g.Hx; jj = a + g.Hy; kk = b + g.Hz;
        area = Axm<LL>(g, ii, jj, kk);
    } else {
        ii = a + g.Hx; jj = FACE == PI_NORTH ? g.Ny + g.Hy : 1 + g.Hy; kk = b + g.Hz;
        area = Aym<LL>(g, ii, jj, kk);
    }
    const int q = gidx(g, ii, jj, kk);
    double r0, r1, r2;
    pi_draw3(seed, (uint32_t)iteration, (uint32_t)sa, PI_DRAW_ABIO_BC, (uint32_t)q, &r0, &r1, &r2);
    flag[q] = (uint32_t)jl_isless(r0 * sz_min * Nsuper, getbc_dev(bc, a, b, iteration) * dT * area);
}

// copy_abiotic_particle_from_field! (particle_interaction.jl:239-250) after the capacity check of
// particles_from_bcs! (:252-271): the n-th flagged cell in column-major order becomes the particle
// of the n-th free slot, at cell − halo − 0.4 computed in Float32 (Int − Float32 is Float32). The
// slot's cell indices are left as they were until find_inds!.
__global__ void k_abio_place(DGrid g, AbioDev A, long long C, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ rank, const uint32_t* __restrict__ fl,
                             const uint32_t* __restrict__ fr, const int32_t* __restrict__ freelist,
                             uint32_t* err, int64_t* err_iter, int64_t iteration) {
    if (*err & PI_DEVERR_CAPACITY) return;
    const long long G = g.G;
    const unsigned long long n = (unsigned long long)rank[G - 1] + flag[G - 1];
    const unsigned long long nfree = (unsigned long long)fr[C - 1] + fl[C - 1];
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n > nfree) {
        if (q == 0) { *err_iter = iteration; __threadfence(); set_err(err, PI_DEVERR_CAPACITY | PI_DEVERR_ABIO); }
        return;
    }
    if (q >= G || !flag[q]) return;
    const int i = (int)(q % g.Gx) + 1, j = (int)((q / g.Gx) % g.Gy) + 1, k = (int)(q / ((long long)g.Gx * g.Gy)) + 1;
    const int32_t d = freelist[rank[q]];
    A.ac[d] = 1;
    A.x[d] = (double)__fsub_rn((float)(i - g.Hx), 0.4f);
    A.y[d] = (double)__fsub_rn((float)(j - g.Hy), 0.4f);
    A.z[d] = (double)__fsub_rn((float)(k - g.Hz), 0.4f);
}

// particle_advection! + particle_diffusion!(κhP, κhP, κvP) + find_inds! of abiotic species sa
// (time_step.jl:29-38), the phytoplankton's particle step with the species' own diffusion draws.
// Inactive slots end at the origin in cell (Hx, Hy, Hz), as every stage multiplies by ac.
template <bool LL>
__global__ void k_abio_move(DGrid g, AbioDev A, long long C, int sa, double dT, uint64_t seed, uint32_t iter,
                            VelPtrs vel, double kappa_h, double kappa_v, uint32_t* err) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= C || (*err & PI_DEVERR_CAPACITY)) return;
    if (!A.ac[k]) {
        int oxi, oyi, ozi;
        unpack_cell(g, A.cell[k], oxi, oyi, ozi);
        clamp_idx((long long)ozi + g.Hz, 1, g.Gz, err);
        if (A.x[k] != 0.0) A.x[k] = 0.0;
        if (A.y[k] != 0.0) A.y[k] = 0.0;
        if (A.z[k] != 0.0) A.z[k] = 0.0;
        A.cell[k] = pack_cell(g, g.Hx, g.Hy, g.Hz);
        return;
    }
    particle_step<LL, false>(g, A, (uint32_t)sa, PI_DRAW_ABIO_DIFFUSION, k, 0, dT, seed, iter, vel, kappa_h, kappa_v,
                             nullptr, nullptr, err);
}

// sort keys of the active particles: their find_inds! cell (G when inactive), value the slot
__global__ void k_abio_keys(DGrid g, AbioDev A, long long C, uint32_t* __restrict__ key, uint32_t* __restrict__ val,
                            const uint32_t* err) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= C) return;
    uint32_t c = (uint32_t)g.G;
    if (!(*err & PI_DEVERR_CAPACITY) && A.ac[k]) {
        int xi, yi, zi;
        unpack_cell(g, A.cell[k], xi, yi, zi);
        c = (uint32_t)gidx(g, xi, yi, zi);
    }
    key[k] = c;
    val[k] = (uint32_t)k;
}

__device__ __forceinline__ long long lower_bound_u32(const uint32_t* __restrict__ a, long long n, uint32_t v) {
    long long lo = 0, hi = n;
    while (lo < hi) { const long long mid = (lo + hi) >> 1; if (a[mid] < v) lo = mid + 1; else hi = mid; }
    return lo;
}

// calc_distance (particle_interaction.jl:3-15) for two particles of the same cell (xi, yi, zi):
// ΔxF, ΔyF, ΔzF at that cell; dx^2.0f0 is Julia's integer power of a Float64.
template <bool LL>
__device__ __forceinline__ double cell_distance(const DGrid& g, int xi, int yi, int zi, double x1, double y1, double z1,
                                                double x2, double y2, double z2) {
    const double dx = (x1 - x2) * dxFm<LL>(g, xi, yi);
    const double dy = (y1 - y2) * dyFm<LL>(g, xi, yi);
    const double dz = (z1 - z2) * dzF1(g, zi);
    return sqrt(pi_pow_int(dx, 2) + pi_pow_int(dy, 2) + pi_pow_int(dz, 2));
}

// particle_interaction! (particle_interaction.jl:75-81) for one (phytoplankton, abiotic) pair. One
// thread per cell holding active particles (the first entry of its run in the sorted keys): for
// each of its particles k in ascending slot, the candidate row intac[k, ·] is rebuilt —
// entry (i % max_candidates) holds the largest 1-based phytoplankton slot i of the cell within Rd
// (calc_interaction_kernel!, :24-40) — and the particle merges into its first candidate whose ptc
// is below max_ptc (merge_particle_kernel!, :50-66). A phytoplankton is a candidate only of
// particles of its own cell, so each ptc is read and written by one thread, in the order of a
// single-threaded run.
template <bool LL>
__global__ void k_interact(DGrid g, SpcDev P, AbioDev A, long long C, const uint32_t* __restrict__ pkey,
                           const uint32_t* __restrict__ pval, const uint32_t* __restrict__ akey,
                           const uint32_t* __restrict__ aval, double Rd, int maxc, double max_ptc,
                           int32_t* __restrict__ intac, uint32_t* err, int64_t* err_iter, int64_t iteration) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= C || (*err & PI_DEVERR_CAPACITY)) return;
    const uint32_t c = akey[p];
    if (c >= (uint32_t)g.G || (p > 0 && akey[p - 1] == c)) return;
    const long long lo = lower_bound_u32(pkey, C, c), hi = lower_bound_u32(pkey, C, c + 1);
    int xi, yi, zi;
    {
        const long long q = c;
        xi = (int)(q % g.Gx) + 1; yi = (int)((q / g.Gx) % g.Gy) + 1; zi = (int)(q / ((long long)g.Gx * g.Gy)) + 1;
    }
    for (long long e = p; e < C && akey[e] == c; ++e) {
        const long long k = aval[e];
        int32_t* row = intac + k * (long long)maxc;
        for (int j = 0; j < maxc; ++j) row[j] = 0;
        const double ax = A.x[k], ay = A.y[k], az = A.z[k];
        for (long long f = lo; f < hi; ++f) {
            const long long i = pval[f];
            if (cell_distance<LL>(g, xi, yi, zi, P.x[i], P.y[i], P.z[i], ax, ay, az) < Rd)
                row[(i + 1) % maxc] = (int32_t)(i + 1);
        }
        for (int j = 0; j < maxc; ++j) {
            const int32_t pid = row[j];
            if (pid <= 0) continue;
            if (max_ptc != max_ptc) {     // the species' parameters have no max_ptc
                *err_iter = iteration;
                __threadfence();
                set_err(err, PI_DEVERR_CAPACITY | PI_DEVERR_MAXPTC);
                return;
            }
            if (P.ptc[pid - 1] < max_ptc) { P.ptc[pid - 1] += 1.0; A.ac[k] = 0; break; }
        }
    }
}

// get_release_probability! (particle_interaction.jl:85-91): an active phytoplankton releases a
// particle when rnd.x < release_P·ΔT·ptc; flag64 = (release << 32) | (slot is a free particle slot),
// the layout k_lists turns into the releaser and free-slot lists.
__global__ void k_release_flags(SpcDev P, AbioDev A, long long C, double release_P, double dT, uint64_t seed,
                                uint32_t iter, int pair, unsigned long long* __restrict__ flag64, const uint32_t* err) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C || (*err & PI_DEVERR_CAPACITY)) return;
    double r0, r1, r2;
    pi_draw3(seed, iter, (uint32_t)pair, PI_DRAW_RELEASE, (uint32_t)i, &r0, &r1, &r2);
    const unsigned long long rel = (jl_isless(r0, release_P * dT * P.ptc[i]) && (P.flags[i] & FL_AC)) ? 1ull : 0ull;
    flag64[i] = (rel << 32) | (A.ac[i] ? 0ull : 1ull);
}

// release_abiotic_particle_kernel! (particle_interaction.jl:93-101): the n-th releaser fills the
// n-th free particle slot at its own position plus (rnd.x, rnd.y, rnd.z) — the release draw and
// the mortality and division draws of the last species' get_probability!, which rnd.y and rnd.z
// still hold — and its ptc drops by one. The slot's cell indices wait for find_inds!.
__global__ void k_release(SpcDev P, AbioDev A, const int32_t* __restrict__ rellist,
                          const int32_t* __restrict__ freelist, const uint32_t* nrel, uint64_t seed, uint32_t iter,
                          int pair, int last_species, const uint32_t* err) {
    if (*err & PI_DEVERR_CAPACITY) return;
    const uint32_t n = *nrel;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int32_t i = rellist[e], d = freelist[e];
        double r0, r1, r2, q0, q1, q2;
        pi_draw3(seed, iter, (uint32_t)pair, PI_DRAW_RELEASE, (uint32_t)i, &r0, &r1, &r2);
        pi_draw3(seed, iter, (uint32_t)last_species, PI_DRAW_DECISION, (uint32_t)i, &q0, &q1, &q2);
        A.ac[d] = 1;
        A.x[d] = P.x[i] + r0;
        A.y[d] = P.y[i] + q1;
        A.z[d] = P.z[i] + q2;
        P.ptc[i] = P.ptc[i] - 1.0;
    }
}

// diags.abiotics[sa].num (time_step.jl:151-158): one per active particle at its stored cell; the
// sums are whole numbers, exact in any order.
__global__ void k_abio_num(DGrid g, AbioDev A, long long C, double* __restrict__ d, const uint32_t* err) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= C || (*err & PI_DEVERR_CAPACITY) || !A.ac[k]) return;
    int xi, yi, zi;
    unpack_cell(g, A.cell[k], xi, yi, zi);
    atomicAdd(&d[gidx(g, xi, yi, zi)], 1.0);
}

}  // namespace pib
