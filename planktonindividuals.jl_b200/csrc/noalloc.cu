// pi_tracer_advection_noalloc — DST3FL advection of one tracer field with no device allocation.
//
// Some callers cannot allocate device memory: a host runtime that owns every device allocation
// through its own pool or garbage collector (a Julia or Python array library embedding this
// step), or a time-critical loop whose policy forbids allocation after start-up. They pass their
// own device buffers for the inputs and the output; the two intermediate fields of the
// dimensionally split sweeps live in the fixed-size device array below, which every GPU that
// loads this library holds until the process exits.
//
// Limits and sharing rules:
//  - at most PI_NOALLOC_MAX_CELLS halo-padded cells ((Nx+2Hx)(Ny+2Hy)(Nz+2Hz)) and
//    PI_NOALLOC_MAX_GZ vertical levels; larger grids are rejected with PI_ERR_ARG;
//  - every call on a device shares the one array, and a call leaves its intermediates there;
//    nothing in it has to start at zero because each call writes every cell it later reads;
//  - calls whose work overlaps on the GPU (different streams, or host threads racing) race on the
//    array; serialise them, e.g. on one stream;
//  - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//    that device current; make that first call before any stream capture. The address is kept for
//    the life of the process, so the entry point must not be called again on a device after
//    cudaDeviceReset (or any other teardown of its primary context);
//  - the grid's dzF, dzC and land mask are host arrays: the call copies them into the fixed array
//    on `stream` and waits for that copy (and so for the work queued on the stream before it)
//    before returning, so the caller may free or change them as soon as the call returns. Only
//    the three sweeps stay queued.
#include <cstring>
#include <mutex>

#include "kernels_fp64.cuh"

#define PI_NOALLOC_MAX_CELLS (1 << 19)
#define PI_NOALLOC_MAX_GZ 4096

namespace {

constexpr size_t kFieldBytes = (size_t)PI_NOALLOC_MAX_CELLS * sizeof(double);
constexpr size_t kDzBytes = (size_t)PI_NOALLOC_MAX_GZ * sizeof(double);
constexpr size_t kScratchBytes = 2 * kFieldBytes + 2 * kDzBytes + (size_t)PI_NOALLOC_MAX_CELLS;

// tracer_temp after the x sweep | after the y sweep | dzF | dzC | landmask
static __device__ __align__(256) unsigned char pi_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_ptr[256] = { nullptr };
thread_local std::string g_err;

// x sweep of one field: calc_Gcˣ + fill_halo_Gcs + multi_dim_x (multi_dim_adv.jl:1-135)
__global__ void k_adv_x1(DGrid g, const double* __restrict__ c, double* __restrict__ tta,
                         const double* __restrict__ u, double dT) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1 + g.Hx;
    int j = blockIdx.y + 1 + g.Hy;
    int k = blockIdx.z + 1 + g.Hz;
    if (i > g.Nx + g.Hx) return;
    int q = gidx(g, i, j, k);
    double ax = g.dy * pib::dzF1(g, k);
    double ui = u[q], up = u[q + 1];
    int last = (i == g.Nx + g.Hx);
    int lm2 = pib::lmask(g, i - 2, j, k), lm1 = pib::lmask(g, i - 1, j, k), l0 = pib::lmask(g, i, j, k);
    int lp1 = pib::lmask(g, i + 1, j, k), lp2 = last ? 0 : pib::lmask(g, i + 2, j, k);
    double ftr = jl_mulb(jl_mulb(ax * up - ax * ui, lp1), l0);
    double c0 = c[q];
    double Fi = pib::dst3_flux_xy(c[q - 2], c[q - 1], c0, c[q + 1], lm2, lm1, l0, lp1, ui, ax, g.dx, dT);
    double Fp;
    if (!last) {
        Fp = pib::dst3_flux_xy(c[q - 1], c0, c[q + 1], c[q + 2], lm1, l0, lp1, lp2, up, ax, g.dx, dT);
    } else if (g.tx == PI_PERIODIC) {
        int qw = gidx(g, g.Hx + 1, j, k);
        Fp = pib::dst3_flux_xy(c[qw - 2], c[qw - 1], c[qw], c[qw + 1],
                               pib::lmask(g, g.Hx - 1, j, k), pib::lmask(g, g.Hx, j, k),
                               pib::lmask(g, g.Hx + 1, j, k), pib::lmask(g, g.Hx + 2, j, k), u[qw], ax, g.dx, dT);
    } else {
        Fp = 0.0;
    }
    double dG = jl_mulb(jl_mulb(Fp - Fi, lp1), l0);
    tta[q] = c0 - dT / pib::vol(g, k) * (dG - c0 * ftr);
}

// y sweep of one field on tracer_temp after x; the original field in the update term
__global__ void k_adv_y1(DGrid g, const double* __restrict__ c, const double* __restrict__ tta,
                         double* __restrict__ ttb, const double* __restrict__ v, double dT) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1 + g.Hx;
    int j = blockIdx.y + 1 + g.Hy;
    int k = blockIdx.z + 1 + g.Hz;
    if (i > g.Nx + g.Hx) return;
    int q = gidx(g, i, j, k);
    int last = (j == g.Ny + g.Hy);
    double ay = g.dx * pib::dzF1(g, k);
    double vj = v[q], vp = v[q + g.Gx];
    auto at = [&](int jj) { return tta[gidx(g, i, pib::wrap_axis(jj, g.Ny, g.Hy, g.ty), k)]; };
    int lm2 = pib::lmask(g, i, j - 2, k), lm1 = pib::lmask(g, i, j - 1, k), l0 = pib::lmask(g, i, j, k);
    int lp1 = pib::lmask(g, i, j + 1, k), lp2 = last ? 0 : pib::lmask(g, i, j + 2, k);
    double ftr = jl_mulb(jl_mulb(ay * vp - ay * vj, lp1), l0);
    double c0 = tta[q];
    double Fj = pib::dst3_flux_xy(at(j - 2), at(j - 1), c0, at(j + 1), lm2, lm1, l0, lp1, vj, ay, g.dy, dT);
    double Fp;
    if (!last) {
        Fp = pib::dst3_flux_xy(at(j - 1), c0, at(j + 1), at(j + 2), lm1, l0, lp1, lp2, vp, ay, g.dy, dT);
    } else if (g.ty == PI_PERIODIC) {
        int js = g.Hy + 1;
        Fp = pib::dst3_flux_xy(at(js - 2), at(js - 1), at(js), at(js + 1),
                               pib::lmask(g, i, js - 2, k), pib::lmask(g, i, js - 1, k), pib::lmask(g, i, js, k),
                               pib::lmask(g, i, js + 1, k), v[gidx(g, i, js, k)], ay, g.dy, dT);
    } else {
        Fp = 0.0;
    }
    double dG = jl_mulb(jl_mulb(Fp - Fj, lp1), l0);
    ttb[q] = c0 - dT / pib::vol(g, k) * (dG - c[q] * ftr);
}

// z sweep, then Gc = tracer_temp - tracer (calc_tracer_tendency!) on the interior
__global__ void k_adv_z1(DGrid g, const double* __restrict__ c, const double* __restrict__ ttb,
                         const double* __restrict__ w, double dT, double* __restrict__ Gc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1 + g.Hx;
    int j = blockIdx.y + 1 + g.Hy;
    int k = blockIdx.z + 1 + g.Hz;
    if (i > g.Nx + g.Hx) return;
    int q = gidx(g, i, j, k);
    const double az = g.dx * g.dy;
    auto at = [&](int kk) { return ttb[gidx(g, i, j, pib::wrap_axis(kk, g.Nz, g.Hz, PI_BOUNDED))]; };
    int last = (k == g.Nz + g.Hz);
    double wk = w[q], wp = w[q + g.Gx * g.Gy];
    int lm2 = pib::lmask(g, i, j, k - 2), lm1 = pib::lmask(g, i, j, k - 1), l0 = pib::lmask(g, i, j, k);
    int lp1 = pib::lmask(g, i, j, k + 1), lp2 = last ? 0 : pib::lmask(g, i, j, k + 2);
    double ftr = jl_mulb(jl_mulb(az * wk - az * wp, lp1), l0);
    double Ft = pib::dst3_flux_z(at(k - 2), at(k - 1), at(k), at(k + 1), lm2, lm1, l0, lp1, wk, az,
                                 pib::dzC1(g, k), dT);
    double Fb = last ? 0.0
                     : pib::dst3_flux_z(at(k - 1), at(k), at(k + 1), at(k + 2), lm1, l0, lp1, lp2, wp, az,
                                        pib::dzC1(g, k + 1), dT);
    double dG = jl_mulb(jl_mulb(Ft - Fb, lp1), l0);
    double cc = c[q];
    double ct = at(k) - dT / pib::vol(g, k) * (dG - cc * ftr);
    Gc[q] = ct - cc;
}

pi_status noalloc_fail(pi_status code, const char* msg) { g_err = msg; return code; }

}  // namespace

extern "C" {

pi_status pi_tracer_advection_noalloc(const pi_grid* grid, const double* c, const double* u,
                                      const double* v, const double* w, double dT, double* Gc,
                                      void* stream) {
    g_err.clear();
    if (!grid || !c || !u || !v || !w || !Gc || !grid->dzF || !grid->dzC)
        return noalloc_fail(PI_ERR_ARG, "pi_tracer_advection_noalloc: NULL argument");
    if (grid->Nx < 1 || grid->Ny < 1 || grid->Nz < 1 || grid->Hx < 2 || grid->Hy < 2 || grid->Hz < 2)
        return noalloc_fail(PI_ERR_ARG, "pi_tracer_advection_noalloc: grid size >= 1 and halo >= 2 required");
    if (grid->topo[2] != PI_BOUNDED || (grid->topo[0] != PI_PERIODIC && grid->topo[0] != PI_BOUNDED) ||
        (grid->topo[1] != PI_PERIODIC && grid->topo[1] != PI_BOUNDED))
        return noalloc_fail(PI_ERR_ARG, "pi_tracer_advection_noalloc: x/y Periodic or Bounded, z Bounded");
    if (grid->Nx < grid->Hx || grid->Ny < grid->Hy || grid->Nz < grid->Hz)
        return noalloc_fail(PI_ERR_ARG, "pi_tracer_advection_noalloc: every axis needs at least as many cells as halo points");
    if (grid->metrics)
        return noalloc_fail(PI_ERR_ARG, "pi_tracer_advection_noalloc: RectilinearGrid only (metrics must be NULL)");
    long long Gx = grid->Nx + 2LL * grid->Hx, Gy = grid->Ny + 2LL * grid->Hy, Gz = grid->Nz + 2LL * grid->Hz;
    long long G = Gx * Gy * Gz;
    if (G > PI_NOALLOC_MAX_CELLS || Gz > PI_NOALLOC_MAX_GZ)
        return noalloc_fail(PI_ERR_ARG, "pi_tracer_advection_noalloc: grid exceeds the fixed scratch "
                                        "(at most 524288 halo-padded cells and 4096 levels)");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256)
        return noalloc_fail(PI_ERR_CUDA, "pi_tracer_advection_noalloc: no current CUDA device");
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, pi_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return noalloc_fail(PI_ERR_CUDA, "pi_tracer_advection_noalloc: cudaGetSymbolAddress failed");
            g_ptr[dev] = p;
        }
        base = (unsigned char*)g_ptr[dev];
    }
    double* tta = (double*)base;
    double* ttb = (double*)(base + kFieldBytes);
    double* dzF = (double*)(base + 2 * kFieldBytes);
    double* dzC = (double*)(base + 2 * kFieldBytes + kDzBytes);
    uint8_t* lm = (uint8_t*)(base + 2 * kFieldBytes + 2 * kDzBytes);
    cudaStream_t st = (cudaStream_t)stream;
    int all_water = 1;
    if (grid->landmask)
        for (long long q = 0; q < G; ++q) if (grid->landmask[q] != 1) { all_water = 0; break; }
    if (cudaMemcpyAsync(dzF, grid->dzF, Gz * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dzC, grid->dzC, Gz * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (!all_water && cudaMemcpyAsync(lm, grid->landmask, G, cudaMemcpyHostToDevice, st) != cudaSuccess))
        return noalloc_fail(PI_ERR_CUDA, "pi_tracer_advection_noalloc: copy of grid metrics failed");
    // the caller's host arrays are released on return: wait until the stream has read them
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return noalloc_fail(PI_ERR_CUDA, "pi_tracer_advection_noalloc: copy of grid metrics failed");
    DGrid g{grid->Nx, grid->Ny, grid->Nz, grid->Hx, grid->Hy, grid->Hz, (int)Gx, (int)Gy, (int)Gz,
            grid->topo[0], grid->topo[1], grid->topo[2], all_water, grid->dx, grid->dy, dzF, dzC, lm, G};
    dim3 blk(128), grd((grid->Nx + 127) / 128, grid->Ny, grid->Nz);
    k_adv_x1<<<grd, blk, 0, st>>>(g, c, tta, u, dT);
    k_adv_y1<<<grd, blk, 0, st>>>(g, c, tta, ttb, v, dT);
    k_adv_z1<<<grd, blk, 0, st>>>(g, c, ttb, w, dT, Gc);
    if (cudaGetLastError() != cudaSuccess)
        return noalloc_fail(PI_ERR_CUDA, "pi_tracer_advection_noalloc: kernel launch failed");
    return PI_OK;
}

pi_status pi_noalloc_last_error(char* buf, size_t len) {
    if (buf && len) {
        size_t n = g_err.size() < len - 1 ? g_err.size() : len - 1;
        memcpy(buf, g_err.c_str(), n);
        buf[n] = 0;
    }
    return PI_OK;
}

}  // extern "C"
