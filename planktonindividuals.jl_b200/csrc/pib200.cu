// libpib200 — C ABI (include/pib200.h) and step orchestration of the B200 model time step.
//
// One handle = one PlanktonModel on the CUDA device current at pi_create, with its own stream.
// A step (TimeStep!, src/Model/time_step.jl:12-180) is this sequence of launches:
//   k_particles          RK4 + diffusion + find_inds! for every species; per-cell counts
//   scan(cnt) → off      cell offsets of the binned individuals
//   radix sort           (cell, species·C + slot) order = the order of a sequential reference run
//   k_setpos             position of each individual in the cell-sorted list
//   k_par                Chl per cell, calc_par! down each column, PAR diagnostic
//   per species:         k_decide → scan(flags) → k_lists → k_daughters → k_physiology
//   k_sweep_x/y          DST3FL sweeps on tracer_temp
//   k_sweep_z            z sweep and the advective tendency
//   k_tracer_tail        diffusion, sinking, forcing, BCs, particle terms, apply_tendency!
//   k_halo<x,y,z>        fill_halo_tracer! on the new tracers
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels_fp64.cuh"
#include "kernels_abiotic.cuh"
#include "kernels_iron.cuh"
#include "host_common.h"

using namespace pib;
using namespace pih;

namespace {

thread_local std::string g_create_error;

struct DevBC {
    int kind = PI_BC_NONE;
    long long nt = 0;
    double* v = nullptr;
};

}  // namespace

struct pi_model {
    int device = 0;
    cudaStream_t stream = nullptr;
    HostGrid hg;
    DGrid dg;
    pi_bgc_params bgc;
    std::vector<pi_quota_params> sp;
    int nsp = 0;
    long long C = 0;
    uint64_t seed = 0;
    int precision = PI_FP64;
    pi_batch* b32 = nullptr;     // PI_FP32: the model is a batch of one member
    int carbon = 0;              // CarbonMode species (pi_create_carbon)
    std::vector<pi_carbon_params> cp;
    int macro = 0;               // MacroMolecularMode species (pi_create_macro)
    std::vector<pi_macro_params> mp;
    int iron = 0;                // IronEnergyMode species (pi_create_iron)
    std::vector<pi_iron_params> ipp;
    double* par0 = nullptr;      // G: par of the previous step (timestepper.par₀), IronEnergyMode only
    int mode() const { return iron ? MODE_IRON : macro ? MODE_MACRO : carbon ? MODE_CARBON : MODE_QUOTA; }
    int64_t iteration = 0;
    double t = 0.0;
    double last_dT = 0.0;
    std::string err;
    std::vector<void*> allocs;

    // device state
    std::vector<SpcDev> h_spc;
    SpcDev* d_spc = nullptr;
    double* tr = nullptr;        // 14 × G
    double* tr_next = nullptr;   // 14 × G
    double* tta = nullptr;       // 14 × G
    double* ttb = nullptr;       // 14 × G
    double* velbuf[2][3] = {{nullptr}};
    const double* vel0[3] = {nullptr, nullptr, nullptr};
    const double* vel1[3] = {nullptr, nullptr, nullptr};
    int vel1_buf = 1;            // own buffer that vel1 points to, -1 when bound to a series
    double* zeros = nullptr;     // G zeros (vel₀ before the first step)
    double* par = nullptr;       // G
    double* PARF = nullptr;      // Nx·Ny
    double* temp_own = nullptr;  // G
    double* stage = nullptr;     // 3 × G staging for interior uploads
    double* velh[3] = {nullptr, nullptr, nullptr};   // vel½
    const double* temp = nullptr;
    double* diag_par = nullptr;  // G
    double* diag_sp = nullptr;   // nsp × 4 × G (num, graz, mort, dvid)
    // optional diagnostics (pi_set_diags)
    uint32_t tr_mask = 0, proc_mask = 0;
    double* diag_tr = nullptr;   // 14 × G
    double* diag_proc = nullptr; // nsp × PI_MAXPROC × G
    double* procv = nullptr;     // PI_MAXPROC × C values of the species being updated
    double* budget_part = nullptr;   // 3 × 512 block partials of pi_get_budget
    uint32_t *dkey = nullptr, *dkey_s = nullptr, *dval = nullptr, *dval_s = nullptr;
    void* dsort_tmp = nullptr;
    size_t dsort_bytes = 0;
    double* dzF = nullptr;
    double* dzC = nullptr;
    uint8_t* lm = nullptr;
    double* met = nullptr;           // LatLonGrid metrics: dxC, dyC, dxF, dyF, Az (Gx·Gy each), Ax, Ay, Vol (G each)
    std::vector<double> met_host;    // their host copy, the source of the upload
    StepBufs sb{};
    uint32_t* iota = nullptr;    // nsp·C
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int key_bits = 1;
    DevBC bcs[PI_NTRACERS][6];
    FluxBCDev* d_bcs = nullptr;
    int any_bc = 0;
    // abiotic particles (pi_set_abiotics): species, their particle flux boundary conditions, the
    // Palat pairs, the candidate rows intac (max_candidates per particle slot) and the scratch of
    // the cell binning, boundary creation and free-slot lists
    int nsa = 0;
    std::vector<pi_abiotic_params> ap;
    std::vector<AbioDev> h_ab;
    std::vector<DevBC> abc;                 // nsa × 6
    std::vector<std::pair<int, int>> pal_intac, pal_release;
    int maxc = 25;
    std::vector<double> max_ptc;
    int32_t* intac = nullptr;
    double* diag_ptc = nullptr;             // nsp × G
    double* diag_abn = nullptr;             // nsa × G
    uint32_t *akey = nullptr, *akey_s = nullptr, *aval = nullptr, *aval_s = nullptr;   // C each
    uint32_t *pkey = nullptr, *pkey_s = nullptr, *pval = nullptr, *pval_s = nullptr;   // C each
    uint32_t *cflag = nullptr, *crank = nullptr;                                        // G each
    uint32_t *afl = nullptr, *afr = nullptr;                                            // C each
    int32_t* afree = nullptr;                                                           // C
    void* atmp = nullptr;
    size_t abytes = 0;
    // optional per-kernel event timing
    int profiling = 0;
    struct Mark { const char* name; cudaEvent_t a, b; };
    std::vector<Mark> marks;            // recorded, not yet read
    std::vector<cudaEvent_t> event_pool;
    std::vector<std::string> prof_names;
    std::vector<int64_t> prof_count;
    std::vector<double> prof_ms;
};

struct pi_sim {
    pi_model* m = nullptr;
    int fp32 = 0;
    double dT = 0.0;
    int64_t iterations = 0;
    int has_vel = 0;
    int64_t nvel = 0, npar = 0, ntemp = 0;
    double dT_vel = 0.0, dT_PAR = 0.0, dT_temp = 0.0;
    std::vector<double*> vel;     // 3 × nvel halo-padded fields
    double* parf = nullptr;       // Nx·Ny × npar
    std::vector<double*> temp;    // ntemp halo-padded fields
};

namespace {

pi_status fail(pi_model* m, pi_status code, const std::string& msg) {
    if (m) m->err = msg; else g_create_error = msg;
    return code;
}

// Result of a call forwarded to the FP32 batch of a PI_FP32 model, with its message.
pi_status fwd32(pi_model* m, pi_status st) {
    if (st != PI_OK) {
        char buf[1024];
        pi_batch_last_error(m->b32, buf, sizeof buf);
        m->err = buf;
    }
    return st;
}

pi_status cuda_fail(pi_model* m, cudaError_t e, const char* what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(m, e == cudaErrorMemoryAllocation ? PI_ERR_NOMEM : PI_ERR_CUDA, msg);
}

#define CK(call, what)                                              \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return cuda_fail(m, e_, what);       \
    } while (0)

template <typename T>
pi_status dalloc(pi_model* m, T** p, size_t n, const char* what) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(m, e, what);
    m->allocs.push_back(q);
    *p = (T*)q;
    return PI_OK;
}

#define AL(ptr, n) do { pi_status s_ = dalloc(m, &(ptr), (size_t)(n), #ptr); if (s_) return s_; } while (0)

void free_all(pi_model* m) {
    for (void* p : m->allocs) cudaFree(p);
    m->allocs.clear();
    for (int n = 0; n < PI_NTRACERS; ++n)
        for (int f = 0; f < 6; ++f)
            if (m->bcs[n][f].v) { cudaFree(m->bcs[n][f].v); m->bcs[n][f].v = nullptr; }
    for (DevBC& b : m->abc)
        if (b.v) { cudaFree(b.v); b.v = nullptr; }
}

inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

cudaEvent_t take_event(pi_model* m) {
    if (!m->event_pool.empty()) { cudaEvent_t e = m->event_pool.back(); m->event_pool.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// Brackets one kernel launch (or library call) with events when profiling is on.
struct ProfScope {
    pi_model* m;
    pi_model::Mark mk;
    ProfScope(pi_model* m_, const char* name) : m(m_) {
        if (!m->profiling) return;
        mk.name = name; mk.a = take_event(m); mk.b = take_event(m);
        cudaEventRecord(mk.a, m->stream);
    }
    ~ProfScope() {
        if (!m->profiling) return;
        cudaEventRecord(mk.b, m->stream);
        m->marks.push_back(mk);
    }
};

void drain_marks(pi_model* m) {
    for (auto& mk : m->marks) {
        float ms = 0.f;
        cudaEventSynchronize(mk.b);
        cudaEventElapsedTime(&ms, mk.a, mk.b);
        size_t q = 0;
        while (q < m->prof_names.size() && m->prof_names[q] != mk.name) ++q;
        if (q == m->prof_names.size()) { m->prof_names.push_back(mk.name); m->prof_count.push_back(0); m->prof_ms.push_back(0.0); }
        m->prof_count[q] += 1;
        m->prof_ms[q] += ms;
        m->event_pool.push_back(mk.a);
        m->event_pool.push_back(mk.b);
    }
    m->marks.clear();
}

// Reads and clears the device error word; converts it to a status.
pi_status check_device_errors(pi_model* m) {
    uint32_t err = 0;
    int64_t it = 0;
    CK(cudaMemcpyAsync(&err, m->sb.err, sizeof err, cudaMemcpyDeviceToHost, m->stream), "read error word");
    CK(cudaMemcpyAsync(&it, m->sb.err_iter, sizeof it, cudaMemcpyDeviceToHost, m->stream), "read error iteration");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    if (!err) return PI_OK;
    CK(cudaMemsetAsync(m->sb.err, 0, sizeof(uint32_t), m->stream), "clear error word");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    if (err & PI_DEVERR_MAXPTC)     // merge_particle_kernel! reads plank_p.max_ptc (particle_interaction.jl:58)
        return fail(m, PI_ERR_PARAM, "type NamedTuple has no field max_ptc");
    if (err & PI_DEVERR_CAPACITY) {
        double tf = (double)it * m->last_dT;    // model.t of the failing step
        return fail(m, PI_ERR_CAPACITY, std::string(err & PI_DEVERR_ABIO ? "number of abiotic particles" : "number of individual") +
                                            " exceeds the capacity at timestep " + julia_float(tf / 86400.0) + " days");
    }
    return fail(m, PI_ERR_DOMAIN, "an individual left the halo-padded grid (cell index out of range)");
}

// The abiotic phase before the phytoplankton (time_step.jl:24-39): for each abiotic species,
// particles_from_bcs! (particle_interaction.jl:252-271), then the particle step.
pi_status enqueue_abiotic_update(pi_model* m, double dT, const VelPtrs& vp) {
    const DGrid& g = m->dg;
    const long long G = g.G, C = m->C;
    const uint32_t iter = (uint32_t)m->iteration;
    cudaStream_t st = m->stream;
    StepBufs& sb = m->sb;
    const bool ll = m->met != nullptr;
    const int BS = 256;
    for (int sa = 0; sa < m->nsa; ++sa) {
        const AbioDev& A = m->h_ab[sa];
        const DevBC* B = &m->abc[(size_t)sa * 6];
        bool any = false;
        for (int f = 0; f < 6; ++f) any = any || B[f].kind != PI_BC_NONE;
        if (any) {
            ProfScope ps_(m, "k_abio_bcs");
            CK(cudaMemsetAsync(m->cflag, 0, G * sizeof(uint32_t), st), "zero tr_temp");
            const HostGrid& hg = m->hg;
            const pi_abiotic_params& p = m->ap[sa];
            auto face = [&](int f) -> FluxBCDev {
                FluxBCDev d;
                d.kind = B[f].kind; d.nt = B[f].nt; d.v = B[f].v;
                d.n1 = f <= PI_EAST ? hg.Ny : hg.Nx;
                d.n2 = f <= PI_NORTH ? hg.Nz : hg.Ny;
                return d;
            };
            const long long nxy = (long long)hg.Nx * hg.Ny, nyz = (long long)hg.Ny * hg.Nz, nxz = (long long)hg.Nx * hg.Nz;
#define ABIO_FACE(F, N) if (B[F].kind) (ll ? k_abio_bc_face<true, F> : k_abio_bc_face<false, F>)<<<nblk(N, BS), BS, 0, st>>>( \
                g, face(F), p.sz_min, p.Nsuper, dT, m->seed, m->iteration, sa, m->cflag, sb.err)
            ABIO_FACE(PI_TOP, nxy); ABIO_FACE(PI_BOTTOM, nxy); ABIO_FACE(PI_EAST, nyz);
            ABIO_FACE(PI_WEST, nyz); ABIO_FACE(PI_NORTH, nxz); ABIO_FACE(PI_SOUTH, nxz);
#undef ABIO_FACE
            CK(cudaGetLastError(), "k_abio_bc_face");
            size_t tb = m->abytes;
            CK(cub::DeviceScan::ExclusiveSum(m->atmp, tb, m->cflag, m->crank, (int)G, st), "scan boundary cells");
            k_abio_free_flags<<<nblk(C, BS), BS, 0, st>>>(A, C, m->afl);
            tb = m->abytes;
            CK(cub::DeviceScan::ExclusiveSum(m->atmp, tb, m->afl, m->afr, (int)C, st), "scan free particle slots");
            k_abio_free_list<<<nblk(C, BS), BS, 0, st>>>(m->afl, m->afr, C, m->afree);
            k_abio_place<<<nblk(G, BS), BS, 0, st>>>(g, A, C, m->cflag, m->crank, m->afl, m->afr, m->afree, sb.err,
                                                      sb.err_iter, m->iteration);
            CK(cudaGetLastError(), "k_abio_place");
        }
        ProfScope ps_(m, "k_abio_move");
        (ll ? k_abio_move<true> : k_abio_move<false>)<<<nblk(C, 128), 128, 0, st>>>(g, A, C, sa, dT, m->seed, iter, vp,
                                                                                     m->bgc.kappa_hP, m->bgc.kappa_vP, sb.err);
        CK(cudaGetLastError(), "k_abio_move");
    }
    return PI_OK;
}

// The interaction, the release and their diagnostics after the phytoplankton (time_step.jl:120-158).
pi_status enqueue_abiotic_exchange(pi_model* m, double dT) {
    const DGrid& g = m->dg;
    const long long G = g.G, C = m->C;
    const uint32_t iter = (uint32_t)m->iteration;
    cudaStream_t st = m->stream;
    StepBufs& sb = m->sb;
    const bool ll = m->met != nullptr;
    const int BS = 256;
    for (const auto& pr : m->pal_intac) {
        ProfScope ps_(m, "k_interact");
        const SpcDev& P = m->h_spc[pr.first];
        const AbioDev& A = m->h_ab[pr.second];
        k_diag_keys<<<nblk(C, BS), BS, 0, st>>>(g, P, C, m->pkey, m->pval, sb.err);
        k_abio_keys<<<nblk(C, BS), BS, 0, st>>>(g, A, C, m->akey, m->aval, sb.err);
        size_t tb = m->abytes;
        CK(cub::DeviceRadixSort::SortPairs(m->atmp, tb, m->pkey, m->pkey_s, m->pval, m->pval_s, (int64_t)C, 0, m->key_bits, st),
           "sort phytoplankton by cell");
        tb = m->abytes;
        CK(cub::DeviceRadixSort::SortPairs(m->atmp, tb, m->akey, m->akey_s, m->aval, m->aval_s, (int64_t)C, 0, m->key_bits, st),
           "sort particles by cell");
        (ll ? k_interact<true> : k_interact<false>)<<<nblk(C, 128), 128, 0, st>>>(
            g, P, A, C, m->pkey_s, m->pval_s, m->akey_s, m->aval_s, m->ap[pr.second].Rd, m->maxc, m->max_ptc[pr.first],
            m->intac, sb.err, sb.err_iter, m->iteration);
        CK(cudaGetLastError(), "k_interact");
    }
    for (size_t q = 0; q < m->pal_release.size(); ++q) {
        ProfScope ps_(m, "k_release");
        const auto& pr = m->pal_release[q];
        const SpcDev& P = m->h_spc[pr.first];
        const AbioDev& A = m->h_ab[pr.second];
        k_release_flags<<<nblk(C, BS), BS, 0, st>>>(P, A, C, m->ap[pr.second].release_P, dT, m->seed, iter, (int)q,
                                                    sb.flag64, sb.err);
        size_t tb = m->cub_bytes;
        CK(cub::DeviceScan::ExclusiveSum(m->cub_tmp, tb, sb.flag64, sb.rank64, (int64_t)C, st), "scan release flags");
        k_lists<<<nblk(C, BS), BS, 0, st>>>(sb.flag64, sb.rank64, C, sb.divlist, sb.freelist, sb.ndiv, sb.err, sb.err_iter,
                                            m->iteration, PI_DEVERR_CAPACITY | PI_DEVERR_ABIO);
        k_release<<<148 * 2, 256, 0, st>>>(P, A, sb.divlist, sb.freelist, sb.ndiv, m->seed, iter, (int)q, m->nsp - 1, sb.err);
        CK(cudaGetLastError(), "k_release");
    }
    {
        ProfScope ps_(m, "k_abio_diags");
        for (int s = 0; s < m->nsp; ++s) {          // diags.phytos[sp].ptc in ascending slot order per cell
            k_diag_keys<<<nblk(C, BS), BS, 0, st>>>(g, m->h_spc[s], C, m->pkey, m->pval, sb.err);
            size_t tb = m->abytes;
            CK(cub::DeviceRadixSort::SortPairs(m->atmp, tb, m->pkey, m->pkey_s, m->pval, m->pval_s, (int64_t)C, 0, m->key_bits, st),
               "sort phytoplankton by cell");
            k_diag_sum<<<nblk(C, BS), BS, 0, st>>>(C, G, m->pkey_s, m->pval_s, m->h_spc[s].ptc, 1u, m->diag_ptc + (size_t)s * G);
        }
        for (int sa = 0; sa < m->nsa; ++sa)
            k_abio_num<<<nblk(C, BS), BS, 0, st>>>(g, m->h_ab[sa], C, m->diag_abn + (size_t)sa * G, sb.err);
        CK(cudaGetLastError(), "k_abio_diags");
    }
    return PI_OK;
}

// Enqueues one TimeStep! on the model's stream (no synchronisation).
pi_status enqueue_step(pi_model* m, double dT) {
    // getbc(bc, i, j, t) of a time-dependent flux reads bc[i, j, iteration] (boundary_conditions.jl:44-52)
    for (int n = 0; n < PI_NTRACERS; ++n)
        for (int f = 0; f < 6; ++f)
            if (m->bcs[n][f].kind == PI_BC_ARRAY3D && m->bcs[n][f].nt < m->iteration + 1)
                return fail(m, PI_ERR_SHAPE, "BoundsError: time-dependent flux boundary condition has " +
                                                 std::to_string(m->bcs[n][f].nt) + " snapshots, step " +
                                                 std::to_string(m->iteration + 1) + " needs one more");
    for (const DevBC& b : m->abc)
        if (b.kind == PI_BC_ARRAY3D && b.nt < m->iteration + 1)
            return fail(m, PI_ERR_SHAPE, "BoundsError: time-dependent particle flux boundary condition has " +
                                             std::to_string(b.nt) + " snapshots, step " + std::to_string(m->iteration + 1) +
                                             " needs one more");
    m->iteration += 1;
    m->t = (double)m->iteration * dT;
    m->last_dT = dT;
    const DGrid& g = m->dg;
    const long long G = g.G, C = m->C, NC = (long long)m->nsp * C;
    const uint32_t iter = (uint32_t)m->iteration;
    cudaStream_t st = m->stream;
    StepBufs& sb = m->sb;
    const int BS = 256;

    CK(cudaMemsetAsync(sb.cnt, 0, (G + 1) * sizeof(uint32_t), st), "zero counts");
    { ProfScope ps_(m, "k_velhalf");
    k_velhalf<<<148 * 8, 256, 0, st>>>(G, m->vel0[0], m->vel0[1], m->vel0[2], m->vel1[0], m->vel1[1], m->vel1[2],
                                       m->velh[0], m->velh[1], m->velh[2], sb.err);
    CK(cudaGetLastError(), "k_velhalf"); }
    VelPtrs vp{m->vel0[0], m->vel0[1], m->vel0[2], m->velh[0], m->velh[1], m->velh[2],
               m->vel1[0], m->vel1[1], m->vel1[2]};
    const bool ll = m->met != nullptr;      // LatLonGrid: the kernels that read grid metrics take their arrays
    if (m->nsa) { pi_status e = enqueue_abiotic_update(m, dT, vp); if (e) return e; }
    { ProfScope ps_(m, "k_particles_sorted");
    (ll ? k_particles_sorted<true> : k_particles_sorted<false>)<<<nblk(NC, 128), 128, 0, st>>>(g, m->d_spc, C, sb.gid_sorted, sb.off, G, dT, m->seed, iter, vp,
                                                      m->bgc.kappa_hP, m->bgc.kappa_vP, sb.cnt, sb.key, sb.err);
    CK(cudaGetLastError(), "k_particles_sorted"); }
    { ProfScope ps_(m, "k_particles");
    (ll ? k_particles<true> : k_particles<false>)<<<nblk(NC, BS), BS, 0, st>>>(g, m->d_spc, m->nsp, C, dT, m->seed, iter, vp,
                                             m->bgc.kappa_hP, m->bgc.kappa_vP, sb.cnt, sb.key,
                                             (uint32_t)G, sb.err);
    CK(cudaGetLastError(), "k_particles"); }
    size_t tb = m->cub_bytes;
    { ProfScope ps_(m, "cub_scan_cells");
    CK(cub::DeviceScan::ExclusiveSum(m->cub_tmp, tb, sb.cnt, sb.off, (int)(G + 1), st), "scan counts"); }
    tb = m->cub_bytes;
    { ProfScope ps_(m, "cub_sort_cells");
    CK(cub::DeviceRadixSort::SortPairs(m->cub_tmp, tb, sb.key, sb.key_sorted, m->iota, sb.gid_sorted,
                                       (int64_t)NC, 0, m->key_bits, st), "sort by cell"); }
    { ProfScope ps_(m, "k_setpos");
    k_setpos<<<nblk(NC, BS), BS, 0, st>>>(sb.off, G, sb.gid_sorted, sb.pos, NC, sb.err);
    CK(cudaGetLastError(), "k_setpos"); }
    {
        dim3 grid(nblk(g.Nx, 128), g.Ny);
        ProfScope ps_(m, "k_par");
        (ll ? k_par<true> : k_par<false>)<<<grid, 128, 0, st>>>(g, m->d_spc, C, sb.off, sb.gid_sorted, m->PARF, m->PARF, m->par,
                                    m->diag_par, m->bgc.kc, m->bgc.kw, sb.err);
        CK(cudaGetLastError(), "k_par");
    }
    const int shared = m->bgc.shared_graz == 1.0;
    for (int s = 0; s < m->nsp; ++s) {
        double* dsp = m->diag_sp + (size_t)s * 4 * G;
        { ProfScope ps_(m, "k_decide");
        const pi_macro_params mpz = m->macro ? m->mp[s] : pi_macro_params{};
        const pi_iron_params ipz = m->iron ? m->ipp[s] : pi_iron_params{};
        k_decide<<<nblk(C, BS), BS, 0, st>>>(g, m->h_spc[s], m->sp[s], mpz, ipz, C, s, sb.pos, sb.loss, sb.evk,
                                             sb.flag64, dsp + 1 * G, dsp + 2 * G, dsp + 3 * G, sb.err, m->mode());
        CK(cudaGetLastError(), "k_decide"); }
        tb = m->cub_bytes;
        { ProfScope ps_(m, "cub_scan_slots");
        CK(cub::DeviceScan::ExclusiveSum(m->cub_tmp, tb, sb.flag64, sb.rank64, (int64_t)C, st), "scan division flags"); }
        { ProfScope ps_(m, "k_lists");
        k_lists<<<nblk(C, BS), BS, 0, st>>>(sb.flag64, sb.rank64, C, sb.divlist, sb.freelist, sb.ndiv,
                                            sb.err, sb.err_iter, m->iteration);
        CK(cudaGetLastError(), "k_lists"); }
        { ProfScope ps_(m, "k_daughters");
        k_daughters<<<148 * 4, 256, 0, st>>>(m->h_spc[s], sb.divlist, sb.freelist, sb.ndiv, sb.err, m->mode());
        CK(cudaGetLastError(), "k_daughters"); }
        const double* trp = m->tr;
        if (m->iron) { ProfScope ps_(m, "k_physiology");
        k_physiology_iron<<<nblk(C, BS), BS, 0, st>>>(g, m->h_spc[s], m->ipp[s], C, s, dT, m->t, m->seed, iter, shared,
                                                      trp + PI_NH4 * G, trp + PI_NO3 * G, trp + PI_PO4 * G,
                                                      trp + PI_DFe * G, m->par, m->par0, m->temp, sb.off, sb.gid_sorted,
                                                      sb.pos, sb.contrib, dsp + 0 * G,
                                                      m->proc_mask ? m->procv : nullptr, sb.err);
        CK(cudaGetLastError(), "k_physiology_iron"); } else
        if (m->macro) { ProfScope ps_(m, "k_physiology");
        k_physiology_macro<<<nblk(C, BS), BS, 0, st>>>(g, m->h_spc[s], m->mp[s], C, s, dT, m->seed, iter, shared,
                                                       trp + PI_NH4 * G, trp + PI_NO3 * G, trp + PI_PO4 * G,
                                                       trp + PI_DOC * G, m->par, m->temp, sb.off, sb.gid_sorted,
                                                       sb.pos, sb.contrib, dsp + 0 * G,
                                                       m->proc_mask ? m->procv : nullptr, sb.err);
        CK(cudaGetLastError(), "k_physiology_macro"); } else
        if (m->carbon) { ProfScope ps_(m, "k_physiology");
        k_physiology_carbon<<<nblk(C, BS), BS, 0, st>>>(g, m->h_spc[s], m->cp[s], C, s, dT, m->t, m->seed, iter,
                                                        shared, m->par, m->temp, sb.off, sb.gid_sorted, sb.pos,
                                                        sb.contrib, dsp + 0 * G, m->proc_mask ? m->procv : nullptr, sb.err);
        CK(cudaGetLastError(), "k_physiology_carbon"); } else
        { ProfScope ps_(m, "k_physiology");
        k_physiology<<<nblk(C, BS), BS, 0, st>>>(g, m->h_spc[s], m->sp[s], C, s, dT, m->t, m->seed, iter,
                                                 shared, trp + PI_NH4 * G, trp + PI_NO3 * G,
                                                 trp + PI_PO4 * G, trp + PI_DOC * G, m->par, m->temp,
                                                 sb.off, sb.gid_sorted, sb.pos, sb.contrib,
                                                 dsp + 0 * G, m->proc_mask ? m->procv : nullptr, sb.err);
        CK(cudaGetLastError(), "k_physiology"); }
        if (m->proc_mask) {
            ProfScope ps_(m, "k_diag_proc");
            k_diag_keys<<<nblk(C, BS), BS, 0, st>>>(g, m->h_spc[s], C, m->dkey, m->dval, sb.err);
            size_t db = m->dsort_bytes;
            CK(cub::DeviceRadixSort::SortPairs(m->dsort_tmp, db, m->dkey, m->dkey_s, m->dval, m->dval_s, (int64_t)C,
                                               0, m->key_bits, st), "sort diagnostics by cell");
            k_diag_sum<<<nblk(C, BS), BS, 0, st>>>(C, G, m->dkey_s, m->dval_s, m->procv, m->proc_mask,
                                                   m->diag_proc + (size_t)s * PI_MAXPROC * G);
            CK(cudaGetLastError(), "k_diag_proc");
        }
    }
    if (m->nsa) { pi_status e = enqueue_abiotic_exchange(m, dT); if (e) return e; }
    {
        { ProfScope ps_(m, "k_sweep_x");
        (ll ? k_sweep_x<true> : k_sweep_x<false>)<<<dim3(nblk(nblk(g.Nx, 31), SWX_WARPS), g.Ny, g.Nz), 32 * SWX_WARPS, 0, st>>>(g, m->tr, m->tta, m->vel1[0], dT, sb.err);
        CK(cudaGetLastError(), "k_sweep_x"); }
        { ProfScope ps_(m, "k_sweep_y");
        (ll ? k_sweep_y<true> : k_sweep_y<false>)<<<dim3(nblk(g.Nx, 32), nblk(nblk(g.Ny, SWY_L), SWY_TY), g.Nz), dim3(32, SWY_TY), 0, st>>>(g, m->tr, m->tta, m->ttb, m->vel1[1], dT, sb.err);
        CK(cudaGetLastError(), "k_sweep_y"); }
        ZFinalArgs za;
        za.g = g; za.tr = m->tr; za.ttb = m->ttb; za.tr_next = m->tr_next; za.w = m->vel1[2];
        za.dT = dT; za.b = m->bgc;
        za.diffuse = (m->bgc.kappa_h != 0.0 || m->bgc.kappa_v != 0.0);
        za.any_bc = m->any_bc; za.bcs = m->d_bcs; za.iter = m->iteration;
        za.spc = m->d_spc; za.C = C; za.off = sb.off; za.gid_sorted = sb.gid_sorted; za.evk = sb.evk;
        za.loss = sb.loss; za.contrib = sb.contrib; za.nsp = m->nsp; za.err = sb.err;
        za.gadv = m->tta;      // the x-sweep output is no longer needed
        { ProfScope ps_(m, "k_sweep_z");
        (ll ? k_sweep_z<true> : k_sweep_z<false>)<<<dim3(nblk(g.Nx, 32), g.Ny, nblk(nblk(g.Nz, SWZ_L), SWZ_TZ)), dim3(32, SWZ_TZ), 0, st>>>(
            g, m->tr, m->ttb, m->tta, m->vel1[2], dT, sb.err);
        CK(cudaGetLastError(), "k_sweep_z"); }
        { ProfScope ps_(m, "k_tracer_tail");
        (m->iron ? (ll ? k_tracer_tail<true, true> : k_tracer_tail<false, true>)
                 : (ll ? k_tracer_tail<true, false> : k_tracer_tail<false, false>))<<<dim3(nblk(g.Nx, 128), g.Ny, g.Nz), 128, 0, st>>>(za);
        CK(cudaGetLastError(), "k_tracer_tail"); }
        // tracers are only replaced when the step completed (a capacity error leaves them)
        { ProfScope ps_(m, "k_halo");
        k_halo<0><<<dim3(nblk(g.Gy, 64), g.Gz, PI_NTRACERS), 64, 0, st>>>(g, m->tr_next, PI_NTRACERS, sb.err);
        k_halo<1><<<dim3(nblk(g.Gx, 64), g.Gz, PI_NTRACERS), 64, 0, st>>>(g, m->tr_next, PI_NTRACERS, sb.err);
        k_halo<2><<<dim3(nblk(g.Gx, 64), g.Gy, PI_NTRACERS), 64, 0, st>>>(g, m->tr_next, PI_NTRACERS, sb.err);
        CK(cudaGetLastError(), "k_halo"); }
        k_copy_if_err<<<148 * 4, 256, 0, st>>>(m->tr_next, m->tr, PI_NTRACERS * G, sb.err);
        CK(cudaGetLastError(), "k_copy_if_err");
        if (m->tr_mask) {
            k_diag_tracers<<<148 * 4, 256, 0, st>>>(m->diag_tr, m->tr_next, m->tr_mask, G, sb.err);
            CK(cudaGetLastError(), "k_diag_tracers");
        }
    }
    std::swap(m->tr, m->tr_next);
    for (int c = 0; c < 3; ++c) m->vel0[c] = m->vel1[c];    // vel₀ .= vel₁ (time_step.jl:174-176)
    if (m->par0) CK(cudaMemcpyAsync(m->par0, m->par, G * sizeof(double), cudaMemcpyDeviceToDevice, st), "par₀ .= par");
    return PI_OK;
}

pi_status upload_bcs(pi_model* m) {
    std::vector<FluxBCDev> h(PI_NTRACERS * 6);
    m->any_bc = 0;
    const HostGrid& g = m->hg;
    for (int n = 0; n < PI_NTRACERS; ++n)
        for (int f = 0; f < 6; ++f) {
            FluxBCDev& d = h[n * 6 + f];
            d.kind = m->bcs[n][f].kind;
            d.nt = m->bcs[n][f].nt;
            d.v = m->bcs[n][f].v;
            d.n1 = f <= PI_EAST ? g.Ny : g.Nx;
            d.n2 = f <= PI_NORTH ? g.Nz : g.Ny;
            if (d.kind) m->any_bc = 1;
        }
    CK(cudaMemcpyAsync(m->d_bcs, h.data(), h.size() * sizeof(FluxBCDev), cudaMemcpyHostToDevice, m->stream), "upload bcs");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

pi_status validate_quota(const pi_quota_params& p, int s, std::string& msg) {
    int ty = (int)p.dvid_type;
    if ((double)ty != p.dvid_type || ty < 1 || ty > 3) {
        msg = "Wrong cell division type, must be in 1 to 3 (species " + std::to_string(s + 1) + ")";
        return PI_ERR_PARAM;
    }
    return PI_OK;
}

}  // namespace

extern "C" {

const char* pi_status_string(pi_status code) {
    switch (code) {
        case PI_OK: return "ok";
        case PI_ERR_ARG: return "invalid argument";
        case PI_ERR_SHAPE: return "dimension mismatch";
        case PI_ERR_PARAM: return "invalid parameter";
        case PI_ERR_CAPACITY: return "number of individuals exceeds the capacity";
        case PI_ERR_CUDA: return "CUDA error";
        case PI_ERR_TIMEOUT: return "device wait timed out";
        case PI_ERR_NAN: return "NaN found";
        case PI_ERR_DOMAIN: return "individual outside the grid";
        case PI_ERR_NOMEM: return "out of device memory";
        case PI_ERR_STATE: return "invalid state";
        default: return "unknown status";
    }
}

pi_status pi_last_error(pi_model* m, char* buf, size_t len) {
    const std::string& e = m ? m->err : g_create_error;
    if (buf && len) {
        size_t n = std::min(len - 1, e.size());
        memcpy(buf, e.c_str(), n);
        buf[n] = 0;
    }
    return PI_OK;
}

pi_status pi_create(const pi_grid* grid, const pi_bgc_params* bgc, const pi_quota_params* species,
                    int32_t nspecies, int64_t capacity, int32_t precision, uint64_t seed, pi_model** out) {
    if (!out) return fail(nullptr, PI_ERR_ARG, "pi_create: out is NULL");
    *out = nullptr;
    if (!grid || !bgc || !species || nspecies < 1 || capacity < 1 || !grid->dzF || !grid->dzC)
        return fail(nullptr, PI_ERR_ARG, "pi_create: NULL argument, nspecies < 1 or capacity < 1");
    if (precision != PI_FP64 && precision != PI_FP32)
        return fail(nullptr, PI_ERR_ARG, "pi_create: precision must be PI_FP64 or PI_FP32");
    if (grid->Nx < 1 || grid->Ny < 1 || grid->Nz < 1)
        return fail(nullptr, PI_ERR_ARG, "pi_create: grid size must be at least 1 in every direction");
    if (grid->Hx < 2 || grid->Hy < 2 || grid->Hz < 2 || grid->Hx > 8 || grid->Hy > 8 || grid->Hz > 8)
        return fail(nullptr, PI_ERR_ARG, "pi_create: halo must be 2..8 points (DST3FL needs at least 2)");
    for (int a = 0; a < 3; ++a)
        if (grid->topo[a] != PI_PERIODIC && grid->topo[a] != PI_BOUNDED)
            return fail(nullptr, PI_ERR_ARG, "pi_create: topology must be Periodic or Bounded");
    if (grid->topo[2] != PI_BOUNDED)
        return fail(nullptr, PI_ERR_ARG, "pi_create: z must be Bounded (tracer sinking has no Periodic rule)");
    long long Gx = grid->Nx + 2LL * grid->Hx, Gy = grid->Ny + 2LL * grid->Hy, Gz = grid->Nz + 2LL * grid->Hz;
    if (Gx * Gy * Gz >= (1LL << 31) - 2 || (Gx + 1) * (Gy + 1) * (Gz + 1) >= (1LL << 31))
        return fail(nullptr, PI_ERR_ARG, "pi_create: grid too large for 32-bit cell indices");
    if (const pi_grid_metrics* mt = grid->metrics) {
        if (precision != PI_FP64)
            return fail(nullptr, PI_ERR_ARG, "pi_create: LatLonGrid is built in the FP64 form only (precision PI_FP64)");
        if (!mt->dxC || !mt->dyC || !mt->dxF || !mt->dyF || !mt->Az || !mt->Ax || !mt->Ay || !mt->Vol)
            return fail(nullptr, PI_ERR_ARG, "pi_create: LatLonGrid metrics: every array is required");
    }
    if ((long long)nspecies * capacity >= (1LL << 31))
        return fail(nullptr, PI_ERR_ARG, "pi_create: nspecies × capacity must be below 2^31");
    for (int s = 0; s < nspecies; ++s) {
        std::string msg;
        pi_status st = validate_quota(species[s], s, msg);
        if (st) return fail(nullptr, st, msg);
    }
    if (precision == PI_FP32) {
        pi_member mb{grid, bgc, species, capacity, seed};
        pi_batch* b32 = nullptr;
        pi_status st = pi_batch_create(&mb, 1, nspecies, &b32);
        if (st) {
            char buf[1024];
            pi_batch_last_error(nullptr, buf, sizeof buf);
            std::string msg = buf;
            const std::string pre = "pi_batch_create: member 0: ";
            if (msg.compare(0, pre.size(), pre) == 0) msg = "pi_create: " + msg.substr(pre.size());
            return fail(nullptr, st, msg);
        }
        pi_model* m = new pi_model();
        m->b32 = b32;
        m->precision = PI_FP32;
        m->nsp = nspecies; m->C = capacity; m->seed = seed;
        m->bgc = *bgc;
        m->sp.assign(species, species + nspecies);
        *out = m;
        return PI_OK;
    }
    pi_model* m = new pi_model();
    if (cudaGetDevice(&m->device) != cudaSuccess) {
        delete m;
        return fail(nullptr, PI_ERR_CUDA, "pi_create: no CUDA device");
    }
    auto bail = [&](pi_status st) { g_create_error = m->err; free_all(m); if (m->stream) cudaStreamDestroy(m->stream); delete m; return st; };
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        m->err = "pi_create: stream creation failed"; return bail(PI_ERR_CUDA);
    }
    HostGrid& hg = m->hg;
    hg.Nx = grid->Nx; hg.Ny = grid->Ny; hg.Nz = grid->Nz; hg.Hx = grid->Hx; hg.Hy = grid->Hy; hg.Hz = grid->Hz;
    hg.Gx = (int)Gx; hg.Gy = (int)Gy; hg.Gz = (int)Gz;
    for (int a = 0; a < 3; ++a) hg.topo[a] = grid->topo[a];
    hg.dx = grid->dx; hg.dy = grid->dy;
    hg.dzF.assign(grid->dzF, grid->dzF + Gz);
    hg.dzC.assign(grid->dzC, grid->dzC + Gz);
    hg.G = Gx * Gy * Gz;
    hg.lm.assign(hg.G, 1);
    int all_water = 1;
    if (grid->landmask) {
        hg.lm.assign(grid->landmask, grid->landmask + hg.G);
        for (uint8_t v : hg.lm) if (v != 1) { all_water = 0; break; }
        for (uint8_t& v : hg.lm) v = v ? 1 : 0;
    }
    m->bgc = *bgc;
    m->sp.assign(species, species + nspecies);
    m->nsp = nspecies; m->C = capacity; m->seed = seed; m->precision = precision;
    const long long G = hg.G, C = capacity, NC = (long long)nspecies * capacity;
    pi_status st;
#define ALB(ptr, n) do { st = dalloc(m, &(ptr), (size_t)(n), #ptr); if (st) return bail(st); } while (0)
    ALB(m->dzF, Gz); ALB(m->dzC, Gz); ALB(m->lm, G);
    const long long G2 = Gx * Gy;
    if (const pi_grid_metrics* mt = grid->metrics) {
        ALB(m->met, 5 * G2 + 3 * G);
        m->met_host.resize((size_t)(5 * G2 + 3 * G));
        const double* a2[5] = { mt->dxC, mt->dyC, mt->dxF, mt->dyF, mt->Az };
        const double* a3[3] = { mt->Ax, mt->Ay, mt->Vol };
        for (int e = 0; e < 5; ++e) std::copy(a2[e], a2[e] + G2, m->met_host.begin() + e * G2);
        for (int e = 0; e < 3; ++e) std::copy(a3[e], a3[e] + G, m->met_host.begin() + 5 * G2 + e * G);
    }
    ALB(m->tr, PI_NTRACERS * G); ALB(m->tr_next, PI_NTRACERS * G);
    ALB(m->tta, PI_NTRACERS * G); ALB(m->ttb, PI_NTRACERS * G);
    for (int b = 0; b < 2; ++b) for (int c = 0; c < 3; ++c) ALB(m->velbuf[b][c], G);
    ALB(m->stage, 3 * G);
    for (int c = 0; c < 3; ++c) ALB(m->velh[c], G);
    ALB(m->zeros, G); ALB(m->par, G); ALB(m->PARF, (long long)hg.Nx * hg.Ny); ALB(m->temp_own, G);
    ALB(m->diag_par, G); ALB(m->diag_sp, 4LL * nspecies * G);
    StepBufs& sb = m->sb;
    ALB(sb.cnt, G + 1); ALB(sb.off, G + 1); ALB(sb.key, NC); ALB(sb.key_sorted, NC);
    ALB(sb.gid_sorted, NC); ALB(sb.pos, NC); ALB(sb.contrib, 5 * NC); ALB(sb.loss, 6 * NC);
    ALB(sb.evk, NC); ALB(sb.flag64, C); ALB(sb.rank64, C); ALB(sb.divlist, C); ALB(sb.freelist, C);
    ALB(sb.ndiv, 1); ALB(sb.err, 1); ALB(sb.err_iter, 1);
    ALB(m->iota, NC);
    ALB(m->d_bcs, PI_NTRACERS * 6);
    m->h_spc.resize(nspecies);
    for (int s = 0; s < nspecies; ++s) {
        SpcDev& P = m->h_spc[s];
        ALB(P.x, C); ALB(P.y, C); ALB(P.z, C); ALB(P.Sz, C); ALB(P.Bm, C); ALB(P.Cq, C); ALB(P.Nq, C);
        ALB(P.Pq, C); ALB(P.Chl, C); ALB(P.gen, C); ALB(P.age, C); ALB(P.flags, C); ALB(P.cell, C);
        ALB(P.stat, C); ALB(P.ptc, C);
    }
    ALB(m->d_spc, nspecies);
#undef ALB
    cudaStream_t s0 = m->stream;
    bool ok = true;
    ok = ok && cudaMemcpyAsync(m->dzF, hg.dzF.data(), Gz * sizeof(double), cudaMemcpyHostToDevice, s0) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(m->dzC, hg.dzC.data(), Gz * sizeof(double), cudaMemcpyHostToDevice, s0) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(m->lm, hg.lm.data(), G, cudaMemcpyHostToDevice, s0) == cudaSuccess;
    if (m->met)
        ok = ok && cudaMemcpyAsync(m->met, m->met_host.data(), m->met_host.size() * sizeof(double), cudaMemcpyHostToDevice, s0) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(m->d_spc, m->h_spc.data(), nspecies * sizeof(SpcDev), cudaMemcpyHostToDevice, s0) == cudaSuccess;
    for (void* p : { (void*)m->tr, (void*)m->tr_next, (void*)m->tta, (void*)m->ttb })
        ok = ok && cudaMemsetAsync(p, 0, PI_NTRACERS * G * sizeof(double), s0) == cudaSuccess;
    for (int b = 0; b < 2; ++b) for (int c = 0; c < 3; ++c)
        ok = ok && cudaMemsetAsync(m->velbuf[b][c], 0, G * sizeof(double), s0) == cudaSuccess;
    for (void* p : { (void*)m->zeros, (void*)m->par, (void*)m->temp_own, (void*)m->diag_par })
        ok = ok && cudaMemsetAsync(p, 0, G * sizeof(double), s0) == cudaSuccess;
    ok = ok && cudaMemsetAsync(m->PARF, 0, hg.Nx * (size_t)hg.Ny * sizeof(double), s0) == cudaSuccess;
    ok = ok && cudaMemsetAsync(m->diag_sp, 0, 4 * nspecies * G * sizeof(double), s0) == cudaSuccess;
    ok = ok && cudaMemsetAsync(sb.cnt, 0, (G + 1) * sizeof(uint32_t), s0) == cudaSuccess;
    ok = ok && cudaMemsetAsync(sb.off, 0, (G + 1) * sizeof(uint32_t), s0) == cudaSuccess;
    ok = ok && cudaMemsetAsync(sb.err, 0, sizeof(uint32_t), s0) == cudaSuccess;
    ok = ok && cudaMemsetAsync(sb.err_iter, 0, sizeof(int64_t), s0) == cudaSuccess;
    for (int s = 0; s < nspecies; ++s) {
        const SpcDev& P = m->h_spc[s];
        for (double* p : { P.x, P.y, P.z, P.Sz, P.Bm, P.Cq, P.Nq, P.Pq, P.Chl, P.gen, P.age, P.ptc })
            ok = ok && cudaMemsetAsync(p, 0, C * sizeof(double), s0) == cudaSuccess;
        ok = ok && cudaMemsetAsync(P.flags, 0, C, s0) == cudaSuccess;
        ok = ok && cudaMemsetAsync(P.stat, 0, C, s0) == cudaSuccess;
        ok = ok && cudaMemsetAsync(P.cell, 0, C * sizeof(int32_t), s0) == cudaSuccess;  // (0,0,0) as constructed
    }
    {
        std::vector<uint32_t> io(NC);
        for (long long q = 0; q < NC; ++q) io[q] = (uint32_t)q;
        ok = ok && cudaMemcpyAsync(m->iota, io.data(), NC * sizeof(uint32_t), cudaMemcpyHostToDevice, s0) == cudaSuccess;
        ok = ok && cudaStreamSynchronize(s0) == cudaSuccess;
    }
    if (!ok) { m->err = "pi_create: device initialisation failed"; return bail(PI_ERR_CUDA); }
    // vel₀ = vel₁ = 0 until set (timestepper.jl:24-26)
    for (int c = 0; c < 3; ++c) { m->vel0[c] = m->velbuf[0][c]; m->vel1[c] = m->velbuf[1][c]; }
    m->vel1_buf = 1;
    m->temp = m->temp_own;
    m->key_bits = 1;
    while ((1LL << m->key_bits) <= G) ++m->key_bits;
    // CUB scratch: the largest of the three uses
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b1, sb.cnt, sb.off, (int)(G + 1), s0);
    cub::DeviceRadixSort::SortPairs(nullptr, b2, sb.key, sb.key_sorted, m->iota, sb.gid_sorted, (int64_t)NC, 0, m->key_bits, s0);
    cub::DeviceScan::ExclusiveSum(nullptr, b3, sb.flag64, sb.rank64, (int64_t)C, s0);
    m->cub_bytes = std::max(b1, std::max(b2, b3));
    st = dalloc(m, (char**)&m->cub_tmp, m->cub_bytes, "cub scratch");
    if (st) return bail(st);
    m->dg = DGrid{hg.Nx, hg.Ny, hg.Nz, hg.Hx, hg.Hy, hg.Hz, hg.Gx, hg.Gy, hg.Gz,
                  hg.topo[0], hg.topo[1], hg.topo[2], all_water, hg.dx, hg.dy, m->dzF, m->dzC, m->lm, G,
                  nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (m->met) {
        double* b = m->met;
        m->dg.mdxC = b; m->dg.mdyC = b + G2; m->dg.mdxF = b + 2 * G2; m->dg.mdyF = b + 3 * G2; m->dg.mAz = b + 4 * G2;
        m->dg.mAx = b + 5 * G2; m->dg.mAy = b + 5 * G2 + G; m->dg.mVol = b + 5 * G2 + 2 * G;
    }
    st = upload_bcs(m);
    if (st) return bail(st);
    *out = m;
    return PI_OK;
}

pi_status pi_create_carbon(const pi_grid* grid, const pi_bgc_params* bgc, const pi_carbon_params* species,
                           int32_t nspecies, int64_t capacity, int32_t precision, uint64_t seed, pi_model** out) {
    if (!out) return fail(nullptr, PI_ERR_ARG, "pi_create_carbon: out is NULL");
    *out = nullptr;
    if (!species || nspecies < 1) return fail(nullptr, PI_ERR_ARG, "pi_create_carbon: NULL species or nspecies < 1");
    if (precision != PI_FP64)
        return fail(nullptr, PI_ERR_ARG, "pi_create_carbon: CarbonMode is built in the FP64 form only (precision PI_FP64)");
    // the QuotaMode setup with the parameters both modes share; the species then switch to CarbonMode
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
    pi_status st = pi_create(grid, bgc, q.data(), nspecies, capacity, PI_FP64, seed, out);
    if (st) return st;
    pi_model* m = *out;
    m->carbon = 1;
    m->cp.assign(species, species + nspecies);
    for (int s = 0; s < nspecies; ++s) {
        SpcDev& P = m->h_spc[s];
        if ((st = dalloc(m, &P.Bd, (size_t)capacity, "damaged biomass")) ||
            cudaMemsetAsync(P.Bd, 0, (size_t)capacity * sizeof(double), m->stream) != cudaSuccess) {
            pi_destroy(m); *out = nullptr;
            return fail(nullptr, st ? st : PI_ERR_CUDA, "pi_create_carbon: device allocation failed");
        }
    }
    if (cudaMemcpyAsync(m->d_spc, m->h_spc.data(), nspecies * sizeof(SpcDev), cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaStreamSynchronize(m->stream) != cudaSuccess) {
        pi_destroy(m); *out = nullptr;
        return fail(nullptr, PI_ERR_CUDA, "pi_create_carbon: device initialisation failed");
    }
    return PI_OK;
}

pi_status pi_create_iron(const pi_grid* grid, const pi_bgc_params* bgc, const pi_iron_params* species,
                         int32_t nspecies, int64_t capacity, int32_t precision, uint64_t seed, pi_model** out) {
    if (!out) return fail(nullptr, PI_ERR_ARG, "pi_create_iron: out is NULL");
    *out = nullptr;
    if (!species || nspecies < 1) return fail(nullptr, PI_ERR_ARG, "pi_create_iron: NULL species or nspecies < 1");
    if (precision != PI_FP64)
        return fail(nullptr, PI_ERR_ARG, "pi_create_iron: IronEnergyMode is built in the FP64 form only (precision PI_FP64)");
    // the QuotaMode setup with the parameters both modes share; the species then switch to IronEnergyMode
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
    pi_status st = pi_create(grid, bgc, q.data(), nspecies, capacity, PI_FP64, seed, out);
    if (st) return st;
    pi_model* m = *out;
    m->iron = 1;
    m->ipp.assign(species, species + nspecies);
    const long long NC = (long long)nspecies * capacity;
    bool ok = dalloc(m, &m->par0, (size_t)m->hg.G, "previous PAR") == PI_OK &&
              cudaMemsetAsync(m->par0, 0, (size_t)m->hg.G * sizeof(double), m->stream) == cudaSuccess &&
              dalloc(m, &m->sb.loss, (size_t)(10 * NC), "iron loss records") == PI_OK;     // ten tracers per record
    for (int s = 0; s < nspecies && ok; ++s) {
        SpcDev& P = m->h_spc[s];
        double** pools[10] = { &P.CH, &P.qNO3, &P.qNH4, &P.qP, &P.qFe, &P.qFePS, &P.qFeNR, &P.qFeNF, &P.exEn, &P.tdark };
        for (double** pp : pools)
            ok = ok && dalloc(m, pp, (size_t)capacity, "iron-energy pools") == PI_OK &&
                 cudaMemsetAsync(*pp, 0, (size_t)capacity * sizeof(double), m->stream) == cudaSuccess;
    }
    if (!ok || cudaMemcpyAsync(m->d_spc, m->h_spc.data(), nspecies * sizeof(SpcDev), cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaStreamSynchronize(m->stream) != cudaSuccess) {
        pi_destroy(m); *out = nullptr;
        return fail(nullptr, PI_ERR_CUDA, "pi_create_iron: device allocation or initialisation failed");
    }
    return PI_OK;
}

pi_status pi_create_macro(const pi_grid* grid, const pi_bgc_params* bgc, const pi_macro_params* species,
                          int32_t nspecies, int64_t capacity, int32_t precision, uint64_t seed, pi_model** out) {
    if (!out) return fail(nullptr, PI_ERR_ARG, "pi_create_macro: out is NULL");
    *out = nullptr;
    if (!species || nspecies < 1) return fail(nullptr, PI_ERR_ARG, "pi_create_macro: NULL species or nspecies < 1");
    if (precision != PI_FP64)
        return fail(nullptr, PI_ERR_ARG, "pi_create_macro: MacroMolecularMode is built in the FP64 form only (precision PI_FP64)");
    // the QuotaMode setup with the parameters both modes share; the species then switch to
    // MacroMolecularMode (dvid_type 1 only passes the shared validation, division is by DNA)
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
    pi_status st = pi_create(grid, bgc, q.data(), nspecies, capacity, PI_FP64, seed, out);
    if (st) return st;
    pi_model* m = *out;
    m->macro = 1;
    m->mp.assign(species, species + nspecies);
    for (int s = 0; s < nspecies; ++s) {
        SpcDev& P = m->h_spc[s];
        double** pools[6] = { &P.PRO, &P.DNA, &P.RNA, &P.CH, &P.NST, &P.PST };
        for (double** pp : pools)
            if ((st = dalloc(m, pp, (size_t)capacity, "macromolecular pools")) ||
                cudaMemsetAsync(*pp, 0, (size_t)capacity * sizeof(double), m->stream) != cudaSuccess) {
                pi_destroy(m); *out = nullptr;
                return fail(nullptr, st ? st : PI_ERR_CUDA, "pi_create_macro: device allocation failed");
            }
    }
    if (cudaMemcpyAsync(m->d_spc, m->h_spc.data(), nspecies * sizeof(SpcDev), cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
        cudaStreamSynchronize(m->stream) != cudaSuccess) {
        pi_destroy(m); *out = nullptr;
        return fail(nullptr, PI_ERR_CUDA, "pi_create_macro: device initialisation failed");
    }
    return PI_OK;
}

pi_status pi_destroy(pi_model* m) {
    if (!m) return PI_OK;
    if (m->b32) {
        pi_batch_destroy(m->b32);
        delete m;
        return PI_OK;
    }
    cudaStreamSynchronize(m->stream);
    drain_marks(m);
    for (cudaEvent_t e : m->event_pool) cudaEventDestroy(e);
    free_all(m);
    cudaStreamDestroy(m->stream);
    delete m;
    return PI_OK;
}

pi_status pi_set_individuals(pi_model* m, int32_t sp, const pi_individuals* in) {
    if (m && m->b32) return fwd32(m, pi_batch_set_individuals(m->b32, 0, sp, in));
    if (!m || !in || sp < 0 || sp >= m->nsp) return fail(m, PI_ERR_ARG, "pi_set_individuals: bad argument");
    const double* dcols[] = { in->x, in->y, in->z, in->Sz, in->Bm, in->Cq, in->Nq, in->Pq, in->Chl, in->gen, in->age,
                              in->graz, in->mort, in->dvid };
    const double* mcols[6] = { in->PRO, in->DNA, in->RNA, in->CH, in->NST, in->PST };
    for (int q = 0; q < 14; ++q) {
        // CarbonMode keeps no quotas; MacroMolecularMode no Sz, Bm or quotas, but its six pools
        const bool unused = ((m->carbon || m->iron) && q >= 5 && q <= 7) || (m->macro && q >= 3 && q <= 7);
        if (!dcols[q] && !unused) return fail(m, PI_ERR_ARG, "pi_set_individuals: NULL attribute");
    }
    if (m->macro)
        for (const double* c : mcols) if (!c) return fail(m, PI_ERR_ARG, "pi_set_individuals: NULL attribute");
    const double* icols[10] = { in->CH, in->qNO3, in->qNH4, in->qP, in->qFe, in->qFePS, in->qFeNR, in->qFeNF, in->exEn, in->tdark };
    if (m->iron)
        for (int q = 0; q < 8; ++q) if (!icols[q]) return fail(m, PI_ERR_ARG, "pi_set_individuals: NULL attribute");
    if (!in->xi || !in->yi || !in->zi || !in->ac) return fail(m, PI_ERR_ARG, "pi_set_individuals: NULL attribute");
    const long long C = m->C;
    const HostGrid& g = m->hg;
    std::vector<uint8_t> flags(C);
    std::vector<int32_t> cell(C);
    for (long long i = 0; i < C; ++i) {
        if (in->ac[i] > 1) return fail(m, PI_ERR_PARAM, "pi_set_individuals: ac must be 0 or 1");
        double d3[3] = { in->graz[i], in->mort[i], in->dvid[i] };
        for (double d : d3)
            if (d != 0.0 && d != 1.0) return fail(m, PI_ERR_PARAM, "pi_set_individuals: graz/mort/dvid must be 0 or 1");
        if (in->xi[i] < 0 || in->xi[i] > g.Gx || in->yi[i] < 0 || in->yi[i] > g.Gy || in->zi[i] < 0 || in->zi[i] > g.Gz)
            return fail(m, PI_ERR_PARAM, "pi_set_individuals: xi/yi/zi outside 0..G");
        flags[i] = (uint8_t)((in->ac[i] ? FL_AC : 0) | (in->graz[i] == 1.0 ? FL_GRAZ : 0) |
                             (in->mort[i] == 1.0 ? FL_MORT : 0) | (in->dvid[i] == 1.0 ? FL_DVID : 0));
        cell[i] = pack_cell(m->dg, (int)in->xi[i], (int)in->yi[i], (int)in->zi[i]);
    }
    const SpcDev& P = m->h_spc[sp];
    double* dptr[] = { P.x, P.y, P.z, P.Sz, P.Bm, P.Cq, P.Nq, P.Pq, P.Chl, P.gen, P.age };
    for (int q = 0; q < 11; ++q)
        if (dcols[q] && !(m->macro && q >= 3 && q <= 7))
            CK(cudaMemcpyAsync(dptr[q], dcols[q], C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload individuals");
    if (m->macro) {
        double* mptr[6] = { P.PRO, P.DNA, P.RNA, P.CH, P.NST, P.PST };
        for (int q = 0; q < 6; ++q)
            CK(cudaMemcpyAsync(mptr[q], mcols[q], C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload individuals");
    }
    if (m->carbon) {
        if (in->Bd) CK(cudaMemcpyAsync(P.Bd, in->Bd, C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload individuals");
        else CK(cudaMemsetAsync(P.Bd, 0, C * sizeof(double), m->stream), "upload individuals");
    }
    if (in->ptc) CK(cudaMemcpyAsync(P.ptc, in->ptc, C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload individuals");
    if (m->iron) {
        double* iptr[10] = { P.CH, P.qNO3, P.qNH4, P.qP, P.qFe, P.qFePS, P.qFeNR, P.qFeNF, P.exEn, P.tdark };
        for (int q = 0; q < 10; ++q) {
            if (icols[q]) CK(cudaMemcpyAsync(iptr[q], icols[q], C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload individuals");
            else CK(cudaMemsetAsync(iptr[q], 0, C * sizeof(double), m->stream), "upload individuals");   // exEn, tdark
        }
    }
    else CK(cudaMemsetAsync(P.ptc, 0, C * sizeof(double), m->stream), "upload individuals");
    CK(cudaMemcpyAsync(P.flags, flags.data(), C, cudaMemcpyHostToDevice, m->stream), "upload flags");
    CK(cudaMemcpyAsync(P.cell, cell.data(), C * sizeof(int32_t), cudaMemcpyHostToDevice, m->stream), "upload cells");
    CK(cudaMemsetAsync(P.stat, 0, C, m->stream), "reset step status");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

pi_status pi_get_individuals(pi_model* m, int32_t sp, pi_individuals* out) {
    if (m && m->b32) return fwd32(m, pi_batch_get_individuals(m->b32, 0, sp, out));
    if (!m || !out || sp < 0 || sp >= m->nsp) return fail(m, PI_ERR_ARG, "pi_get_individuals: bad argument");
    const long long C = m->C;
    const SpcDev& P = m->h_spc[sp];
    double* hptr[] = { out->x, out->y, out->z, out->Sz, out->Bm, out->Cq, out->Nq, out->Pq, out->Chl, out->gen, out->age };
    const double* dptr[] = { P.x, P.y, P.z, P.Sz, P.Bm, P.Cq, P.Nq, P.Pq, P.Chl, P.gen, P.age };
    for (int q = 0; q < 11; ++q)
        if (hptr[q]) CK(cudaMemcpyAsync(hptr[q], dptr[q], C * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download individuals");
    if (m->carbon && out->Bd) CK(cudaMemcpyAsync(out->Bd, P.Bd, C * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download individuals");
    if (out->ptc) CK(cudaMemcpyAsync(out->ptc, P.ptc, C * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download individuals");
    if (m->iron) {
        double* ih[10] = { out->CH, out->qNO3, out->qNH4, out->qP, out->qFe, out->qFePS, out->qFeNR, out->qFeNF, out->exEn, out->tdark };
        const double* id[10] = { P.CH, P.qNO3, P.qNH4, P.qP, P.qFe, P.qFePS, P.qFeNR, P.qFeNF, P.exEn, P.tdark };
        for (int q = 0; q < 10; ++q)
            if (ih[q]) CK(cudaMemcpyAsync(ih[q], id[q], C * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download individuals");
    }
    if (m->macro) {
        double* mh[6] = { out->PRO, out->DNA, out->RNA, out->CH, out->NST, out->PST };
        const double* md[6] = { P.PRO, P.DNA, P.RNA, P.CH, P.NST, P.PST };
        for (int q = 0; q < 6; ++q)
            if (mh[q]) CK(cudaMemcpyAsync(mh[q], md[q], C * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download individuals");
    }
    std::vector<uint8_t> flags(C);
    std::vector<int32_t> cell(C);
    CK(cudaMemcpyAsync(flags.data(), P.flags, C, cudaMemcpyDeviceToHost, m->stream), "download flags");
    CK(cudaMemcpyAsync(cell.data(), P.cell, C * sizeof(int32_t), cudaMemcpyDeviceToHost, m->stream), "download cells");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    for (long long i = 0; i < C; ++i) {
        uint8_t f = flags[i];
        if (out->ac) out->ac[i] = (f & FL_AC) ? 1 : 0;
        if (out->graz) out->graz[i] = (f & FL_GRAZ) ? 1.0 : 0.0;
        if (out->mort) out->mort[i] = (f & FL_MORT) ? 1.0 : 0.0;
        if (out->dvid) out->dvid[i] = (f & FL_DVID) ? 1.0 : 0.0;
        int xi, yi, zi;
        unpack_cell(m->dg, cell[i], xi, yi, zi);
        if (out->xi) out->xi[i] = xi;
        if (out->yi) out->yi[i] = yi;
        if (out->zi) out->zi[i] = zi;
    }
    return PI_OK;
}

pi_status pi_set_tracer(pi_model* m, int32_t idx, const double* data) {
    if (m && m->b32) return fwd32(m, pi_batch_set_tracer(m->b32, 0, idx, data));
    if (!m || !data || idx < 0 || idx >= PI_NTRACERS) return fail(m, PI_ERR_ARG, "pi_set_tracer: bad argument");
    CK(cudaMemcpyAsync(m->tr + (size_t)idx * m->hg.G, data, m->hg.G * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload tracer");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

pi_status pi_get_tracer(pi_model* m, int32_t idx, double* out) {
    if (m && m->b32) return fwd32(m, pi_batch_get_tracer(m->b32, 0, idx, out));
    if (!m || !out || idx < 0 || idx >= PI_NTRACERS) return fail(m, PI_ERR_ARG, "pi_get_tracer: bad argument");
    CK(cudaMemcpyAsync(out, m->tr + (size_t)idx * m->hg.G, m->hg.G * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download tracer");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

// vel_copy! on the device: interior arrays go to staging, then scatter + halo fill there. When an
// axis has fewer cells than halo points the reference's aliased halo copy reads stale values, so
// that case keeps the exact host-side fill.
static pi_status device_vel_copy(pi_model* m, const double* u, const double* v, const double* w,
                                 double* U, double* V, double* W) {
    const HostGrid& g = m->hg;
    const DGrid& dg = m->dg;
    cudaStream_t st = m->stream;
    int b[3] = { g.topo[0] == PI_BOUNDED, g.topo[1] == PI_BOUNDED, g.topo[2] == PI_BOUNDED };
    int dims[3][3] = { { g.Nx + b[0], g.Ny, g.Nz }, { g.Nx, g.Ny + b[1], g.Nz }, { g.Nx, g.Ny, g.Nz + b[2] } };
    const double* src[3] = { u, v, w };
    double* dst[3] = { U, V, W };
    for (int c = 0; c < 3; ++c) {
        size_t n = (size_t)dims[c][0] * dims[c][1] * dims[c][2];
        double* sg = m->stage + (size_t)c * g.G;
        CK(cudaMemcpyAsync(sg, src[c], n * sizeof(double), cudaMemcpyDefault, st), "upload velocity");
        k_scatter_interior<<<nblk((long long)n, 256), 256, 0, st>>>(dg, dst[c], sg, dims[c][0], dims[c][1], dims[c][2]);
        k_halo_vel<0><<<dim3(nblk(g.Gy, 64), g.Gz), 64, 0, st>>>(dg, dst[c], c);
        k_halo_vel<1><<<dim3(nblk(g.Gx, 64), g.Gz), 64, 0, st>>>(dg, dst[c], c);
        k_halo_vel<2><<<dim3(nblk(g.Gx, 64), g.Gy), 64, 0, st>>>(dg, dst[c], c);
        CK(cudaGetLastError(), "velocity halo");
    }
    return PI_OK;
}

pi_status pi_set_velocity(pi_model* m, const double* u, const double* v, const double* w) {
    if (m && m->b32) return fwd32(m, pi_batch_set_velocity(m->b32, 0, u, v, w));
    if (!m || !u || !v || !w) return fail(m, PI_ERR_ARG, "pi_set_velocity: NULL argument");
    // write into the own buffer that vel₀ does not alias
    int b = (m->vel0[0] == m->velbuf[0][0]) ? 1 : 0;
    const HostGrid& g = m->hg;
    if (g.Nx >= g.Hx && g.Ny >= g.Hy && g.Nz >= g.Hz) {
        pi_status st = device_vel_copy(m, u, v, w, m->velbuf[b][0], m->velbuf[b][1], m->velbuf[b][2]);
        if (st) return st;
    } else {
        std::vector<double> U, V, W;
        host_vel_copy(g, u, v, w, U, V, W);
        const size_t bytes = g.G * sizeof(double);
        CK(cudaMemcpyAsync(m->velbuf[b][0], U.data(), bytes, cudaMemcpyHostToDevice, m->stream), "upload u");
        CK(cudaMemcpyAsync(m->velbuf[b][1], V.data(), bytes, cudaMemcpyHostToDevice, m->stream), "upload v");
        CK(cudaMemcpyAsync(m->velbuf[b][2], W.data(), bytes, cudaMemcpyHostToDevice, m->stream), "upload w");
    }
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    for (int c = 0; c < 3; ++c) m->vel1[c] = m->velbuf[b][c];
    m->vel1_buf = b;
    return PI_OK;
}

pi_status pi_set_velocity0(pi_model* m, const double* u, const double* v, const double* w) {
    if (m && m->b32) return fwd32(m, pi_batch_set_velocity0(m->b32, 0, u, v, w));
    if (!m || !u || !v || !w) return fail(m, PI_ERR_ARG, "pi_set_velocity0: NULL argument");
    // write into the own buffer that vel₁ does not alias
    int b = (m->vel1[0] == m->velbuf[0][0]) ? 1 : 0;
    const HostGrid& g = m->hg;
    if (g.Nx >= g.Hx && g.Ny >= g.Hy && g.Nz >= g.Hz) {
        pi_status st = device_vel_copy(m, u, v, w, m->velbuf[b][0], m->velbuf[b][1], m->velbuf[b][2]);
        if (st) return st;
    } else {
        std::vector<double> U, V, W;
        host_vel_copy(g, u, v, w, U, V, W);
        const size_t bytes = g.G * sizeof(double);
        CK(cudaMemcpyAsync(m->velbuf[b][0], U.data(), bytes, cudaMemcpyHostToDevice, m->stream), "upload u");
        CK(cudaMemcpyAsync(m->velbuf[b][1], V.data(), bytes, cudaMemcpyHostToDevice, m->stream), "upload v");
        CK(cudaMemcpyAsync(m->velbuf[b][2], W.data(), bytes, cudaMemcpyHostToDevice, m->stream), "upload w");
    }
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    for (int c = 0; c < 3; ++c) m->vel0[c] = m->velbuf[b][c];
    return PI_OK;
}

pi_status pi_set_PARF(pi_model* m, const double* parf) {
    if (m && m->b32) return fwd32(m, pi_batch_set_PARF(m->b32, 0, parf));
    if (!m || !parf) return fail(m, PI_ERR_ARG, "pi_set_PARF: NULL argument");
    CK(cudaMemcpyAsync(m->PARF, parf, (size_t)m->hg.Nx * m->hg.Ny * sizeof(double), cudaMemcpyDefault, m->stream), "upload PARF");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

pi_status pi_set_temp(pi_model* m, const double* temp) {
    if (m && m->b32) return fwd32(m, pi_batch_set_temp(m->b32, 0, temp));
    if (!m || !temp) return fail(m, PI_ERR_ARG, "pi_set_temp: NULL argument");
    const HostGrid& g = m->hg;
    size_t n = (size_t)g.Nx * g.Ny * g.Nz;
    // copy_interior!: only the interior is written; the halo of timestepper.temp stays zero
    CK(cudaMemcpyAsync(m->stage, temp, n * sizeof(double), cudaMemcpyDefault, m->stream), "upload temp");
    k_scatter_interior<<<nblk((long long)n, 256), 256, 0, m->stream>>>(m->dg, m->temp_own, m->stage, g.Nx, g.Ny, g.Nz);
    CK(cudaGetLastError(), "scatter temp");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    m->temp = m->temp_own;
    return PI_OK;
}

pi_status pi_set_flux_bc(pi_model* m, int32_t tracer, int32_t face, int32_t kind, const double* values, int64_t nt) {
    if (m && m->b32) return fwd32(m, pi_batch_set_flux_bc(m->b32, 0, tracer, face, kind, values, nt));
    if (!m || tracer < 0 || tracer >= PI_NTRACERS || face < 0 || face > 5 || kind < 0 || kind > 3)
        return fail(m, PI_ERR_ARG, "pi_set_flux_bc: bad argument");
    const HostGrid& g = m->hg;
    size_t n1 = face <= PI_EAST ? g.Ny : g.Nx, n2 = face <= PI_NORTH ? g.Nz : g.Ny;
    size_t n = kind == PI_BC_CONST ? 1 : kind == PI_BC_ARRAY2D ? n1 * n2 : kind == PI_BC_ARRAY3D ? n1 * n2 * (size_t)std::max<int64_t>(nt, 0) : 0;
    if (kind == PI_BC_ARRAY3D && nt < 1) return fail(m, PI_ERR_SHAPE, "BC: time-dependent flux needs nt >= 1");
    if (n && !values) return fail(m, PI_ERR_ARG, "pi_set_flux_bc: NULL values");
    DevBC& b = m->bcs[tracer][face];
    if (b.v) { cudaFree(b.v); b.v = nullptr; }
    b.kind = kind; b.nt = nt;
    if (n) {
        CK(cudaMalloc(&b.v, n * sizeof(double)), "bc values");
        CK(cudaMemcpyAsync(b.v, values, n * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload bc");
    }
    return upload_bcs(m);
}

pi_status pi_set_abiotics(pi_model* m, int32_t nsa, const pi_abiotic_params* params, int32_t n_intac, const int32_t* intac,
                          int32_t n_release, const int32_t* release, int32_t max_candidates, const double* max_ptc) {
    if (m && m->b32) return fail(m, PI_ERR_ARG, "pi_set_abiotics: abiotic particles are built in the FP64 form only");
    if (!m || nsa < 1 || !params || max_candidates < 1 || !max_ptc || n_intac < 0 || n_release < 0 ||
        (n_intac && !intac) || (n_release && !release))
        return fail(m, PI_ERR_ARG, "pi_set_abiotics: bad argument");
    if (m->nsa) return fail(m, PI_ERR_STATE, "pi_set_abiotics: the model already has abiotic particles");
    for (int32_t q = 0; q < n_intac + n_release; ++q) {       // models.jl:127-142
        const int32_t* pr = q < n_intac ? intac + 2 * q : release + 2 * (q - n_intac);
        if (pr[0] < 0 || pr[0] >= m->nsp) return fail(m, PI_ERR_ARG, "Abiotic: sp" + std::to_string(pr[0] + 1) + " is not generated");
        if (pr[1] < 0 || pr[1] >= nsa) return fail(m, PI_ERR_ARG, "Abiotic: sa" + std::to_string(pr[1] + 1) + " is not generated");
    }
    const long long C = m->C, G = m->hg.G;
    if ((double)max_candidates * (double)C > 9.0e18) return fail(m, PI_ERR_ARG, "pi_set_abiotics: max_candidates too large");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    pi_status e;
    std::vector<AbioDev> ab((size_t)nsa);
    for (AbioDev& A : ab) {
        if ((e = dalloc(m, &A.x, C, "abiotic particles")) || (e = dalloc(m, &A.y, C, "abiotic particles")) ||
            (e = dalloc(m, &A.z, C, "abiotic particles")) || (e = dalloc(m, &A.ac, C, "abiotic particles")) ||
            (e = dalloc(m, &A.cell, C, "abiotic particles")))
            return e;
        for (double* p : { A.x, A.y, A.z }) CK(cudaMemsetAsync(p, 0, C * sizeof(double), m->stream), "zero abiotic particles");
        CK(cudaMemsetAsync(A.ac, 0, C, m->stream), "zero abiotic particles");
        CK(cudaMemsetAsync(A.cell, 0, C * sizeof(int32_t), m->stream), "zero abiotic particles");   // (0, 0, 0) as constructed
    }
    if ((e = dalloc(m, &m->intac, (size_t)max_candidates * C, "interaction candidates")) ||
        (e = dalloc(m, &m->diag_ptc, (size_t)m->nsp * G, "ptc diagnostics")) ||
        (e = dalloc(m, &m->diag_abn, (size_t)nsa * G, "abiotic diagnostics")) ||
        (e = dalloc(m, &m->cflag, G, "boundary cells")) || (e = dalloc(m, &m->crank, G, "boundary cells")) ||
        (e = dalloc(m, &m->afl, C, "free particle slots")) || (e = dalloc(m, &m->afr, C, "free particle slots")) ||
        (e = dalloc(m, &m->afree, C, "free particle slots")))
        return e;
    for (uint32_t** p : { &m->akey, &m->akey_s, &m->aval, &m->aval_s, &m->pkey, &m->pkey_s, &m->pval, &m->pval_s })
        if ((e = dalloc(m, p, (size_t)C, "cell binning"))) return e;
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, m->akey, m->akey_s, m->aval, m->aval_s, (int64_t)C, 0, m->key_bits, m->stream);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, m->cflag, m->crank, (int)G, m->stream);
    cub::DeviceScan::ExclusiveSum(nullptr, b3, m->afl, m->afr, (int)C, m->stream);
    m->abytes = std::max(b1, std::max(b2, b3));
    unsigned char* tmp = nullptr;
    if ((e = dalloc(m, &tmp, std::max<size_t>(m->abytes, 1), "abiotic scratch"))) return e;
    m->atmp = tmp;
    CK(cudaMemsetAsync(m->diag_ptc, 0, (size_t)m->nsp * G * sizeof(double), m->stream), "zero diagnostics");
    CK(cudaMemsetAsync(m->diag_abn, 0, (size_t)nsa * G * sizeof(double), m->stream), "zero diagnostics");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    m->h_ab = ab;
    m->ap.assign(params, params + nsa);
    m->abc.assign((size_t)nsa * 6, DevBC{});
    for (int32_t q = 0; q < n_intac; ++q) m->pal_intac.emplace_back(intac[2 * q], intac[2 * q + 1]);
    for (int32_t q = 0; q < n_release; ++q) m->pal_release.emplace_back(release[2 * q], release[2 * q + 1]);
    m->maxc = max_candidates;
    m->max_ptc.assign(max_ptc, max_ptc + m->nsp);
    m->nsa = nsa;
    return PI_OK;
}

pi_status pi_set_abiotic_particles(pi_model* m, int32_t sa, const pi_abiotic_particles* in) {
    if (!m || sa < 0 || sa >= m->nsa || !in || !in->x || !in->y || !in->z || !in->ac)
        return fail(m, PI_ERR_ARG, "pi_set_abiotic_particles: bad argument");
    const long long C = m->C;
    const HostGrid& g = m->hg;
    std::vector<int32_t> cell((size_t)C);
    for (long long k = 0; k < C; ++k) {
        if (in->ac[k] > 1) return fail(m, PI_ERR_PARAM, "pi_set_abiotic_particles: ac must be 0 or 1");
        const int64_t xi = in->xi ? in->xi[k] : 0, yi = in->yi ? in->yi[k] : 0, zi = in->zi ? in->zi[k] : 0;
        if (xi < 0 || xi > g.Gx || yi < 0 || yi > g.Gy || zi < 0 || zi > g.Gz)
            return fail(m, PI_ERR_PARAM, "pi_set_abiotic_particles: xi/yi/zi outside 0..G");
        cell[k] = pack_cell(m->dg, (int)xi, (int)yi, (int)zi);
    }
    const AbioDev& A = m->h_ab[sa];
    CK(cudaMemcpyAsync(A.x, in->x, C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload abiotic particles");
    CK(cudaMemcpyAsync(A.y, in->y, C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload abiotic particles");
    CK(cudaMemcpyAsync(A.z, in->z, C * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload abiotic particles");
    CK(cudaMemcpyAsync(A.ac, in->ac, C, cudaMemcpyHostToDevice, m->stream), "upload abiotic particles");
    CK(cudaMemcpyAsync(A.cell, cell.data(), C * sizeof(int32_t), cudaMemcpyHostToDevice, m->stream), "upload abiotic particles");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

pi_status pi_get_abiotic_particles(pi_model* m, int32_t sa, pi_abiotic_particles* out) {
    if (!m || sa < 0 || sa >= m->nsa || !out) return fail(m, PI_ERR_ARG, "pi_get_abiotic_particles: bad argument");
    const long long C = m->C;
    const AbioDev& A = m->h_ab[sa];
    double* hp[3] = { out->x, out->y, out->z };
    const double* dp[3] = { A.x, A.y, A.z };
    for (int q = 0; q < 3; ++q)
        if (hp[q]) CK(cudaMemcpyAsync(hp[q], dp[q], C * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download abiotic particles");
    if (out->ac) CK(cudaMemcpyAsync(out->ac, A.ac, C, cudaMemcpyDeviceToHost, m->stream), "download abiotic particles");
    std::vector<int32_t> cell((size_t)C);
    CK(cudaMemcpyAsync(cell.data(), A.cell, C * sizeof(int32_t), cudaMemcpyDeviceToHost, m->stream), "download abiotic particles");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    for (long long k = 0; k < C; ++k) {
        int xi, yi, zi;
        unpack_cell(m->dg, cell[k], xi, yi, zi);
        if (out->xi) out->xi[k] = xi;
        if (out->yi) out->yi[k] = yi;
        if (out->zi) out->zi[k] = zi;
    }
    return PI_OK;
}

pi_status pi_count_abiotic(pi_model* m, int32_t sa, int64_t* n) {
    if (!m || !n || sa < 0 || sa >= m->nsa) return fail(m, PI_ERR_ARG, "pi_count_abiotic: bad argument");
    unsigned long long* d = (unsigned long long*)m->sb.rank64;   // scratch between steps
    unsigned long long h = 0;
    CK(cudaMemsetAsync(d, 0, sizeof h, m->stream), "zero count");
    k_count_active<<<148 * 2, 256, 0, m->stream>>>(m->h_ab[sa].ac, m->C, d);
    CK(cudaGetLastError(), "k_count_active");
    CK(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, m->stream), "download count");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    *n = (int64_t)h;
    return PI_OK;
}

pi_status pi_set_abiotic_bc(pi_model* m, int32_t sa, int32_t face, int32_t kind, const double* values, int64_t nt) {
    if (!m || sa < 0 || sa >= m->nsa || face < 0 || face > 5 || kind < 0 || kind > 3)
        return fail(m, PI_ERR_ARG, "pi_set_abiotic_bc: bad argument");
    const HostGrid& g = m->hg;
    size_t n1 = face <= PI_EAST ? g.Ny : g.Nx, n2 = face <= PI_NORTH ? g.Nz : g.Ny;
    size_t n = kind == PI_BC_CONST ? 1 : kind == PI_BC_ARRAY2D ? n1 * n2 : kind == PI_BC_ARRAY3D ? n1 * n2 * (size_t)std::max<int64_t>(nt, 0) : 0;
    if (kind == PI_BC_ARRAY3D && nt < 1) return fail(m, PI_ERR_SHAPE, "BC: time-dependent flux needs nt >= 1");
    if (n && !values) return fail(m, PI_ERR_ARG, "pi_set_abiotic_bc: NULL values");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    DevBC& b = m->abc[(size_t)sa * 6 + face];
    if (b.v) { cudaFree(b.v); b.v = nullptr; }
    b.kind = kind; b.nt = nt;
    if (n) {
        CK(cudaMalloc(&b.v, n * sizeof(double)), "bc values");
        CK(cudaMemcpyAsync(b.v, values, n * sizeof(double), cudaMemcpyHostToDevice, m->stream), "upload bc");
        CK(cudaStreamSynchronize(m->stream), "synchronize");
    }
    return PI_OK;
}

pi_status pi_time_step(pi_model* m, double dT) {
    if (m && m->b32) return fwd32(m, pi_batch_step(m->b32, dT, 1, 1));
    if (!m) return fail(m, PI_ERR_ARG, "pi_time_step: NULL model");
    pi_status st = enqueue_step(m, dT);
    if (st) return st;
    return check_device_errors(m);
}

pi_status pi_time_step_async(pi_model* m, double dT) {
    if (m && m->b32) return fwd32(m, pi_batch_step(m->b32, dT, 1, 0));
    if (!m) return fail(m, PI_ERR_ARG, "pi_time_step_async: NULL model");
    return enqueue_step(m, dT);
}

pi_status pi_set_velocity_f32(pi_model* m, const float* u, const float* v, const float* w) {
    if (m && m->b32) return fwd32(m, pi_batch_set_velocity_f32(m->b32, 0, u, v, w));
    return fail(m, PI_ERR_ARG, "pi_set_velocity_f32: Float32 forcing is for a PI_FP32 model");
}
pi_status pi_set_PARF_f32(pi_model* m, const float* parf) {
    if (m && m->b32) return fwd32(m, pi_batch_set_PARF_f32(m->b32, 0, parf));
    return fail(m, PI_ERR_ARG, "pi_set_PARF_f32: Float32 forcing is for a PI_FP32 model");
}
pi_status pi_set_temp_f32(pi_model* m, const float* temp) {
    if (m && m->b32) return fwd32(m, pi_batch_set_temp_f32(m->b32, 0, temp));
    return fail(m, PI_ERR_ARG, "pi_set_temp_f32: Float32 forcing is for a PI_FP32 model");
}

pi_status pi_get_stream(pi_model* m, void** stream) {
    if (m && m->b32) return fwd32(m, pi_batch_get_stream(m->b32, stream));
    if (!m || !stream) return fail(m, PI_ERR_ARG, "pi_get_stream: NULL argument");
    *stream = (void*)m->stream;
    return PI_OK;
}

pi_status pi_profile_enable(pi_model* m, int32_t on) {
    if (m && m->b32) return fwd32(m, pi_batch_profile_enable(m->b32, on));
    if (!m) return fail(m, PI_ERR_ARG, "pi_profile_enable: NULL model");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    drain_marks(m);
    m->prof_names.clear(); m->prof_count.clear(); m->prof_ms.clear();
    m->profiling = on ? 1 : 0;
    return PI_OK;
}

pi_status pi_profile_read(pi_model* m, int32_t max, char* names, size_t names_len,
                          int64_t* launches, double* ms, int32_t* n) {
    if (m && m->b32) return fwd32(m, pi_batch_profile_read(m->b32, max, names, names_len, launches, ms, n));
    if (!m || !n) return fail(m, PI_ERR_ARG, "pi_profile_read: NULL argument");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    drain_marks(m);
    int32_t k = (int32_t)m->prof_names.size();
    *n = k;
    size_t off = 0;
    for (int32_t q = 0; q < k && q < max; ++q) {
        if (launches) launches[q] = m->prof_count[q];
        if (ms) ms[q] = m->prof_ms[q];
        if (names) {
            const std::string& nm = m->prof_names[q];
            if (off + nm.size() + 1 <= names_len) { memcpy(names + off, nm.c_str(), nm.size() + 1); off += nm.size() + 1; }
        }
    }
    return PI_OK;
}

pi_status pi_synchronize(pi_model* m) {
    if (m && m->b32) return fwd32(m, pi_batch_synchronize(m->b32));
    if (!m) return fail(m, PI_ERR_ARG, "pi_synchronize: NULL model");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return check_device_errors(m);
}

pi_status pi_get_time(pi_model* m, int64_t* iteration, double* t) {
    if (m && m->b32) return fwd32(m, pi_batch_get_time(m->b32, iteration, t));
    if (!m) return fail(m, PI_ERR_ARG, "pi_get_time: NULL model");
    if (iteration) *iteration = m->iteration;
    if (t) *t = m->t;
    return PI_OK;
}

pi_status pi_set_time(pi_model* m, int64_t iteration, double t) {
    if (m && m->b32) return fwd32(m, pi_batch_set_time(m->b32, iteration, t));
    if (!m) return fail(m, PI_ERR_ARG, "pi_set_time: NULL model");
    m->iteration = iteration; m->t = t;
    return PI_OK;
}

pi_status pi_count_active(pi_model* m, int32_t sp, int64_t* n) {
    if (m && m->b32) {
        if (sp < 0 || sp >= m->nsp) return fail(m, PI_ERR_ARG, "pi_count_active: bad argument");
        return fwd32(m, pi_batch_count_active(m->b32, 0, sp, n));
    }
    if (!m || !n || sp < 0 || sp >= m->nsp) return fail(m, PI_ERR_ARG, "pi_count_active: bad argument");
    unsigned long long* d = (unsigned long long*)m->sb.rank64;   // scratch between steps
    unsigned long long h = 0;
    CK(cudaMemsetAsync(d, 0, sizeof h, m->stream), "zero count");
    k_count_active<<<148 * 2, 256, 0, m->stream>>>(m->h_spc[sp].flags, m->C, d);
    CK(cudaGetLastError(), "k_count_active");
    CK(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, m->stream), "download count");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    *n = (int64_t)h;
    return PI_OK;
}

pi_status pi_check_finite(pi_model* m) {
    if (m && m->b32) return fwd32(m, pi_batch_check_finite(m->b32, 0));
    if (!m) return fail(m, PI_ERR_ARG, "pi_check_finite: NULL model");
    unsigned long long* d = (unsigned long long*)m->sb.rank64;   // scratch between steps
    const unsigned long long none = ~0ull;
    const long long G = m->hg.G;
    auto first = [&](auto launch, unsigned long long& out) -> pi_status {
        CK(cudaMemcpyAsync(d, &none, sizeof none, cudaMemcpyHostToDevice, m->stream), "check finite");
        launch();
        CK(cudaGetLastError(), "check finite");
        CK(cudaMemcpyAsync(&out, d, sizeof out, cudaMemcpyDeviceToHost, m->stream), "check finite");
        CK(cudaStreamSynchronize(m->stream), "synchronize");
        return PI_OK;
    };
    unsigned long long q = none;
    pi_status e = first([&] { k_first_nonfinite<<<148 * 4, 256, 0, m->stream>>>(m->tr, PI_NTRACERS * G, d); }, q);
    if (e) return e;
    if (q != none) {
        const long long n = (long long)q / G, c = (long long)q % G;
        const long long i = c % m->hg.Gx + 1, j = (c / m->hg.Gx) % m->hg.Gy + 1, k = c / ((long long)m->hg.Gx * m->hg.Gy) + 1;
        return fail(m, PI_ERR_NAN, "NaN or Inf in tracer " + std::string(tracer_name((int)n)) + " at (" + std::to_string(i) + ", " +
                                       std::to_string(j) + ", " + std::to_string(k) + ")");
    }
    for (int s = 0; s < m->nsp; ++s) {
        e = first([&] { k_first_nonfinite_inds<<<148 * 2, 256, 0, m->stream>>>(m->h_spc[s], m->C, d); }, q);
        if (e) return e;
        if (q != none)
            return fail(m, PI_ERR_NAN, "NaN or Inf in an attribute of individual " + std::to_string(q + 1) + " of species " + std::to_string(s + 1));
    }
    return PI_OK;
}

pi_status pi_count_active_async(pi_model* m, int32_t sp, int64_t* n) {
    if (m && m->b32) {
        if (sp < 0 || sp >= m->nsp) return fail(m, PI_ERR_ARG, "pi_count_active_async: bad argument");
        return fwd32(m, pi_batch_count_active_async(m->b32, 0, sp, n));
    }
    if (!m || !n || sp < 0 || sp >= m->nsp) return fail(m, PI_ERR_ARG, "pi_count_active_async: bad argument");
    unsigned long long* d = (unsigned long long*)m->sb.rank64;   // scratch between steps, stream-ordered
    CK(cudaMemsetAsync(d, 0, sizeof *d, m->stream), "zero count");
    k_count_active<<<148 * 2, 256, 0, m->stream>>>(m->h_spc[sp].flags, m->C, d);
    CK(cudaGetLastError(), "k_count_active");
    CK(cudaMemcpyAsync(n, d, sizeof *d, cudaMemcpyDeviceToHost, m->stream), "download count");
    return PI_OK;
}

pi_status pi_set_diags(pi_model* m, uint32_t tracer_mask, uint32_t proc_mask) {
    if (m && m->b32) return fwd32(m, pi_batch_set_diags(m->b32, tracer_mask, proc_mask));
    const int nproc = !m ? 0 : m->iron ? (int)PI_NIPROC : m->macro ? (int)PI_NMPROC : m->carbon ? (int)PI_NCPROC : (int)PI_NPROC;
    if (!m || tracer_mask >> PI_NTRACERS || (nproc < 32 && proc_mask >> nproc))
        return fail(m, PI_ERR_ARG, "pi_set_diags: bad argument");
    const long long G = m->hg.G, C = m->C;
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    if (tracer_mask && !m->diag_tr) { pi_status e = dalloc(m, &m->diag_tr, (size_t)PI_NTRACERS * G, "tracer diagnostics"); if (e) return e; }
    if (proc_mask && !m->diag_proc) {
        pi_status e;
        if ((e = dalloc(m, &m->diag_proc, (size_t)m->nsp * PI_MAXPROC * G, "process diagnostics"))) return e;
        if ((e = dalloc(m, &m->procv, (size_t)PI_MAXPROC * C, "process values"))) return e;
        for (uint32_t** p : { &m->dkey, &m->dkey_s, &m->dval, &m->dval_s })
            if ((e = dalloc(m, p, (size_t)C, "diagnostic sort"))) return e;
        size_t db = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, db, m->dkey, m->dkey_s, m->dval, m->dval_s, (int64_t)C, 0, m->key_bits, m->stream);
        unsigned char* tmp = nullptr;
        if ((e = dalloc(m, &tmp, std::max<size_t>(db, 1), "diagnostic sort"))) return e;
        m->dsort_tmp = tmp; m->dsort_bytes = db;
    }
    if (m->diag_tr) CK(cudaMemsetAsync(m->diag_tr, 0, (size_t)PI_NTRACERS * G * sizeof(double), m->stream), "clear diagnostics");
    if (m->diag_proc) CK(cudaMemsetAsync(m->diag_proc, 0, (size_t)m->nsp * PI_MAXPROC * G * sizeof(double), m->stream), "clear diagnostics");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    m->tr_mask = tracer_mask; m->proc_mask = proc_mask;
    return PI_OK;
}

pi_status pi_get_diag(pi_model* m, int32_t kind, int32_t sp, double* out) {
    if (m && m->b32) return fwd32(m, pi_batch_get_diag(m->b32, 0, kind, sp, out));
    if (!m || !out) return fail(m, PI_ERR_ARG, "pi_get_diag: bad argument");
    const long long G = m->hg.G;
    const double* src = nullptr;
    if (kind == PI_DIAG_PAR) src = m->diag_par;
    else if (kind >= PI_DIAG_TRACER && kind < PI_DIAG_TRACER + PI_NTRACERS) {
        if (!(m->tr_mask >> (kind - PI_DIAG_TRACER) & 1u)) return fail(m, PI_ERR_ARG, "pi_get_diag: tracer diagnostic not enabled");
        src = m->diag_tr + (size_t)(kind - PI_DIAG_TRACER) * G;
    } else if (kind >= PI_DIAG_PROC && kind < PI_DIAG_PROC + PI_MAXPROC) {
        if (sp < 0 || sp >= m->nsp || !(m->proc_mask >> (kind - PI_DIAG_PROC) & 1u))
            return fail(m, PI_ERR_ARG, "pi_get_diag: process diagnostic not enabled or bad species");
        src = m->diag_proc + ((size_t)sp * PI_MAXPROC + (kind - PI_DIAG_PROC)) * G;
    } else if (kind == PI_DIAG_PTC || kind == PI_DIAG_ABIO_NUM) {
        const int n = kind == PI_DIAG_PTC ? m->nsp : m->nsa;
        if (sp < 0 || sp >= n || !m->nsa) return fail(m, PI_ERR_ARG, "pi_get_diag: no abiotic particles or bad species");
        src = (kind == PI_DIAG_PTC ? m->diag_ptc : m->diag_abn) + (size_t)sp * G;
    } else {
        if (sp < 0 || sp >= m->nsp || kind < PI_DIAG_NUM || kind > PI_DIAG_DVID) return fail(m, PI_ERR_ARG, "pi_get_diag: bad kind/species");
        src = m->diag_sp + ((size_t)sp * 4 + (kind - PI_DIAG_NUM)) * G;
    }
    CK(cudaMemcpyAsync(out, src, G * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download diag");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

pi_status pi_get_budget(pi_model* m, double out[6]) {
    if (m && m->b32) return fwd32(m, pi_batch_budget(m->b32, 0, out));
    if (!m || !out) return fail(m, PI_ERR_ARG, "pi_get_budget: NULL argument");
    const int nb = 512;
    if (!m->budget_part) { pi_status e = dalloc(m, &m->budget_part, 3 * nb, "budget partials"); if (e) return e; }
    std::vector<double> h(3 * nb);
    auto collect = [&](double* dst) -> pi_status {
        CK(cudaGetLastError(), "budget");
        CK(cudaMemcpyAsync(h.data(), m->budget_part, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download budget");
        CK(cudaStreamSynchronize(m->stream), "synchronize");
        for (int r = 0; r < 3; ++r) { double x = 0.0; for (int q = 0; q < nb; ++q) x += h[q * 3 + r]; dst[r] += x; }
        return PI_OK;
    };
    for (int r = 0; r < 6; ++r) out[r] = 0.0;
    k_budget_cells<<<nb, 256, 0, m->stream>>>(m->dg, m->tr, m->budget_part);
    pi_status e = collect(out);
    if (e) return e;
    for (int s = 0; s < m->nsp; ++s) {
        if (m->iron) k_budget_inds_iron<<<nb, 256, 0, m->stream>>>(m->h_spc[s], m->C, m->ipp[s].R_NC, m->ipp[s].R_PC, m->budget_part);
        else if (m->macro) k_budget_inds_macro<<<nb, 256, 0, m->stream>>>(m->h_spc[s], m->C, m->mp[s], m->budget_part);
        else k_budget_inds<<<nb, 256, 0, m->stream>>>(m->h_spc[s], m->C, m->sp[s].R_NC, m->sp[s].R_PC, m->budget_part);
        if ((e = collect(out + 3))) return e;
    }
    return PI_OK;
}

pi_status pi_reset_diags(pi_model* m) {
    if (m && m->b32) return fwd32(m, pi_batch_reset_diags(m->b32));
    if (!m) return fail(m, PI_ERR_ARG, "pi_reset_diags: NULL model");
    const long long G = m->hg.G;
    CK(cudaMemsetAsync(m->diag_par, 0, G * sizeof(double), m->stream), "reset diags");
    CK(cudaMemsetAsync(m->diag_sp, 0, 4 * m->nsp * G * sizeof(double), m->stream), "reset diags");
    if (m->diag_tr) CK(cudaMemsetAsync(m->diag_tr, 0, (size_t)PI_NTRACERS * G * sizeof(double), m->stream), "reset diags");
    if (m->diag_proc) CK(cudaMemsetAsync(m->diag_proc, 0, (size_t)m->nsp * PI_MAXPROC * G * sizeof(double), m->stream), "reset diags");
    if (m->diag_ptc) CK(cudaMemsetAsync(m->diag_ptc, 0, (size_t)m->nsp * G * sizeof(double), m->stream), "reset diags");
    if (m->diag_abn) CK(cudaMemsetAsync(m->diag_abn, 0, (size_t)m->nsa * G * sizeof(double), m->stream), "reset diags");
    CK(cudaStreamSynchronize(m->stream), "synchronize");
    return PI_OK;
}

// ---- PlanktonSimulation / update! -------------------------------------------------------------

pi_status pi_sim_create(pi_model* m, double dT, int64_t iterations,
                        const double* u, const double* v, const double* w, int64_t nvel, double dT_vel,
                        const double* parf, int64_t npar, double dT_PAR,
                        const double* temp, int64_t ntemp, double dT_temp, pi_sim** out) {
    if (!m || !out) return fail(m, PI_ERR_ARG, "pi_sim_create: NULL argument");
    *out = nullptr;
    if (!parf || !temp || npar < 1 || ntemp < 1 || iterations < 0)
        return fail(m, PI_ERR_ARG, "pi_sim_create: PARF and temp series are required");
    const HostGrid& g = m->hg;
    int has_vel = (u != nullptr);
    // validate_velocity / validate_PARF / validate_temp (Simulation/utils.jl:213-304)
    if (has_vel) {
        if (!v || !w || nvel < 1) return fail(m, PI_ERR_ARG, "pi_sim_create: u, v and w are required together");
        if (std::floor(dT_vel / dT) * dT != dT_vel)
            return fail(m, PI_ERR_SHAPE, "ΔT_vel must be an integer times of " + julia_float(dT) + ".");
        if ((double)nvel < std::floor((double)iterations * dT / dT_vel))
            return fail(m, PI_ERR_SHAPE, "Velocities provided cannot cover the time period of (iterations+1)*ΔT (" +
                                          julia_float((double)iterations * dT) + " seconds) with ΔT_vel = " + julia_float(dT_vel) + ".");
    }
    if (std::floor(dT_PAR / dT) * dT != dT_PAR)
        return fail(m, PI_ERR_SHAPE, "ΔT_PAR must be an integer times of " + julia_float(dT) + ".");
    if ((double)npar < std::floor((double)iterations * dT / dT_PAR))
        return fail(m, PI_ERR_SHAPE, "Surface PAR provided cannot cover the time period of (iterations+1)*ΔT (" +
                                      julia_float((double)iterations * dT) + " seconds) with ΔT_PAR = " + julia_float(dT_PAR) + ".");
    if (std::floor(dT_temp / dT) * dT != dT_temp)
        return fail(m, PI_ERR_SHAPE, "ΔT_temp must be an integer times of " + julia_float(dT) + ".");
    if ((double)ntemp < std::floor((double)iterations * dT / dT_temp))
        return fail(m, PI_ERR_SHAPE, "Temperature provided cannot cover the time period of (iterations+1)*ΔT (" +
                                      julia_float((double)iterations * dT) + " seconds) with ΔT_temp = " + julia_float(dT_temp) + ".");
    if (m->b32) {
        pi_status st = pi_batch_set_series(m->b32, 0, u, v, w, nvel, dT_vel, parf, npar, dT_PAR, temp, ntemp, dT_temp, 0);
        if (st) return fwd32(m, st);
        pi_sim* s = new pi_sim();
        s->m = m; s->fp32 = 1; s->dT = dT; s->iterations = iterations; s->has_vel = has_vel;
        *out = s;
        return PI_OK;
    }
    pi_sim* s = new pi_sim();
    s->m = m; s->dT = dT; s->iterations = iterations; s->has_vel = has_vel;
    s->nvel = nvel; s->npar = npar; s->ntemp = ntemp; s->dT_vel = dT_vel; s->dT_PAR = dT_PAR; s->dT_temp = dT_temp;
    auto cleanup = [&](pi_status st) { pi_sim_destroy(s); return st; };
    const size_t bytes = g.G * sizeof(double);
    if (has_vel) {
        int ex = g.topo[0] == PI_BOUNDED, ey = g.topo[1] == PI_BOUNDED, ez = g.topo[2] == PI_BOUNDED;
        size_t nu = (size_t)(g.Nx + ex) * g.Ny * g.Nz, nv = (size_t)g.Nx * (g.Ny + ey) * g.Nz, nw = (size_t)g.Nx * g.Ny * (g.Nz + ez);
        std::vector<double> U, V, W;
        for (int64_t t = 0; t < nvel; ++t) {
            host_vel_copy(g, u + t * nu, v + t * nv, w + t * nw, U, V, W);
            for (auto* hv : { &U, &V, &W }) {
                double* d = nullptr;
                if (cudaMalloc(&d, bytes) != cudaSuccess) return cleanup(fail(m, PI_ERR_NOMEM, "pi_sim_create: velocity series"));
                s->vel.push_back(d);
                if (cudaMemcpyAsync(d, hv->data(), bytes, cudaMemcpyHostToDevice, m->stream) != cudaSuccess)
                    return cleanup(fail(m, PI_ERR_CUDA, "pi_sim_create: upload velocity"));
                if (cudaStreamSynchronize(m->stream) != cudaSuccess) return cleanup(fail(m, PI_ERR_CUDA, "pi_sim_create: synchronize"));
            }
        }
    }
    size_t nf = (size_t)g.Nx * g.Ny;
    if (cudaMalloc(&s->parf, nf * npar * sizeof(double)) != cudaSuccess) return cleanup(fail(m, PI_ERR_NOMEM, "pi_sim_create: PARF series"));
    if (cudaMemcpyAsync(s->parf, parf, nf * npar * sizeof(double), cudaMemcpyHostToDevice, m->stream) != cudaSuccess)
        return cleanup(fail(m, PI_ERR_CUDA, "pi_sim_create: upload PARF"));
    std::vector<double> T(g.G, 0.0);
    size_t nt = (size_t)g.Nx * g.Ny * g.Nz;
    for (int64_t q = 0; q < ntemp; ++q) {
        const double* src = temp + q * nt;
        for (int k = 1; k <= g.Nz; ++k) for (int j = 1; j <= g.Ny; ++j) for (int i = 1; i <= g.Nx; ++i)
            T[g.id(i + g.Hx, j + g.Hy, k + g.Hz)] = src[(size_t)(i - 1) + (size_t)g.Nx * ((size_t)(j - 1) + (size_t)g.Ny * (size_t)(k - 1))];
        double* d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess) return cleanup(fail(m, PI_ERR_NOMEM, "pi_sim_create: temperature series"));
        s->temp.push_back(d);
        if (cudaMemcpyAsync(d, T.data(), bytes, cudaMemcpyHostToDevice, m->stream) != cudaSuccess)
            return cleanup(fail(m, PI_ERR_CUDA, "pi_sim_create: upload temperature"));
        if (cudaStreamSynchronize(m->stream) != cudaSuccess) return cleanup(fail(m, PI_ERR_CUDA, "pi_sim_create: synchronize"));
    }
    *out = s;
    return PI_OK;
}

pi_status pi_sim_update(pi_sim* s, int32_t time_offset, int32_t sync) {
    if (!s || !s->m) return PI_ERR_ARG;
    return pi_sim_update_steps(s, 1, s->iterations, time_offset, sync);
}

pi_status pi_sim_update_steps(pi_sim* s, int64_t first, int64_t n, int32_t time_offset, int32_t sync) {
    if (!s || !s->m) return PI_ERR_ARG;
    pi_model* m = s->m;
    if (first < 1 || n < 0) return fail(m, PI_ERR_ARG, "pi_sim_update_steps: first >= 1 and n >= 0 required");
    if (s->fp32) {
        pi_status st = pi_batch_set_time_offset(m->b32, 0, time_offset);
        if (st) return fwd32(m, st);
        return fwd32(m, pi_batch_step_from(m->b32, s->dT, first, n, sync));
    }
    const HostGrid& g = m->hg;
    const size_t nf = (size_t)g.Nx * g.Ny;
    for (int64_t i = first; i < first + n; ++i) {
        double tv = (time_offset & 1) ? (double)(i - 1) * s->dT : m->t;
        double tp = (time_offset & 2) ? (double)(i - 1) * s->dT : m->t;
        double tt = (time_offset & 4) ? (double)(i - 1) * s->dT : m->t;
        if (s->has_vel) {
            int64_t t_vel = (int64_t)std::floor(tv / s->dT_vel) + 1;
            if (t_vel < 1 || t_vel > s->nvel) return fail(m, PI_ERR_SHAPE, "BoundsError: velocity snapshot " + std::to_string(t_vel) + " not provided");
            for (int c = 0; c < 3; ++c) m->vel1[c] = s->vel[(size_t)(t_vel - 1) * 3 + c];
            m->vel1_buf = -1;
        }
        int64_t t_par = (int64_t)std::floor(tp / s->dT_PAR) + 1;
        if (t_par < 1 || t_par > s->npar) return fail(m, PI_ERR_SHAPE, "BoundsError: PARF snapshot " + std::to_string(t_par) + " not provided");
        CK(cudaMemcpyAsync(m->PARF, s->parf + (size_t)(t_par - 1) * nf, nf * sizeof(double), cudaMemcpyDeviceToDevice, m->stream), "PARF copy");
        int64_t t_temp = (int64_t)std::floor(tt / s->dT_temp) + 1;
        if (t_temp < 1 || t_temp > s->ntemp) return fail(m, PI_ERR_SHAPE, "BoundsError: temperature snapshot " + std::to_string(t_temp) + " not provided");
        m->temp = s->temp[(size_t)(t_temp - 1)];
        pi_status st = enqueue_step(m, s->dT);
        if (st) return st;
    }
    if (sync) return pi_synchronize(m);
    return PI_OK;
}

pi_status pi_sim_destroy(pi_sim* s) {
    if (!s) return PI_OK;
    pi_model* m = s->m;
    if (s->fp32) {
        pi_status st = m ? fwd32(m, pi_batch_clear_series(m->b32, 0)) : PI_OK;
        delete s;
        return st;
    }
    if (m) {
        cudaStreamSynchronize(m->stream);
        // the model must not keep pointers into the series
        bool bound = false;
        for (double* d : s->vel) for (int c = 0; c < 3; ++c) if (m->vel1[c] == d || m->vel0[c] == d) bound = true;
        if (bound) {
            // copy the bound snapshot into own buffers so the model stays usable
            for (int c = 0; c < 3; ++c) {
                int b = 0;
                cudaMemcpyAsync(m->velbuf[b][c], m->vel1[c], m->hg.G * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
                m->vel1[c] = m->velbuf[b][c];
                m->vel0[c] = m->velbuf[b][c];
            }
            m->vel1_buf = 0;
        }
        for (double* d : s->temp) if (m->temp == d) {
            cudaMemcpyAsync(m->temp_own, d, m->hg.G * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
            m->temp = m->temp_own;
        }
        cudaStreamSynchronize(m->stream);
    }
    for (double* d : s->vel) cudaFree(d);
    for (double* d : s->temp) cudaFree(d);
    if (s->parf) cudaFree(s->parf);
    delete s;
    return PI_OK;
}

}  // extern "C"

// Allocation-free tracer advection entry point (its own file; compiled in this translation unit
// so the kernels above are shared rather than defined twice).
#include "noalloc.cu"
