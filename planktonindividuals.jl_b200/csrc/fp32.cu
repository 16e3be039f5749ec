// libpib200 — FP32 form: batches of independent members stepped together (pi_batch_* of
// include/pib200.h). A PlanktonModel created with PI_FP32 is a batch of one member.
//
// One step is this sequence of launches, each covering every member:
//   k32_bind             forcing of the step from device-resident series; vel½ buffer choice
//   k32_velhalf          vel½ for members whose vel₀ and vel₁ differ
//   k32_move             RK4 + diffusion + find_inds!, pop/Chl sums, previous decisions; dividers
//                        and newly freed slots marked in bitmaps over logical slots
//   k32_par              calc_par! down each column
//   k32_count_tiles      dividers and free slots of every tile of logical slots
//   scan(tile counts)    division and free-slot offsets of every tile
//   k32_assign           k-th divider → k-th free slot per (member, species) segment
//   k32_daughters        copy_daughter_individuals! + divide_to_half!
//   k32_physiology       QuotaMode growth, consumption sums, decisions for the next step
//   k32_tracer           the whole tracer update when no member has tracer diffusion or flux
//                        boundary conditions: x, y and z sweeps of TMA-staged level tiles, sinking,
//                        forcing, particle terms, apply_tendency! and the halo fill in one walk
//                        down the levels
//   (otherwise, and in the first step after a tracer upload, these three:)
//   k32_xy               DST3FL x and y sweeps of every tracer on level tiles in shared memory
//   k32_ztail            z sweep walking columns, then diffusion, sinking, forcing, BCs, particle
//                        terms and apply_tendency!
//   k32_halo<x,y,z>      fill_halo_tracer!
//   k32_end_step         vel₀ ← vel₁, iteration and t
// Every sort_interval steps (and before the first step after an upload) the slots of every segment
// are put back in cell order by a counting sort into the second buffer of the individual arrays
// (k32_sort_count, a scan of the bin populations, k32_sort_scatter).
// Nothing in a step reads a host value, so the step is captured once as a CUDA graph (one per
// tracer-buffer parity and individual-buffer parity) and replayed. The results do not depend on block shapes, tile-per-block
// assignment, tracer tile heights or z walk lengths (integer sums commute; every other value is computed by
// exactly one thread from the same inputs), which lets the autotuner time real steps.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels_fp32.cuh"
#include "kernels_tracer.cuh"
#include "host_common.h"

using namespace p32;
using namespace pih;

namespace {

thread_local std::string g_batch_error;

inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

struct HostBC {
    int kind = PI_BC_NONE;
    long long nt = 0;
    float* v = nullptr;
};

struct MemberHost {
    HostGrid g;
    long long C = 0;
    uint64_t seed = 0;
    pi_bgc_params bgc{};
    std::vector<pi_quota_params> sp;
    int all_water = 1;
    // device-resident forcing series (owned), or none
    float* ser_vel = nullptr;
    float* ser_parf = nullptr;
    float* ser_temp = nullptr;
    HostBC bcs[PI_NTRACERS][6];
};

// Defaults: the autotuner's choices on a 256×256×64 model with 4 M individuals (pi_batch_autotune
// retunes them for other sizes; no result depends on them)
struct Tuning {
    int bs_move = 256, bs_phys = 128, bs_assign = 128;
    int persist_move = 2, persist_phys = 0;   // 0: one tile per block; k: k blocks per SM, looping
    int ty = 16;                              // rows of an x-y tracer tile (4, 8, 16 or 28)
    int lz = 32;                              // levels walked by a z thread (8, 16, 32 or 64)
    int wpb_par = 2;
    int occ_move = 2, occ_phys = 4;           // register fit of k32_move / k32_physiology (blocks of 256 per SM)
    int concurrent = 0;                       // k32_xy on a second branch beside the particle kernels
    int fused = 0;                            // k32_tracer when the batch allows it (the autotuner
                                              // picks it where it beats k32_xy + k32_ztail + halo fill)
    int lz_fused = 32;                        // levels finished per k32_tracer block
};

}  // namespace

struct pi_batch {
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    int nm = 0, nsp = 0, nseg = 0;
    std::vector<MemberHost> mh;
    std::vector<MemberDev> mdh;
    std::vector<MemberSeries> serh;
    std::vector<FluxBC32> bch;
    std::string err;
    std::vector<void*> allocs;
    long long Gtot = 0, Stot = 0, ncol = 0, maxG = 0, maxcol = 0, maxhalo = 0;
    bool halo_direct = true;        // every member has N >= H on every axis: one-pass halo fill
    int nlev = 0;
    // device
    MemberDev* md = nullptr;
    SpeciesDev32* sp = nullptr;
    SpeciesDec64* dec64 = nullptr;
    // optional diagnostics (pi_batch_set_diags)
    uint32_t tr_mask = 0, proc_mask = 0;
    float* diag_tr = nullptr;                // 14 × Gtot
    unsigned long long* diag_proc = nullptr; // nsp × PI_NPROC × Gtot, fixed point
    unsigned long long* guard = nullptr;    // guard band: decisions recomputed, decisions changed
    BgcDev32* bgc = nullptr;
    FluxBC32* bcs = nullptr;
    MemberForcing* F = nullptr;
    MemberSeries* S = nullptr;
    StepState* st = nullptr;
    uint32_t* errw = nullptr;
    float* trbuf[2] = {nullptr, nullptr};
    int cur = 0;                    // trbuf[cur] holds the current tracers
    float *par = nullptr, *diag_par = nullptr, *PARF = nullptr;
    float *dzF = nullptr, *dzC = nullptr;
    uint8_t* lm = nullptr;
    float* velown = nullptr;        // 6 planes of Gtot: buffer b, component c at (b*3+c)*Gtot
    float* velh = nullptr;          // 3 planes of Gtot
    float* tempown = nullptr;       // Gtot
    uint32_t* dcnt = nullptr;
    int* pop = nullptr;
    int* pop_sp = nullptr;
    unsigned long long* acc = nullptr;
    unsigned long long* chl_acc = nullptr;
    float4* env = nullptr;          // 2 per cell: packed environment of occupied cells
    IndDev32 P{};                   // the current individual buffer (Pbuf[pcur])
    IndDev32 Pbuf[2]{};
    int pcur = 0;
    // storage-order sort
    unsigned long long* sort_bins = nullptr;    // nbins populations
    unsigned long long* sort_offs = nullptr;    // their exclusive scan, then the fill cursors
    long long nbins = 0;
    unsigned long long* sort_sums = nullptr;    // chunk sums of the bin scan
    int sort_interval = 32;         // steps between sorts; 0: never
    long long since_sort = 0;
    bool need_sort = true;
    long long nwords = 0;           // words of each logical-slot bitmap
    int ntiles = 0;
    int2* tiles = nullptr;
    int* seg_tile0 = nullptr;
    unsigned long long *tile_cnt = nullptr, *tile_off = nullptr;
    int *divlist = nullptr, *freelist = nullptr;
    uint32_t* ndiv = nullptr;
    long long* line_off[3] = {nullptr, nullptr, nullptr};
    long long nlines[3] = {0, 0, 0};
    double last_dT = 0.0;
    double* stage = nullptr;        // 3 × maxG doubles of upload staging (synchronous calls)
    cudaEvent_t copied = nullptr;   // recorded after a setter's host→device copies
    // forcing setters: host→device copies on their own stream into double-buffered staging, so
    // they overlap the steps already queued; the conversion runs on the model stream
    cudaStream_t cstream = nullptr;
    cudaStream_t s2 = nullptr;                 // second branch of a step (k32_xy beside the particle kernels)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    struct Stage { unsigned char* p[2] = {nullptr, nullptr}; cudaEvent_t copied[2] = {nullptr, nullptr};
                   cudaEvent_t freed[2] = {nullptr, nullptr}; int k = 0; };
    Stage vst, tst, pst;            // velocity (3 × maxG values), temperature (maxG), PARF (maxcol)
    // own velocity buffers (0/1) per member, tracked on the host so setters need not wait for the
    // queued steps: the buffer vel₁ is bound to (-1: a series snapshot), whether a setter bound it
    // after the last queued step, and the buffer that is vel₀ of the next step (-1: none)
    std::vector<int> vel1_buf, vel1_pending, vel0_buf;
    double* partial = nullptr;      // budget partials
    unsigned long long* scratch = nullptr;
    // work tables (device) built for the current tuning
    Tab32 T{};
    std::vector<void*> table_allocs;
    int tables_ty = -1, tables_lz = -1;
    int4* xy_items = nullptr;
    int nxy_items = 0;
    int4* z_items = nullptr;
    int nz_items = 0;
    float* tb = nullptr;
    float* rdzC = nullptr;
    int4* trk_items = nullptr;
    int ntrk_items = 0;
    int tables_lzf = -1;
    unsigned char* tmaps = nullptr;  // CUtensorMap per member, [tracer buffer][member], 128 bytes each
    bool tracers_dirty = true;       // a tracer was uploaded since the last step
    int64_t call_step0 = 0;          // source of the call-step copy (kept alive for the async copy)
    Tuning tune;
    // graphs
    cudaGraphExec_t gexec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [tracer buffer][individual buffer]
    double graph_dT = -1.0;
    int use_graph = 1;
    // profiling
    int profiling = 0;
    struct Mark { const char* name; cudaEvent_t a, b; };
    std::vector<Mark> marks;
    std::vector<cudaEvent_t> event_pool;
    std::vector<std::string> prof_names;
    std::vector<int64_t> prof_count;
    std::vector<double> prof_ms;
};

namespace {

pi_status bfail(pi_batch* b, pi_status code, const std::string& msg) {
    if (b) b->err = msg; else g_batch_error = msg;
    return code;
}
pi_status bcuda(pi_batch* b, cudaError_t e, const char* what) {
    return bfail(b, e == cudaErrorMemoryAllocation ? PI_ERR_NOMEM : PI_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define BK(call, what)                                              \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return bcuda(b, e_, what);           \
    } while (0)

template <typename T>
pi_status balloc(pi_batch* b, T** p, size_t n, const char* what, std::vector<void*>* list = nullptr) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return bcuda(b, e, what);
    (list ? *list : b->allocs).push_back(q);
    *p = (T*)q;
    return PI_OK;
}

cudaEvent_t take_event(pi_batch* b) {
    if (!b->event_pool.empty()) { cudaEvent_t e = b->event_pool.back(); b->event_pool.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

struct BScope {
    pi_batch* b;
    pi_batch::Mark mk;
    bool on;
    cudaStream_t st;
    BScope(pi_batch* b_, const char* name, cudaStream_t s_ = nullptr) : b(b_), on(b_->profiling != 0), st(s_ ? s_ : b_->stream) {
        if (!on) return;
        mk.name = name; mk.a = take_event(b); mk.b = take_event(b);
        cudaEventRecord(mk.a, st);
    }
    ~BScope() {
        if (!on) return;
        cudaEventRecord(mk.b, st);
        b->marks.push_back(mk);
    }
};

void drain(pi_batch* b) {
    for (auto& mk : b->marks) {
        float ms = 0.f;
        cudaEventSynchronize(mk.b);
        cudaEventElapsedTime(&ms, mk.a, mk.b);
        size_t q = 0;
        while (q < b->prof_names.size() && b->prof_names[q] != mk.name) ++q;
        if (q == b->prof_names.size()) { b->prof_names.push_back(mk.name); b->prof_count.push_back(0); b->prof_ms.push_back(0.0); }
        b->prof_count[q] += 1;
        b->prof_ms[q] += ms;
        b->event_pool.push_back(mk.a);
        b->event_pool.push_back(mk.b);
    }
    b->marks.clear();
}

void free_graphs(pi_batch* b) {
    for (int p = 0; p < 2; ++p)
        for (int q = 0; q < 2; ++q)
            if (b->gexec[p][q]) { cudaGraphExecDestroy(b->gexec[p][q]); b->gexec[p][q] = nullptr; }
    b->graph_dT = -1.0;
}

void free_tables(pi_batch* b) {
    for (void* p : b->table_allocs) cudaFree(p);
    b->table_allocs.clear();
    b->tables_ty = b->tables_lz = b->tables_lzf = -1;
}

// k32_tracer applies when no member has tracer diffusion or flux boundary conditions (k32_ztail's
// general path), every axis of every member has at least as many cells as halo points (one-pass
// halo fill), and the tracers' halos are filled (not the first step after an upload).
bool use_fused(const pi_batch* b) {
    if (!b->tune.fused || !b->halo_direct || b->tracers_dirty) return false;
    for (int m = 0; m < b->nm; ++m) {
        if (b->mdh[m].any_bc) return false;
        const pi_bgc_params& p = b->mh[m].bgc;
        if ((float)p.kappa_h != 0.0f || (float)p.kappa_v != 0.0f) return false;
    }
    return true;
}

// TMA descriptors of every member's tracers (x, y, z, tracer) in each tracer buffer, for members
// whose row pitch is a multiple of 16 bytes; the kernel copies the others with cp.async.
pi_status build_tensor_maps(pi_batch* b) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return bfail(b, PI_ERR_CUDA, "cuTensorMapEncodeTiled not available");
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    std::vector<CUtensorMap> maps(2 * (size_t)b->nm);
    memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    for (int p = 0; p < 2; ++p)
        for (int m = 0; m < b->nm; ++m) {
            const MemberDev& d = b->mdh[m];
            if (d.Gx % 4 != 0) continue;
            const cuuint64_t dims[4] = { (cuuint64_t)d.Gx, (cuuint64_t)d.Gy, (cuuint64_t)d.Gz, (cuuint64_t)PI_NTRACERS };
            const cuuint64_t strides[3] = { (cuuint64_t)d.Gx * 4, (cuuint64_t)d.Gx * d.Gy * 4, (cuuint64_t)b->Gtot * 4 };
            const cuuint32_t box[4] = { TRK_W, TRK_R, 1, 1 };
            const cuuint32_t es[4] = { 1, 1, 1, 1 };
            CUresult r = encode(&maps[(size_t)p * b->nm + m], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                                (void*)(b->trbuf[p] + d.cell_off), dims, strides, box, es,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return bfail(b, PI_ERR_CUDA, "cuTensorMapEncodeTiled failed for member " + std::to_string(m));
        }
    BK(cudaMemcpyAsync(b->tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, b->stream), "upload tensor maps");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

void free_series(MemberHost& h) {
    if (h.ser_vel) cudaFree(h.ser_vel);
    if (h.ser_parf) cudaFree(h.ser_parf);
    if (h.ser_temp) cudaFree(h.ser_temp);
    h.ser_vel = h.ser_parf = h.ser_temp = nullptr;
}

void free_batch(pi_batch* b) {
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_graphs(b);
    free_tables(b);
    for (auto& h : b->mh) {
        free_series(h);
        for (int n = 0; n < PI_NTRACERS; ++n) for (int f = 0; f < 6; ++f) if (h.bcs[n][f].v) cudaFree(h.bcs[n][f].v);
    }
    for (void* p : b->allocs) cudaFree(p);
    b->allocs.clear();
    for (cudaEvent_t e : b->event_pool) cudaEventDestroy(e);
    b->event_pool.clear();
    if (b->copied) cudaEventDestroy(b->copied);
    for (pi_batch::Stage* st : { &b->vst, &b->tst, &b->pst })
        for (int k = 0; k < 2; ++k) {
            if (st->copied[k]) cudaEventDestroy(st->copied[k]);
            if (st->freed[k]) cudaEventDestroy(st->freed[k]);
        }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->s2) cudaStreamDestroy(b->s2);
    if (b->cstream) cudaStreamDestroy(b->cstream);
    if (b->stream) cudaStreamDestroy(b->stream);
    b->stream = nullptr;
}

SpeciesDev32 to_dev(const pi_quota_params& p) {
    SpeciesDev32 d;
    d.Nsuper = (float)p.Nsuper; d.Cquota = (float)p.Cquota; d.Chl2Cint = (float)p.Chl2Cint;
    d.alpha = (float)p.alpha; d.Phi = (float)p.Phi; d.Topt = (float)p.Topt; d.Tmax = (float)p.Tmax;
    d.Ea = (float)p.Ea; d.PCmax = (float)p.PCmax; d.VDOCmax = (float)p.VDOCmax; d.VNO3max = (float)p.VNO3max;
    d.VNH4max = (float)p.VNH4max; d.VPO4max = (float)p.VPO4max; d.KsatDOC = (float)p.KsatDOC;
    d.KsatNH4 = (float)p.KsatNH4; d.KsatNO3 = (float)p.KsatNO3; d.KsatPO4 = (float)p.KsatPO4;
    d.Cqmax = (float)p.Cqmax; d.Nqmax = (float)p.Nqmax; d.Pqmax = (float)p.Pqmax; d.Chl2N = (float)p.Chl2N;
    d.R_NC = (float)p.R_NC; d.R_PC = (float)p.R_PC; d.k_mtb = (float)p.k_mtb; d.respir = (float)p.respir;
    d.grz_P = (float)p.grz_P; d.dvid_P = (float)p.dvid_P; d.dvid_reg = (float)p.dvid_reg;
    d.dvid_reg2 = (float)p.dvid_reg2; d.mort_P = (float)p.mort_P; d.mort_reg = (float)p.mort_reg;
    d.grazFracC = (float)p.grazFracC; d.grazFracN = (float)p.grazFracN; d.grazFracP = (float)p.grazFracP;
    d.mortFracC = (float)p.mortFracC; d.mortFracN = (float)p.mortFracN; d.mortFracP = (float)p.mortFracP;
    d.dvid_type = (int)p.dvid_type;
    // tempFunc's normaliser (growth_kernels.jl:2-16), a constant of the species
    d.OGT_rate = (float)std::exp(-(double)d.Ea / (8.3145 * ((double)d.Topt + 273.15)));
    return d;
}

BgcDev32 to_dev(const pi_bgc_params& p) {
    BgcDev32 d;
    d.kw = (float)p.kw; d.kc = (float)p.kc; d.kDOC = (float)p.kDOC; d.Nit = (float)p.Nit; d.kDON = (float)p.kDON;
    d.kDOP = (float)p.kDOP; d.kPOC = (float)p.kPOC; d.kPON = (float)p.kPON; d.kPOP = (float)p.kPOP;
    d.kappa_h = (float)p.kappa_h; d.kappa_v = (float)p.kappa_v; d.kappa_hP = (float)p.kappa_hP;
    d.kappa_vP = (float)p.kappa_vP; d.shared_graz = p.shared_graz == 1.0;
    d.w_sink_org = (float)p.w_sink_org; d.w_sink_inorg = (float)p.w_sink_inorg; d.lambda_POC = (float)p.lambda_POC;
    d.lambda_min = (float)p.lambda_min; d.kdiss = (float)p.kdiss; d.lambda_dust = (float)p.lambda_dust;
    d.lambda_Fe = (float)p.lambda_Fe; d.ligand = (float)p.ligand; d.DFeFrac = (float)p.DFeFrac;
    return d;
}

pi_status check_member(const pi_member& mb, int nsp, std::string& msg) {
    const pi_grid* grid = mb.grid;
    if (!grid || !mb.bgc || !mb.species || mb.capacity < 1 || !grid->dzF || !grid->dzC) { msg = "NULL grid/params or capacity < 1"; return PI_ERR_ARG; }
    if (grid->Nx < 1 || grid->Ny < 1 || grid->Nz < 1) { msg = "grid size must be at least 1 in every direction"; return PI_ERR_ARG; }
    if (grid->Hx < 2 || grid->Hy < 2 || grid->Hz < 2 || grid->Hx > 8 || grid->Hy > 8 || grid->Hz > 8) { msg = "halo must be 2..8 points (DST3FL needs at least 2)"; return PI_ERR_ARG; }
    for (int a = 0; a < 3; ++a)
        if (grid->topo[a] != PI_PERIODIC && grid->topo[a] != PI_BOUNDED) { msg = "topology must be Periodic or Bounded"; return PI_ERR_ARG; }
    if (grid->topo[2] != PI_BOUNDED) { msg = "z must be Bounded (tracer sinking has no Periodic rule)"; return PI_ERR_ARG; }
    if (grid->metrics) { msg = "LatLonGrid is built in the FP64 form only (precision PI_FP64)"; return PI_ERR_ARG; }
    long long Gx = grid->Nx + 2LL * grid->Hx, Gy = grid->Ny + 2LL * grid->Hy, Gz = grid->Nz + 2LL * grid->Hz;
    if (Gx * Gy * Gz >= (1LL << 31) - 2 || f32_bits(Gx) + f32_bits(Gy) + f32_bits(Gz) > 31) { msg = "grid too large for 32-bit cell indices"; return PI_ERR_ARG; }
    if (mb.capacity >= (1LL << 31)) { msg = "capacity must be below 2^31"; return PI_ERR_ARG; }
    for (int s = 0; s < nsp; ++s) {
        const pi_quota_params& p = mb.species[s];
        int ty = (int)p.dvid_type;
        if ((double)ty != p.dvid_type || ty < 1 || ty > 3) { msg = "dvid_type must be 1 (Sizer), 2 (Timer) or 3 (Sizer_Timer)"; return PI_ERR_PARAM; }
        if (!(p.Cquota > 0.0) || !(p.Nsuper > 0.0)) { msg = "Cquota and Nsuper must be positive"; return PI_ERR_PARAM; }
    }
    return PI_OK;
}

// Work tables for the current tuning (tracer tile height, z walk length) on the device.
pi_status build_tables(pi_batch* b) {
    const int ty = b->tune.ty, lz = b->tune.lz, lzf = b->tune.lz_fused;
    if (b->tables_ty == ty && b->tables_lz == lz && b->tables_lzf == lzf) return PI_OK;
    free_tables(b);
    std::vector<int4> xy, zz, icol, trk;
    for (int m = 0; m < b->nm; ++m) {
        const HostGrid& g = b->mh[m].g;
        for (int L = 1 + g.Hz; L <= g.Nz + g.Hz; ++L)
            for (int j0 = 1 + g.Hy; j0 <= g.Ny + g.Hy; j0 += ty)
                for (int i0 = 1 + g.Hx; i0 <= g.Nx + g.Hx; i0 += 28) xy.push_back(make_int4(m, i0, j0, L));
        for (int k0 = 1 + g.Hz; k0 <= g.Nz + g.Hz; k0 += lz)
            for (int j = 1 + g.Hy; j <= g.Ny + g.Hy; ++j)
                for (int i0 = 1 + g.Hx; i0 <= g.Nx + g.Hx; i0 += 32) zz.push_back(make_int4(m, i0, j, k0));
        for (int j = 1; j <= g.Ny; ++j)
            for (int i0 = 1; i0 <= g.Nx; i0 += 32) icol.push_back(make_int4(m, i0, j, 0));
        for (int k0 = 1 + g.Hz; k0 <= g.Nz + g.Hz; k0 += lzf)
            for (int j0 = 1 + g.Hy; j0 <= g.Ny + g.Hy; j0 += TRK_TY)
                for (int i0 = 1 + g.Hx; i0 <= g.Nx + g.Hx; i0 += TRK_TX) trk.push_back(make_int4(m, i0, j0, k0));
    }
    if (xy.size() >= (size_t)INT32_MAX || zz.size() >= (size_t)INT32_MAX) return bfail(b, PI_ERR_ARG, "work tables too large");
    auto up = [&](std::vector<int4>& v, int4** dst, int* n) -> pi_status {
        int4* d = nullptr;
        pi_status s = balloc(b, &d, v.size(), "work table", &b->table_allocs);
        if (s) return s;
        BK(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(int4), cudaMemcpyHostToDevice, b->stream), "upload work table");
        *dst = d; *n = (int)v.size();
        return PI_OK;
    };
    pi_status s;
    int4* ic = nullptr;
    if ((s = up(xy, &b->xy_items, &b->nxy_items))) return s;
    if ((s = up(zz, &b->z_items, &b->nz_items))) return s;
    if ((s = up(icol, &ic, &b->T.nicol))) return s;
    if ((s = up(trk, &b->trk_items, &b->ntrk_items))) return s;
    b->T.icol = ic;
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    b->tables_ty = ty; b->tables_lz = lz; b->tables_lzf = lzf;
    return PI_OK;
}

size_t xy_smem(int ty) { return (size_t)(3 * ty + 5) * PI_NTRACERS * 32 * sizeof(float); }

float* velown(pi_batch* b, int m, int buf, int c) { return b->velown + ((long long)(buf * 3 + c)) * b->Gtot + b->mdh[m].cell_off; }

// Launch grid of a tile kernel: one block per tile, or a persistent grid of k blocks per SM.
unsigned tile_grid(pi_batch* b, int persist) {
    if (!persist) return (unsigned)std::max(1, b->ntiles);
    return (unsigned)std::max(1, std::min(b->ntiles, persist * b->nsm));
}
unsigned warp_grid(long long nitems, int wpb) { return std::max(1u, nblk(nitems, wpb)); }

// Enqueues one step on the batch stream (eager launches, or the body of a graph capture).
pi_status enqueue_step(pi_batch* b, double dT, int cur) {
    cudaStream_t s = b->stream;
    const long long G = b->Gtot;
    const float fdT = (float)dT;
    float* tr = b->trbuf[cur];
    float* trn = b->trbuf[cur ^ 1];
    const bool fused = use_fused(b);
    BK(cudaMemsetAsync(b->pop, 0, G * sizeof(int), s), "zero pop");
    if (b->pop_sp) BK(cudaMemsetAsync(b->pop_sp, 0, (size_t)b->nsp * G * sizeof(int), s), "zero pop");
    { BScope sc(b, "k32_bind");
      const unsigned gx = std::max(1u, std::min<unsigned>(nblk(b->maxcol, 256), 64));
      k32_bind<<<dim3(gx, b->nm), 256, 0, s>>>(b->nm, b->md, b->S, b->F, b->st, dT, b->PARF, b->errw); }
    // grids of the field passes: about 8 blocks per SM over all members
    const unsigned fgx = std::max(1u, std::min<unsigned>(nblk(b->maxG, 256), std::max(1, b->nsm * 8 / b->nm)));
    { BScope sc(b, "k32_velhalf");
      const unsigned gx = fgx;
      k32_velhalf<<<dim3(gx, b->nm), 256, 0, s>>>(b->md, b->F, b->errw); }
    TrArgs ta;
    ta.T = b->T; ta.lm = b->lm; ta.dzF = b->dzF; ta.dzC = b->dzC; ta.rdzC = b->rdzC; ta.bgc = b->bgc;
    ta.bcs = b->bcs; ta.st = b->st; ta.F = b->F; ta.Gtot = G; ta.tr = tr; ta.tb = b->tb; ta.tr_next = trn;
    ta.acc = b->acc; ta.pop = b->pop; ta.dT = fdT; ta.err = b->errw;
    // k32_xy reads the tracers at the start of the step and this step's u and v only, so it can run
    // on a second branch beside the particle kernels; k32_ztail joins the two
    auto launch_xy = [&](cudaStream_t st) {
        TrArgs a = ta;
        a.items = b->xy_items; a.nitems = b->nxy_items;
        BScope sc(b, "k32_xy", st);
        // persistent: as many blocks as fit at once, each looping over items with the next
        // item's loads in flight
        int per_sm = 1;
        const int ty = b->tune.ty;
        if (ty == 28) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k32_xy<28>, 32 * 32, xy_smem(28));
        else if (ty == 16) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k32_xy<16>, 32 * 20, xy_smem(16));
        else if (ty == 8) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k32_xy<8>, 32 * 12, xy_smem(8));
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k32_xy<4>, 32 * 8, xy_smem(4));
        const unsigned grid = (unsigned)std::max(1, std::min(b->nxy_items, std::max(1, per_sm) * b->nsm));
        if (ty == 28) k32_xy<28><<<grid, 32 * 32, xy_smem(28), st>>>(a);
        else if (ty == 16) k32_xy<16><<<grid, 32 * 20, xy_smem(16), st>>>(a);
        else if (ty == 8) k32_xy<8><<<grid, 32 * 12, xy_smem(8), st>>>(a);
        else k32_xy<4><<<grid, 32 * 8, xy_smem(4), st>>>(a);
    };
    const bool branch = !fused && b->tune.concurrent;
    if (branch) {
        BK(cudaEventRecord(b->ev_fork, s), "fork");
        BK(cudaStreamWaitEvent(b->s2, b->ev_fork, 0), "fork");
        launch_xy(b->s2);
        BK(cudaEventRecord(b->ev_join, b->s2), "join");
    }
    {
        MoveArgs a;
        a.T = b->T; a.P = b->P; a.sp = b->sp; a.bgc = b->bgc; a.F = b->F; a.rdzC = b->rdzC; a.st = b->st;
        a.dT = fdT; a.Gtot = G; a.pop = b->pop; a.pop_sp = b->pop_sp; a.chl_acc = b->chl_acc; a.acc = b->acc;
        a.dcnt = b->dcnt; a.err = b->errw;
        BScope sc(b, "k32_move");
        const unsigned g = tile_grid(b, b->tune.persist_move);
        if (b->tune.occ_move == 4) k32_move<4><<<g, b->tune.bs_move, 0, s>>>(a);
        else if (b->tune.occ_move == 3) k32_move<3><<<g, b->tune.bs_move, 0, s>>>(a);
        else k32_move<2><<<g, b->tune.bs_move, 0, s>>>(a);
    }
    { BScope sc(b, "k32_par");
      k32_par<<<warp_grid(b->T.nicol, b->tune.wpb_par), 32 * b->tune.wpb_par, 0, s>>>(b->T, b->dzF, b->bgc, b->chl_acc, b->PARF,
                                                                                   b->par, b->diag_par, tr, G, b->F, b->pop,
                                                                                   b->env, b->errw); }
    { BScope sc(b, "k32_count_tiles");
      k32_count_tiles<<<nblk((long long)b->ntiles * 32, 256), 256, 0, s>>>(b->T, b->P, b->tile_cnt, b->errw); }
    { BScope sc(b, "k32_scan_tiles");
      k32_scan_tiles<<<std::min(b->nseg, 65535), 1024, 0, s>>>(b->T, b->tile_cnt, b->tile_off, b->nseg, b->errw); }
    { BScope sc(b, "k32_assign");
      k32_assign<<<nblk((long long)b->ntiles * 32, b->tune.bs_assign), b->tune.bs_assign, 0, s>>>(
          b->T, b->P, b->tile_cnt, b->tile_off, b->divlist, b->freelist, b->ndiv, b->st, b->errw); }
    { BScope sc(b, "k32_daughters");
      k32_daughters<<<dim3(4, b->nseg), 128, 0, s>>>(b->T, b->P, b->divlist, b->freelist, b->ndiv, b->errw); }
    {
        PhysArgs a;
        a.T = b->T; a.P = b->P; a.sp = b->sp; a.F = b->F; a.st = b->st; a.dT = fdT; a.Gtot = G; a.tr = tr;
        a.par = b->par; a.pop = b->pop; a.pop_sp = b->pop_sp; a.env = b->env; a.acc = b->acc; a.dcnt = b->dcnt;
        a.err = b->errw; a.dec64 = b->dec64; a.guard = b->guard;
        a.dproc = b->diag_proc; a.pmask = b->proc_mask;
        BScope sc(b, "k32_physiology");
        const unsigned g = tile_grid(b, b->tune.persist_phys);
        if (b->tune.occ_phys == 4) k32_physiology<4><<<g, b->tune.bs_phys, 0, s>>>(a);
        else if (b->tune.occ_phys == 3) k32_physiology<3><<<g, b->tune.bs_phys, 0, s>>>(a);
        else k32_physiology<2><<<g, b->tune.bs_phys, 0, s>>>(a);
    }
    {
        TrArgs a = ta;
        if (fused) {
            TrkArgs A;
            A.a = a;
            A.a.items = b->trk_items; A.a.nitems = b->ntrk_items;
            A.maps = b->tmaps + (size_t)cur * b->nm * sizeof(CUtensorMap);
            A.lz = b->tune.lz_fused;
            BScope sc(b, "k32_tracer");
            k32_tracer<<<dim3((unsigned)std::max(1, b->ntrk_items), 2), TRK_THREADS, tracer_smem_bytes(), s>>>(A);
        } else {
        if (branch) BK(cudaStreamWaitEvent(s, b->ev_join, 0), "join");
        else launch_xy(s);
        {
            a.items = b->z_items; a.nitems = b->nz_items;
            BScope sc(b, "k32_ztail");
            const unsigned grid = (unsigned)std::max(1, b->nz_items);
            const dim3 blk(32, PI_NTRACERS);
            const size_t zs = ztail_smem(b->tune.lz);
            if (b->tune.lz == 8) k32_ztail<8><<<grid, blk, zs, s>>>(a);
            else if (b->tune.lz == 32) k32_ztail<32><<<grid, blk, zs, s>>>(a);
            else if (b->tune.lz == 64) k32_ztail<64><<<grid, blk, zs, s>>>(a);
            else k32_ztail<16><<<grid, blk, zs, s>>>(a);
        }
        }
    }
    if (fused) {
        // k32_tracer wrote the halo cells with the interior
    } else if (b->halo_direct) { BScope sc(b, "k32_halo");
      // about 16 blocks per SM over all members, enough for every member's halo cells
      const unsigned gx = std::max(1u, std::min<unsigned>(nblk(b->maxhalo, 256), std::max(1, b->nsm * 16 / b->nm)));
      k32_halo_direct<<<dim3(gx, b->nm), 256, 0, s>>>(b->md, G, trn, PI_NTRACERS, b->errw);
    } else { BScope sc(b, "k32_halo");
      k32_halo<0><<<std::min<unsigned>(nblk(b->nlines[0], 128), 148 * 8), 128, 0, s>>>(b->md, b->line_off[0], b->nm, G, trn, PI_NTRACERS, b->errw);
      k32_halo<1><<<std::min<unsigned>(nblk(b->nlines[1], 128), 148 * 8), 128, 0, s>>>(b->md, b->line_off[1], b->nm, G, trn, PI_NTRACERS, b->errw);
      k32_halo<2><<<std::min<unsigned>(nblk(b->nlines[2], 128), 148 * 8), 128, 0, s>>>(b->md, b->line_off[2], b->nm, G, trn, PI_NTRACERS, b->errw); }
    k32_copy_if_err<<<148 * 4, 256, 0, s>>>(trn, tr, (long long)PI_NTRACERS * G, b->errw);
    if (b->tr_mask) k32_diag_tracers<<<148 * 4, 256, 0, s>>>(b->diag_tr, trn, b->tr_mask, G, b->errw);
    k32_end_step<<<nblk(b->nm, 128), 128, 0, s>>>(b->nm, b->F, b->st, dT, b->errw);
    BK(cudaGetLastError(), "step launch");
    return PI_OK;
}

pi_status capture_graphs(pi_batch* b, double dT) {
    free_graphs(b);
    pi_status st = PI_OK;
    const bool dirty = b->tracers_dirty;
    b->tracers_dirty = false;           // the graphs serve the steps with filled tracer halos
    for (int q = 0; q < 2 && !st; ++q) {
        b->P = b->Pbuf[q];
        for (int p = 0; p < 2; ++p) {
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) { st = bcuda(b, e, "begin capture"); break; }
            st = enqueue_step(b, dT, p);
            e = cudaStreamEndCapture(b->stream, &g);
            if (st) { if (g) cudaGraphDestroy(g); break; }
            if (e != cudaSuccess) { st = bcuda(b, e, "end capture"); break; }
            e = cudaGraphInstantiate(&b->gexec[p][q], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) { st = bcuda(b, e, "instantiate graph"); break; }
        }
    }
    b->P = b->Pbuf[b->pcur];
    b->tracers_dirty = dirty;
    if (st) return st;
    b->graph_dT = dT;
    return PI_OK;
}

// Puts every segment's slots back in cell order (into the other individual buffer).
pi_status enqueue_sort(pi_batch* b) {
    cudaStream_t s = b->stream;
    IndDev32& P = b->Pbuf[b->pcur];
    IndDev32& Q = b->Pbuf[b->pcur ^ 1];
    { BScope sc(b, "k32_sort");
      BK(cudaMemsetAsync(b->sort_bins, 0, (size_t)b->nbins * sizeof(unsigned long long), s), "zero sort bins");
      k32_sort_count<<<tile_grid(b, 8), 256, 0, s>>>(b->T, P, b->sort_bins);
      const long long nch = (b->nbins + 1024 * SCAN_PER - 1) / (1024 * SCAN_PER);
      k32_scan_sums<<<(unsigned)nch, 1024, 0, s>>>(b->sort_bins, b->nbins, b->sort_sums);
      k32_scan_chunks<<<1, 1024, 0, s>>>(b->sort_sums, nch);
      k32_scan_apply<<<(unsigned)nch, 1024, 0, s>>>(b->sort_bins, b->nbins, b->sort_sums, b->sort_offs);
      k32_sort_scatter<<<tile_grid(b, 8), 256, 0, s>>>(b->T, P, Q, b->sort_offs);
      BK(cudaGetLastError(), "sort launch"); }
    b->pcur ^= 1;
    b->P = b->Pbuf[b->pcur];
    b->since_sort = 0;
    b->need_sort = false;
    return PI_OK;
}

// Bookkeeping after a step was queued: the sort cycle and the own velocity buffers (vel₁ of the
// step is vel₀ of the next).
void after_step(pi_batch* b) {
    b->since_sort += 1;
    for (int m = 0; m < b->nm; ++m) {
        b->vel0_buf[m] = b->vel1_buf[m];
        b->vel1_pending[m] = 0;
    }
}

// A sort before the next step when one is due.
pi_status maybe_sort(pi_batch* b) {
    if (b->sort_interval <= 0) return PI_OK;
    if (!b->need_sort && b->since_sort < b->sort_interval) return PI_OK;
    return enqueue_sort(b);
}

pi_status check_errors(pi_batch* b) {
    uint32_t e = 0;
    StepState hs{};
    BK(cudaMemcpyAsync(&e, b->errw, sizeof e, cudaMemcpyDeviceToHost, b->stream), "read error word");
    BK(cudaMemcpyAsync(&hs, b->st, sizeof hs, cudaMemcpyDeviceToHost, b->stream), "read step state");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    if (!e) return PI_OK;
    BK(cudaMemsetAsync(b->errw, 0, sizeof(uint32_t), b->stream), "clear error word");
    if (e & F32_ERR_CAPACITY) {
        // the step stopped after the decisions: drop the unconsumed loss sums and divider marks
        BK(cudaMemsetAsync(b->acc, 0, (size_t)ACC_N * b->Gtot * sizeof(unsigned long long), b->stream), "clear sums");
        BK(cudaMemsetAsync(b->P.dvbits, 0, (size_t)b->nwords * sizeof(uint32_t), b->stream), "clear divider marks");
        BK(cudaStreamSynchronize(b->stream), "synchronize");
        // TimeStep! advanced model.iteration and model.t before it threw (time_step.jl:14-15)
        hs.iteration = hs.err_iter;
        hs.t = (double)hs.err_iter * b->last_dT;
        BK(cudaMemcpyAsync(b->st, &hs, sizeof hs, cudaMemcpyHostToDevice, b->stream), "write step state");
        BK(cudaStreamSynchronize(b->stream), "synchronize");
        const double tf = hs.t;
        std::string msg = "number of individual exceeds the capacity at timestep " + julia_float(tf / 86400.0) + " days";
        if (b->nm > 1) msg += " (member " + std::to_string(hs.err_member) + ")";
        return bfail(b, PI_ERR_CAPACITY, msg);
    }
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    if (e & F32_ERR_TIMEOUT) return bfail(b, PI_ERR_TIMEOUT, "a bounded wait for staged tracer data gave up");
    if (e & F32_ERR_FORCING) return bfail(b, PI_ERR_SHAPE, "BoundsError: forcing snapshot not provided for the step time");
    if (e & F32_ERR_LISTS) return bfail(b, PI_ERR_STATE, "internal error: a division list entry outside its segment");
    return bfail(b, PI_ERR_DOMAIN, "an individual left the halo-padded grid (cell index out of range)");
}

}  // namespace

extern "C" {

pi_status pi_batch_last_error(pi_batch* b, char* buf, size_t len) {
    const std::string& e = b ? b->err : g_batch_error;
    if (buf && len) {
        size_t n = std::min(len - 1, e.size());
        memcpy(buf, e.c_str(), n);
        buf[n] = 0;
    }
    return PI_OK;
}

pi_status pi_batch_create(const pi_member* members, int32_t nmembers, int32_t nspecies, pi_batch** out) {
    if (!out) return bfail(nullptr, PI_ERR_ARG, "pi_batch_create: out is NULL");
    *out = nullptr;
    if (!members || nmembers < 1 || nspecies < 1) return bfail(nullptr, PI_ERR_ARG, "pi_batch_create: no members or nspecies < 1");
    if ((long long)nmembers * nspecies > 65535) return bfail(nullptr, PI_ERR_ARG, "pi_batch_create: members × species must be at most 65535");
    for (int m = 0; m < nmembers; ++m) {
        std::string msg;
        pi_status st = check_member(members[m], nspecies, msg);
        if (st) return bfail(nullptr, st, "pi_batch_create: member " + std::to_string(m) + ": " + msg);
    }
    pi_batch* b = new pi_batch();
    auto bail = [&](pi_status st) { g_batch_error = b->err; free_batch(b); delete b; return st; };
    if (cudaGetDevice(&b->device) != cudaSuccess) { b->err = "pi_batch_create: no CUDA device"; return bail(PI_ERR_CUDA); }
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) { b->err = "pi_batch_create: stream"; return bail(PI_ERR_CUDA); }
    if (cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming) != cudaSuccess) { b->err = "pi_batch_create: event"; return bail(PI_ERR_CUDA); }
    if (cudaStreamCreateWithFlags(&b->cstream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->s2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess) { b->err = "pi_batch_create: stream"; return bail(PI_ERR_CUDA); }
    for (pi_batch::Stage* st : { &b->vst, &b->tst, &b->pst })
        for (int k = 0; k < 2; ++k)
            if (cudaEventCreateWithFlags(&st->copied[k], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&st->freed[k], cudaEventDisableTiming) != cudaSuccess) {
                b->err = "pi_batch_create: event"; return bail(PI_ERR_CUDA);
            }
    b->nm = nmembers; b->nsp = nspecies; b->nseg = nmembers * nspecies;
    b->mh.resize(nmembers);
    b->mdh.resize(nmembers);
    std::vector<SpeciesDev32> sph;
    std::vector<SpeciesDec64> dech;
    std::vector<BgcDev32> bgch;
    std::vector<float> dzF, dzC;
    std::vector<int2> tiles;
    std::vector<int> seg_tile0;
    long long cell = 0, slot = 0, col = 0, words = 0, bins = 0;
    int lev = 0;
    bool any_land = false;
    for (int m = 0; m < nmembers; ++m) {
        const pi_member& mb = members[m];
        const pi_grid* grid = mb.grid;
        MemberHost& h = b->mh[m];
        HostGrid& g = h.g;
        g.Nx = grid->Nx; g.Ny = grid->Ny; g.Nz = grid->Nz; g.Hx = grid->Hx; g.Hy = grid->Hy; g.Hz = grid->Hz;
        g.Gx = g.Nx + 2 * g.Hx; g.Gy = g.Ny + 2 * g.Hy; g.Gz = g.Nz + 2 * g.Hz;
        for (int a = 0; a < 3; ++a) g.topo[a] = grid->topo[a];
        g.dx = grid->dx; g.dy = grid->dy;
        g.dzF.assign(grid->dzF, grid->dzF + g.Gz);
        g.dzC.assign(grid->dzC, grid->dzC + g.Gz);
        g.G = (long long)g.Gx * g.Gy * g.Gz;
        h.all_water = 1;
        if (grid->landmask) {
            g.lm.assign(grid->landmask, grid->landmask + g.G);
            for (uint8_t& v : g.lm) { v = v ? 1 : 0; if (!v) h.all_water = 0; }
            if (!h.all_water) any_land = true;
        }
        h.C = mb.capacity; h.seed = mb.seed; h.bgc = *mb.bgc;
        h.sp.assign(mb.species, mb.species + nspecies);
        MemberDev& d = b->mdh[m];
        d.Nx = g.Nx; d.Ny = g.Ny; d.Nz = g.Nz; d.Hx = g.Hx; d.Hy = g.Hy; d.Hz = g.Hz;
        d.Gx = g.Gx; d.Gy = g.Gy; d.Gz = g.Gz; d.tx = g.topo[0]; d.ty = g.topo[1]; d.tz = g.topo[2];
        d.all_water = h.all_water; d.any_bc = 0;
        d.dx = (float)g.dx; d.dy = (float)g.dy;
        d.rdx = 1.0f / d.dx; d.rdy = 1.0f / d.dy;
        d.cbx = f32_bits(g.Nx); d.cby = f32_bits(g.Ny);
        d.hbx = f32_bits(g.Gx); d.hby = f32_bits(g.Gy);
        d.cell_off = cell; d.G = g.G; d.col_off = col; d.slot_off = slot; d.C = h.C;
        d.dz_off = lev; d.bc_off = m * PI_NTRACERS * 6; d.seed = h.seed;
        d.woff = words; d.wps = (h.C + F32_TILE - 1) / F32_TILE * (F32_TILE / 32);
        d.bin_off = bins;
        double cmin = 1e300, chlmin = 1e300;
        for (int s = 0; s < nspecies; ++s) {
            const pi_quota_params& p = h.sp[s];
            cmin = std::min(cmin, p.Cquota * p.Nsuper);
            if (p.Chl2Cint > 0.0) chlmin = std::min(chlmin, p.Chl2Cint * p.Cquota * p.Nsuper);
            sph.push_back(to_dev(p));
            dech.push_back(SpeciesDec64{p.grz_P, p.mort_P, p.mort_reg, p.dvid_P, p.dvid_reg, p.dvid_reg2,
                                        p.Cquota * p.Nsuper, (int)p.dvid_type});
        }
        if (chlmin > 1e299) chlmin = cmin;
        // 2^40 units per nominal individual: sums of up to ~2^22 individuals per cell fit in 63 bits
        d.fx_unit = cmin * 0x1p-40;
        d.chl_unit = chlmin * 0x1p-40;
        d.fx_inv = 1.0 / d.fx_unit;
        d.chl_inv = 1.0 / d.chl_unit;
        bgch.push_back(to_dev(h.bgc));
        for (int k = 0; k < g.Gz; ++k) { dzF.push_back((float)g.dzF[k]); dzC.push_back((float)g.dzC[k]); }
        for (int s = 0; s < nspecies; ++s) {
            seg_tile0.push_back((int)tiles.size());
            for (long long t0 = 0; t0 < h.C; t0 += F32_TILE) tiles.push_back(make_int2(m * nspecies + s, (int)t0));
        }
        cell += (g.G + 63) / 64 * 64;       // members start on 256-byte boundaries
        slot += (long long)nspecies * h.C;
        words += (long long)nspecies * d.wps;
        bins += (long long)nspecies * ((long long)g.Nx * g.Ny * g.Nz + (h.C + F32_TILE - 1) / F32_TILE);
        col += (long long)g.Nx * g.Ny;
        lev += g.Gz;
        b->maxG = std::max(b->maxG, g.G);
        if (g.Nx < g.Hx || g.Ny < g.Hy || g.Nz < g.Hz) b->halo_direct = false;
        b->maxhalo = std::max(b->maxhalo, g.G - (long long)g.Nx * g.Ny * g.Nz);
        b->maxcol = std::max(b->maxcol, (long long)g.Nx * g.Ny);
    }
    seg_tile0.push_back((int)tiles.size());
    if (tiles.size() >= (size_t)INT32_MAX) { b->err = "pi_batch_create: too many slots"; return bail(PI_ERR_ARG); }
    b->Gtot = cell; b->Stot = slot; b->ncol = col; b->nlev = lev; b->ntiles = (int)tiles.size();
    b->nwords = words; b->nbins = bins;
    const long long G = b->Gtot, S = b->Stot;
    pi_status st;
#define BA(ptr, n) do { st = balloc(b, &(ptr), (size_t)(n), #ptr); if (st) return bail(st); } while (0)
    BA(b->md, nmembers); BA(b->sp, sph.size()); BA(b->dec64, dech.size()); BA(b->guard, 2); BA(b->bgc, nmembers); BA(b->bcs, (size_t)nmembers * PI_NTRACERS * 6);
    BA(b->F, nmembers); BA(b->S, nmembers); BA(b->st, 1); BA(b->errw, 1);
    BA(b->trbuf[0], PI_NTRACERS * G); BA(b->trbuf[1], PI_NTRACERS * G); BA(b->tb, PI_NTRACERS * G);
    BA(b->par, G); BA(b->diag_par, G); BA(b->PARF, std::max<long long>(col, 1));
    BA(b->dzF, lev); BA(b->dzC, lev); BA(b->rdzC, lev);
    if (any_land) BA(b->lm, G);
    BA(b->velown, 6 * G); BA(b->velh, 3 * G); BA(b->tempown, G);
    BA(b->dcnt, (size_t)nspecies * 4 * G); BA(b->pop, G);
    bool shared = true;
    for (auto& h : b->mh) if (h.bgc.shared_graz != 1.0) shared = false;
    if (!shared) BA(b->pop_sp, (size_t)nspecies * G);
    BA(b->acc, (size_t)ACC_N * G); BA(b->chl_acc, G); BA(b->env, 2 * G);
    for (int q = 0; q < 2; ++q) {
        IndDev32& Pq = b->Pbuf[q];
        BA(Pq.cell, S); BA(Pq.scell, S); BA(Pq.ox, S); BA(Pq.oy, S); BA(Pq.oz, S); BA(Pq.Bm, S); BA(Pq.Cq, S);
        BA(Pq.Nq, S); BA(Pq.Pq, S); BA(Pq.Chl, S); BA(Pq.age, S); BA(Pq.gen, S); BA(Pq.flags, S); BA(Pq.stat, S);
        BA(Pq.lslot, S);
    }
    BA(b->Pbuf[0].phys, S); BA(b->Pbuf[0].freebits, words); BA(b->Pbuf[0].dvbits, words);
    b->Pbuf[1].phys = b->Pbuf[0].phys; b->Pbuf[1].freebits = b->Pbuf[0].freebits; b->Pbuf[1].dvbits = b->Pbuf[0].dvbits;
    b->pcur = 0;
    b->P = b->Pbuf[0];
    IndDev32& P = b->P;
    BA(b->sort_bins, bins); BA(b->sort_offs, bins);
    BA(b->tiles, tiles.size()); BA(b->seg_tile0, seg_tile0.size());
    BA(b->tile_cnt, tiles.size()); BA(b->tile_off, tiles.size());
    BA(b->divlist, S); BA(b->freelist, S); BA(b->ndiv, b->nseg);
    for (int a = 0; a < 3; ++a) BA(b->line_off[a], nmembers + 1);
    BA(b->stage, std::max<long long>(3 * b->maxG, col));
    for (int k = 0; k < 2; ++k) {
        BA(b->vst.p[k], 3 * b->maxG * sizeof(double));
        BA(b->tst.p[k], b->maxG * sizeof(double));
        BA(b->pst.p[k], std::max<long long>(b->maxcol, 1) * sizeof(double));
    }
    b->vel1_buf.assign(nmembers, 1);
    b->vel1_pending.assign(nmembers, 0);
    b->vel0_buf.assign(nmembers, 0);
    BA(b->partial, 3 * 1024); BA(b->scratch, 4);
    BA(b->tmaps, 2 * (size_t)nmembers * sizeof(CUtensorMap));
    BA(b->sort_sums, (b->nbins + 1024 * SCAN_PER - 1) / (1024 * SCAN_PER));
#undef BA
    // series and forcing tables
    b->serh.assign(nmembers, MemberSeries{});
    std::vector<MemberForcing> Fh(nmembers);
    for (int m = 0; m < nmembers; ++m) {
        for (int c = 0; c < 3; ++c) {
            b->serh[m].velh_buf[c] = b->velh + (long long)c * G + b->mdh[m].cell_off;
            Fh[m].vel0[c] = velown(b, m, 0, c);
            Fh[m].vel1[c] = velown(b, m, 1, c);
            Fh[m].velh[c] = b->serh[m].velh_buf[c];
        }
        Fh[m].temp = b->tempown + b->mdh[m].cell_off;
        b->serh[m].dT_vel = b->serh[m].dT_PAR = b->serh[m].dT_temp = 1.0;
    }
    b->bch.assign((size_t)nmembers * PI_NTRACERS * 6, FluxBC32{PI_BC_NONE, 0, 0, 0, nullptr});
    std::vector<long long> lo[3];
    for (int a = 0; a < 3; ++a) lo[a].assign(nmembers + 1, 0);
    for (int m = 0; m < nmembers; ++m) {
        const HostGrid& g = b->mh[m].g;
        lo[0][m + 1] = lo[0][m] + (long long)g.Gy * g.Gz;
        lo[1][m + 1] = lo[1][m] + (long long)g.Gx * g.Gz;
        lo[2][m + 1] = lo[2][m] + (long long)g.Gx * g.Gy;
    }
    for (int a = 0; a < 3; ++a) b->nlines[a] = lo[a][nmembers];
    cudaStream_t s0 = b->stream;
    bool ok = true;
    auto H2D = [&](void* d, const void* h, size_t n) { ok = ok && cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, s0) == cudaSuccess; };
    auto Z = [&](void* d, size_t n) { ok = ok && cudaMemsetAsync(d, 0, n, s0) == cudaSuccess; };
    H2D(b->md, b->mdh.data(), nmembers * sizeof(MemberDev));
    H2D(b->sp, sph.data(), sph.size() * sizeof(SpeciesDev32));
    H2D(b->dec64, dech.data(), dech.size() * sizeof(SpeciesDec64));
    Z(b->guard, 2 * sizeof(unsigned long long));
    H2D(b->bgc, bgch.data(), bgch.size() * sizeof(BgcDev32));
    H2D(b->bcs, b->bch.data(), b->bch.size() * sizeof(FluxBC32));
    H2D(b->F, Fh.data(), nmembers * sizeof(MemberForcing));
    H2D(b->S, b->serh.data(), nmembers * sizeof(MemberSeries));
    H2D(b->dzF, dzF.data(), dzF.size() * sizeof(float));
    H2D(b->dzC, dzC.data(), dzC.size() * sizeof(float));
    std::vector<float> rdzC(dzC.size());
    for (size_t q = 0; q < dzC.size(); ++q) rdzC[q] = 1.0f / dzC[q];
    H2D(b->rdzC, rdzC.data(), rdzC.size() * sizeof(float));
    H2D(b->tiles, tiles.data(), tiles.size() * sizeof(int2));
    H2D(b->seg_tile0, seg_tile0.data(), seg_tile0.size() * sizeof(int));
    for (int a = 0; a < 3; ++a) H2D(b->line_off[a], lo[a].data(), (nmembers + 1) * sizeof(long long));
    if (b->lm) {
        std::vector<uint8_t> lmh(G, 1);
        for (int m = 0; m < nmembers; ++m)
            if (!b->mh[m].g.lm.empty()) std::copy(b->mh[m].g.lm.begin(), b->mh[m].g.lm.end(), lmh.begin() + b->mdh[m].cell_off);
        H2D(b->lm, lmh.data(), G);
        ok = ok && cudaStreamSynchronize(s0) == cudaSuccess;
    }
    Z(b->st, sizeof(StepState)); Z(b->errw, sizeof(uint32_t));
    for (int q = 0; q < 2; ++q) Z(b->trbuf[q], PI_NTRACERS * G * sizeof(float));
    Z(b->par, G * sizeof(float)); Z(b->diag_par, G * sizeof(float)); Z(b->PARF, std::max<long long>(col, 1) * sizeof(float));
    Z(b->velown, 6 * G * sizeof(float)); Z(b->velh, 3 * G * sizeof(float)); Z(b->tempown, G * sizeof(float));
    Z(b->dcnt, (size_t)nspecies * 4 * G * sizeof(uint32_t)); Z(b->pop, G * sizeof(int));
    if (b->pop_sp) Z(b->pop_sp, (size_t)nspecies * G * sizeof(int));
    Z(b->acc, (size_t)ACC_N * G * 8); Z(b->chl_acc, G * 8);
    for (void* p : { (void*)P.ox, (void*)P.oy, (void*)P.oz, (void*)P.Bm, (void*)P.Cq, (void*)P.Nq, (void*)P.Pq,
                     (void*)P.Chl, (void*)P.age, (void*)P.gen }) Z(p, S * sizeof(float));
    Z(P.flags, S); Z(P.stat, S); Z(P.scell, S * sizeof(int32_t));
    // constructor state: inactive, find_inds! cell (0, 0, 0) (plankton_generation.jl:3); storage
    // in logical order; every slot free, no divider
    ok = ok && cudaMemsetAsync(P.cell, 0xff, S * sizeof(int32_t), s0) == cudaSuccess;
    Z(P.dvbits, words * sizeof(uint32_t));
    {
        std::vector<uint32_t> fb(words, 0u);
        for (int m = 0; m < nmembers; ++m) {
            const MemberDev& d = b->mdh[m];
            for (int sp = 0; sp < nspecies; ++sp)
                for (long long L = 0; L < d.C; ++L) fb[d.woff + sp * d.wps + (L >> 5)] |= 1u << (L & 31);
        }
        H2D(P.freebits, fb.data(), words * sizeof(uint32_t));
        ok = ok && cudaStreamSynchronize(s0) == cudaSuccess;
    }
    for (int m = 0; m < nmembers && ok; ++m)
        for (int sp = 0; sp < nspecies; ++sp) {
            const MemberDev& d = b->mdh[m];
            k32_identity_order<<<std::min<unsigned>(nblk(d.C, 256), 1024), 256, 0, s0>>>(P, d.slot_off + sp * d.C, d.C);
        }
    ok = ok && cudaGetLastError() == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s0) == cudaSuccess;
    if (!ok) { b->err = "pi_batch_create: device initialisation failed"; return bail(PI_ERR_CUDA); }
    cudaFuncSetAttribute(k32_xy<28>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xy_smem(28));
    cudaFuncSetAttribute(k32_xy<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xy_smem(16));
    cudaFuncSetAttribute(k32_xy<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xy_smem(8));
    cudaFuncSetAttribute(k32_xy<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xy_smem(4));
    cudaFuncSetAttribute(k32_ztail<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ztail_smem(8));
    cudaFuncSetAttribute(k32_ztail<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ztail_smem(16));
    cudaFuncSetAttribute(k32_ztail<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ztail_smem(32));
    cudaFuncSetAttribute(k32_ztail<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ztail_smem(64));
    cudaFuncSetAttribute(k32_tracer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tracer_smem_bytes());
    st = build_tensor_maps(b);
    if (st) return bail(st);
    b->T.md = b->md; b->T.nsp = nspecies; b->T.tiles = b->tiles; b->T.ntiles = b->ntiles; b->T.seg_tile0 = b->seg_tile0;
    st = build_tables(b);
    if (st) return bail(st);
    *out = b;
    return PI_OK;
}

pi_status pi_batch_destroy(pi_batch* b) {
    if (!b) return PI_OK;
    drain(b);
    free_batch(b);
    delete b;
    return PI_OK;
}

static pi_status check_mem(pi_batch* b, int32_t member, const char* fn) {
    if (!b) return bfail(b, PI_ERR_ARG, std::string(fn) + ": NULL batch");
    if (member < 0 || member >= b->nm) return bfail(b, PI_ERR_ARG, std::string(fn) + ": member out of range");
    return PI_OK;
}

pi_status pi_batch_set_individuals(pi_batch* b, int32_t member, int32_t sp, const pi_individuals* in) {
    pi_status e = check_mem(b, member, "pi_set_individuals");
    if (e) return e;
    if (!in || sp < 0 || sp >= b->nsp) return bfail(b, PI_ERR_ARG, "pi_set_individuals: bad argument");
    const double* dcols[] = { in->x, in->y, in->z, in->Bm, in->Cq, in->Nq, in->Pq, in->Chl, in->gen, in->age,
                              in->graz, in->mort, in->dvid };
    for (const double* p : dcols) if (!p) return bfail(b, PI_ERR_ARG, "pi_set_individuals: NULL attribute");
    if (!in->xi || !in->yi || !in->zi || !in->ac) return bfail(b, PI_ERR_ARG, "pi_set_individuals: NULL attribute");
    const MemberHost& h = b->mh[member];
    const HostGrid& g = h.g;
    const MemberDev& d = b->mdh[member];
    const long long C = h.C;
    std::vector<int32_t> cell(C), scell(C, 0);
    std::vector<float> o[3], f[7];
    for (auto& v : o) v.assign(C, 0.0f);
    for (auto& v : f) v.assign(C, 0.0f);
    std::vector<uint8_t> flags(C), stat(C, 0);
    const double* pos[3] = { in->x, in->y, in->z };
    const int N[3] = { g.Nx, g.Ny, g.Nz }, Hh[3] = { g.Hx, g.Hy, g.Hz }, Gg[3] = { g.Gx, g.Gy, g.Gz };
    const int64_t* idx[3] = { in->xi, in->yi, in->zi };
    for (long long i = 0; i < C; ++i) {
        if (in->ac[i] > 1) return bfail(b, PI_ERR_PARAM, "pi_set_individuals: ac must be 0 or 1");
        double d3[3] = { in->graz[i], in->mort[i], in->dvid[i] };
        for (double v : d3) if (v != 0.0 && v != 1.0) return bfail(b, PI_ERR_PARAM, "pi_set_individuals: graz/mort/dvid must be 0 or 1");
        for (int a = 0; a < 3; ++a)
            if (idx[a][i] < 0 || idx[a][i] > Gg[a]) return bfail(b, PI_ERR_PARAM, "pi_set_individuals: xi/yi/zi outside 0..G");
        flags[i] = (uint8_t)((in->ac[i] ? F32_AC : 0) | (in->graz[i] == 1.0 ? F32_GRAZ : 0) |
                             (in->mort[i] == 1.0 ? F32_MORT : 0) | (in->dvid[i] == 1.0 ? F32_DVID : 0));
        const double* cols[7] = { in->Bm, in->Cq, in->Nq, in->Pq, in->Chl, in->age, in->gen };
        for (int q = 0; q < 7; ++q) f[q][i] = (float)cols[q][i];
        if (!in->ac[i]) { cell[i] = -1; continue; }
        int c[3];
        for (int a = 0; a < 3; ++a) {
            const double x = pos[a][i];
            if (!(x >= 0.0 && x <= (double)N[a])) return bfail(b, PI_ERR_PARAM, "pi_set_individuals: position outside [0, N] of an active individual");
            double fl = std::floor(x);
            c[a] = (int)fl;
            // keep the cell of the FP64 position: an offset that rounds up to 1 becomes the
            // largest float below 1 instead of moving to the next cell
            float of = (float)(x - fl);
            if (of >= 1.0f) of = 0x1.fffffep-1f;
            o[a][i] = of;
        }
        cell[i] = f32_pack(c[0], c[1], c[2], d.cbx, d.cby);
        bool same = true;
        for (int a = 0; a < 3; ++a) same = same && idx[a][i] == c[a] + 1 + Hh[a];
        if (!same) {
            stat[i] = F32_ST_STALE;
            scell[i] = f32_pack((int)in->xi[i], (int)in->yi[i], (int)in->zi[i], d.hbx, d.hby);
        }
    }
    const long long g0 = d.slot_off + (long long)sp * C;
    const IndDev32& P = b->P;
    cudaStream_t s = b->stream;
    BK(cudaMemcpyAsync(P.cell + g0, cell.data(), C * 4, cudaMemcpyHostToDevice, s), "upload individuals");
    BK(cudaMemcpyAsync(P.scell + g0, scell.data(), C * 4, cudaMemcpyHostToDevice, s), "upload individuals");
    float* od[3] = { P.ox, P.oy, P.oz };
    for (int a = 0; a < 3; ++a) BK(cudaMemcpyAsync(od[a] + g0, o[a].data(), C * 4, cudaMemcpyHostToDevice, s), "upload individuals");
    float* fd[7] = { P.Bm, P.Cq, P.Nq, P.Pq, P.Chl, P.age, P.gen };
    for (int q = 0; q < 7; ++q) BK(cudaMemcpyAsync(fd[q] + g0, f[q].data(), C * 4, cudaMemcpyHostToDevice, s), "upload individuals");
    BK(cudaMemcpyAsync(P.flags + g0, flags.data(), C, cudaMemcpyHostToDevice, s), "upload individuals");
    BK(cudaMemcpyAsync(P.stat + g0, stat.data(), C, cudaMemcpyHostToDevice, s), "upload individuals");
    // stored in logical order until the next sort; free-slot bits from ac, no divider marks
    k32_identity_order<<<std::min<unsigned>(nblk(C, 256), 1024), 256, 0, s>>>(P, g0, C);
    BK(cudaGetLastError(), "upload individuals");
    std::vector<uint32_t> fb(d.wps, 0u);
    for (long long i = 0; i < C; ++i) if (!in->ac[i]) fb[i >> 5] |= 1u << (i & 31);
    const long long w0 = d.woff + (long long)sp * d.wps;
    BK(cudaMemcpyAsync(P.freebits + w0, fb.data(), d.wps * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "upload individuals");
    BK(cudaMemsetAsync(P.dvbits + w0, 0, d.wps * sizeof(uint32_t), s), "upload individuals");
    BK(cudaStreamSynchronize(s), "synchronize");
    b->need_sort = true;
    return PI_OK;
}

pi_status pi_batch_get_individuals(pi_batch* b, int32_t member, int32_t sp, pi_individuals* out) {
    pi_status e = check_mem(b, member, "pi_get_individuals");
    if (e) return e;
    if (!out || sp < 0 || sp >= b->nsp) return bfail(b, PI_ERR_ARG, "pi_get_individuals: bad argument");
    const MemberHost& h = b->mh[member];
    const HostGrid& g = h.g;
    const long long C = h.C;
    const long long g0 = b->mdh[member].slot_off + (long long)sp * C;
    std::vector<int32_t> cell(C), scell(C), lslot(C);
    std::vector<float> o[3], f[7];
    std::vector<uint8_t> flags(C), stat(C);
    const IndDev32& P = b->P;
    cudaStream_t s = b->stream;
    BK(cudaMemcpyAsync(lslot.data(), P.lslot + g0, C * 4, cudaMemcpyDeviceToHost, s), "download individuals");
    BK(cudaMemcpyAsync(cell.data(), P.cell + g0, C * 4, cudaMemcpyDeviceToHost, s), "download individuals");
    BK(cudaMemcpyAsync(scell.data(), P.scell + g0, C * 4, cudaMemcpyDeviceToHost, s), "download individuals");
    const float* od[3] = { P.ox, P.oy, P.oz };
    for (int a = 0; a < 3; ++a) { o[a].resize(C); BK(cudaMemcpyAsync(o[a].data(), od[a] + g0, C * 4, cudaMemcpyDeviceToHost, s), "download individuals"); }
    const float* fd[7] = { P.Bm, P.Cq, P.Nq, P.Pq, P.Chl, P.age, P.gen };
    for (int q = 0; q < 7; ++q) { f[q].resize(C); BK(cudaMemcpyAsync(f[q].data(), fd[q] + g0, C * 4, cudaMemcpyDeviceToHost, s), "download individuals"); }
    BK(cudaMemcpyAsync(flags.data(), P.flags + g0, C, cudaMemcpyDeviceToHost, s), "download individuals");
    BK(cudaMemcpyAsync(stat.data(), P.stat + g0, C, cudaMemcpyDeviceToHost, s), "download individuals");
    BK(cudaStreamSynchronize(s), "synchronize");
    const pi_quota_params& p = h.sp[sp];
    const float cq_ns = (float)p.Cquota * (float)p.Nsuper;
    // stored position k holds logical slot lslot[k]: the outputs are in logical order
    std::vector<char> seen(C, 0);
    for (long long k = 0; k < C; ++k) {
        if (lslot[k] < 0 || lslot[k] >= C || seen[lslot[k]]) return bfail(b, PI_ERR_STATE, "pi_get_individuals: storage order corrupted");
        seen[lslot[k]] = 1;
    }
    for (long long k = 0; k < C; ++k) {
        const long long i = lslot[k];       // logical slot written from stored position k
        const uint8_t fl = flags[k];
        const int32_t code = cell[k];
        int ci = 0, cj = 0, ck = 0;
        const MemberDev& md = b->mdh[member];
        if (code >= 0) f32_unpack(code, md.cbx, md.cby, ci, cj, ck);
        const double xyz[3] = { code < 0 ? 0.0 : ci + (double)o[0][k], code < 0 ? 0.0 : cj + (double)o[1][k],
                                code < 0 ? 0.0 : ck + (double)o[2][k] };
        int64_t xi, yi, zi;
        if (stat[k] & F32_ST_STALE) {
            int a0, a1, a2;
            f32_unpack(scell[k], md.hbx, md.hby, a0, a1, a2);
            xi = a0; yi = a1; zi = a2;
        } else if (code < 0) { xi = g.Hx; yi = g.Hy; zi = g.Hz; }
        else { xi = ci + 1 + g.Hx; yi = cj + 1 + g.Hy; zi = ck + 1 + g.Hz; }
        if (out->x) out->x[i] = xyz[0];
        if (out->y) out->y[i] = xyz[1];
        if (out->z) out->z[i] = xyz[2];
        if (out->xi) out->xi[i] = xi;
        if (out->yi) out->yi[i] = yi;
        if (out->zi) out->zi[i] = zi;
        double* cols[7] = { out->Bm, out->Cq, out->Nq, out->Pq, out->Chl, out->age, out->gen };
        for (int q = 0; q < 7; ++q) if (cols[q]) cols[q][i] = (double)f[q][k];
        if (out->Sz) out->Sz[i] = (double)(f[0][k] / cq_ns);
        if (out->ac) out->ac[i] = (fl & F32_AC) ? 1 : 0;
        if (out->graz) out->graz[i] = (fl & F32_GRAZ) ? 1.0 : 0.0;
        if (out->mort) out->mort[i] = (fl & F32_MORT) ? 1.0 : 0.0;
        if (out->dvid) out->dvid[i] = (fl & F32_DVID) ? 1.0 : 0.0;
    }
    return PI_OK;
}

pi_status pi_batch_set_tracer(pi_batch* b, int32_t member, int32_t idx, const double* data) {
    pi_status e = check_mem(b, member, "pi_set_tracer");
    if (e) return e;
    if (!data || idx < 0 || idx >= PI_NTRACERS) return bfail(b, PI_ERR_ARG, "pi_set_tracer: bad argument");
    const long long G = b->mdh[member].G;
    BK(cudaMemcpyAsync(b->stage, data, G * sizeof(double), cudaMemcpyHostToDevice, b->stream), "upload tracer");
    k32_d2f<<<std::min<unsigned>(nblk(G, 256), 1024), 256, 0, b->stream>>>(b->trbuf[b->cur] + idx * b->Gtot + b->mdh[member].cell_off, b->stage, G);
    BK(cudaGetLastError(), "convert tracer");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    b->tracers_dirty = true;
    return PI_OK;
}

pi_status pi_batch_get_tracer(pi_batch* b, int32_t member, int32_t idx, double* out) {
    pi_status e = check_mem(b, member, "pi_get_tracer");
    if (e) return e;
    if (!out || idx < 0 || idx >= PI_NTRACERS) return bfail(b, PI_ERR_ARG, "pi_get_tracer: bad argument");
    const long long G = b->mdh[member].G;
    k32_f2d<<<std::min<unsigned>(nblk(G, 256), 1024), 256, 0, b->stream>>>(b->stage, b->trbuf[b->cur] + idx * b->Gtot + b->mdh[member].cell_off, G);
    BK(cudaGetLastError(), "convert tracer");
    BK(cudaMemcpyAsync(out, b->stage, G * sizeof(double), cudaMemcpyDeviceToHost, b->stream), "download tracer");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

// Interior velocity snapshot (reference layout) into three halo-padded FP32 member fields
// (vel_copy!, Simulation/utils.jl:5-34 with fill_halo_vel!).
}  // extern "C"

// Host → device copies of one setter into the next staging buffer of `st`, on the copy stream; the
// model stream then waits for them. Returns the buffer. The caller queues its conversion on the
// model stream, records st.freed[k] after it, and waits for st.copied[k] before returning (the
// host arrays are free from then on).
static pi_status stage_copy(pi_batch* b, pi_batch::Stage& st, const void* const* src, const size_t* bytes, int n,
                            size_t stride, unsigned char** out) {
    const int k = st.k ^= 1;
    BK(cudaStreamWaitEvent(b->cstream, st.freed[k], 0), "order staging");
    for (int c = 0; c < n; ++c)
        BK(cudaMemcpyAsync(st.p[k] + c * stride, src[c], bytes[c], cudaMemcpyDefault, b->cstream), "upload forcing");
    BK(cudaEventRecord(st.copied[k], b->cstream), "record copies");
    BK(cudaStreamWaitEvent(b->stream, st.copied[k], 0), "order conversion");
    *out = st.p[k];
    return PI_OK;
}
static pi_status stage_done(pi_batch* b, pi_batch::Stage& st) {
    BK(cudaEventRecord(st.freed[st.k], b->stream), "record conversion");
    BK(cudaEventSynchronize(st.copied[st.k]), "synchronize copies");
    return PI_OK;
}

// vel_copy! (Simulation/utils.jl:5-34 with fill_halo_vel!) of an interior snapshot (reference
// layout, Float64 or Float32) into three halo-padded FP32 member fields, queued on the model stream.
template <typename S>
static pi_status vel_copy32(pi_batch* b, int m, const S* u, const S* v, const S* w, float* U, float* V, float* W) {
    const HostGrid& g = b->mh[m].g;
    const MemberDev& d = b->mdh[m];
    cudaStream_t s = b->stream;
    int bd[3] = { g.topo[0] == PI_BOUNDED, g.topo[1] == PI_BOUNDED, g.topo[2] == PI_BOUNDED };
    int dims[3][3] = { { g.Nx + bd[0], g.Ny, g.Nz }, { g.Nx, g.Ny + bd[1], g.Nz }, { g.Nx, g.Ny, g.Nz + bd[2] } };
    float* dst[3] = { U, V, W };
    if (g.Nx >= g.Hx && g.Ny >= g.Hy && g.Nz >= g.Hz) {
        const void* src[3] = { u, v, w };
        size_t bytes[3];
        for (int c = 0; c < 3; ++c) bytes[c] = (size_t)dims[c][0] * dims[c][1] * dims[c][2] * sizeof(S);
        unsigned char* stg = nullptr;
        pi_status e = stage_copy(b, b->vst, src, bytes, 3, b->maxG * sizeof(S), &stg);
        if (e) return e;
        for (int c = 0; c < 3; ++c) {
            BK(cudaMemsetAsync(dst[c], 0, g.G * sizeof(float), s), "clear velocity");
            k32_scatter_interior<S><<<std::min<unsigned>(nblk((long long)dims[c][0] * dims[c][1] * dims[c][2], 256), 1024), 256, 0, s>>>(
                d, dst[c], (const S*)(stg + c * b->maxG * sizeof(S)), dims[c][0], dims[c][1], dims[c][2]);
            k32_halo_vel<0><<<std::min<unsigned>(nblk((long long)g.Gy * g.Gz, 128), 1024), 128, 0, s>>>(d, dst[c], c);
            k32_halo_vel<1><<<std::min<unsigned>(nblk((long long)g.Gx * g.Gz, 128), 1024), 128, 0, s>>>(d, dst[c], c);
            k32_halo_vel<2><<<std::min<unsigned>(nblk((long long)g.Gx * g.Gy, 128), 1024), 128, 0, s>>>(d, dst[c], c);
        }
        BK(cudaGetLastError(), "velocity halo");
        return stage_done(b, b->vst);
    }
    // an axis with fewer cells than halo points: the halo rule of the host grid code, synchronously
    const size_t n[3] = { (size_t)dims[0][0] * dims[0][1] * dims[0][2], (size_t)dims[1][0] * dims[1][1] * dims[1][2],
                          (size_t)dims[2][0] * dims[2][1] * dims[2][2] };
    std::vector<double> hd[3];
    const S* hs[3] = { u, v, w };
    for (int c = 0; c < 3; ++c) hd[c].assign(hs[c], hs[c] + n[c]);
    std::vector<double> Ud, Vd, Wd;
    host_vel_copy(g, hd[0].data(), hd[1].data(), hd[2].data(), Ud, Vd, Wd);
    std::vector<float> tmp(g.G);
    const std::vector<double>* hv[3] = { &Ud, &Vd, &Wd };
    BK(cudaStreamSynchronize(s), "synchronize");
    for (int c = 0; c < 3; ++c) {
        for (long long q = 0; q < g.G; ++q) tmp[q] = (float)(*hv[c])[q];
        BK(cudaMemcpyAsync(dst[c], tmp.data(), g.G * sizeof(float), cudaMemcpyHostToDevice, s), "upload velocity");
        BK(cudaStreamSynchronize(s), "synchronize");
    }
    return PI_OK;
}

extern "C" {

static pi_status read_forcing(pi_batch* b, int m, MemberForcing& f) {
    BK(cudaMemcpyAsync(&f, b->F + m, sizeof f, cudaMemcpyDeviceToHost, b->stream), "read forcing");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}
static pi_status write_forcing(pi_batch* b, int m, const MemberForcing& f) {
    BK(cudaMemcpyAsync(b->F + m, &f, sizeof f, cudaMemcpyHostToDevice, b->stream), "write forcing");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

}  // extern "C"

// New own vel₁ of a member: the own buffer that the velocity bound by the previous setter does not
// occupy (that one is vel₀ by the time this step runs), bound on the device in stream order.
template <typename S>
static pi_status set_velocity_any(pi_batch* b, int32_t member, const S* u, const S* v, const S* w) {
    pi_status e = check_mem(b, member, "pi_set_velocity");
    if (e) return e;
    if (!u || !v || !w) return bfail(b, PI_ERR_ARG, "pi_set_velocity: NULL argument");
    // a buffer bound since the last queued step is reused; otherwise the one that is not vel₀
    const int buf = b->vel1_pending[member] ? b->vel1_buf[member] : (b->vel0_buf[member] == 0 ? 1 : 0);
    float* dst[3] = { velown(b, member, buf, 0), velown(b, member, buf, 1), velown(b, member, buf, 2) };
    if ((e = vel_copy32<S>(b, member, u, v, w, dst[0], dst[1], dst[2]))) return e;
    k32_bind_own<<<1, 32, 0, b->stream>>>(b->F, member, dst[0], dst[1], dst[2], nullptr);
    BK(cudaGetLastError(), "bind velocity");
    b->vel1_buf[member] = buf;
    b->vel1_pending[member] = 1;
    return PI_OK;
}

extern "C" {

pi_status pi_batch_set_velocity(pi_batch* b, int32_t member, const double* u, const double* v, const double* w) {
    return set_velocity_any<double>(b, member, u, v, w);
}
pi_status pi_batch_set_velocity_f32(pi_batch* b, int32_t member, const float* u, const float* v, const float* w) {
    return set_velocity_any<float>(b, member, u, v, w);
}

pi_status pi_batch_set_velocity0(pi_batch* b, int32_t member, const double* u, const double* v, const double* w) {
    pi_status e = check_mem(b, member, "pi_set_velocity0");
    if (e) return e;
    if (!u || !v || !w) return bfail(b, PI_ERR_ARG, "pi_set_velocity0: NULL argument");
    MemberForcing f;
    if ((e = read_forcing(b, member, f))) return e;
    const int buf = (f.vel1[0] == velown(b, member, 0, 0)) ? 1 : 0;   // the own buffer vel₁ does not alias
    if ((e = vel_copy32<double>(b, member, u, v, w, velown(b, member, buf, 0), velown(b, member, buf, 1), velown(b, member, buf, 2)))) return e;
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    for (int c = 0; c < 3; ++c) f.vel0[c] = velown(b, member, buf, c);
    b->vel0_buf[member] = buf;
    return write_forcing(b, member, f);
}

}  // extern "C"

template <typename S>
static pi_status set_PARF_any(pi_batch* b, int32_t member, const S* parf) {
    pi_status e = check_mem(b, member, "pi_set_PARF");
    if (e) return e;
    if (!parf) return bfail(b, PI_ERR_ARG, "pi_set_PARF: NULL argument");
    const long long n = (long long)b->mdh[member].Nx * b->mdh[member].Ny;
    const void* src[1] = { parf };
    const size_t bytes[1] = { n * sizeof(S) };
    unsigned char* stg = nullptr;
    if ((e = stage_copy(b, b->pst, src, bytes, 1, 0, &stg))) return e;
    k32_to_f32<S><<<std::min<unsigned>(nblk(n, 256), 1024), 256, 0, b->stream>>>(b->PARF + b->mdh[member].col_off, (const S*)stg, n);
    BK(cudaGetLastError(), "convert PARF");
    return stage_done(b, b->pst);
}

extern "C" {

pi_status pi_batch_set_PARF(pi_batch* b, int32_t member, const double* parf) { return set_PARF_any<double>(b, member, parf); }
pi_status pi_batch_set_PARF_f32(pi_batch* b, int32_t member, const float* parf) { return set_PARF_any<float>(b, member, parf); }

}  // extern "C"

// copy_interior!: only the interior is written; the halo stays zero
template <typename S>
static pi_status set_temp_any(pi_batch* b, int32_t member, const S* temp) {
    pi_status e = check_mem(b, member, "pi_set_temp");
    if (e) return e;
    if (!temp) return bfail(b, PI_ERR_ARG, "pi_set_temp: NULL argument");
    const MemberDev& d = b->mdh[member];
    const long long n = (long long)d.Nx * d.Ny * d.Nz;
    float* dst = b->tempown + d.cell_off;
    const void* src[1] = { temp };
    const size_t bytes[1] = { n * sizeof(S) };
    unsigned char* stg = nullptr;
    if ((e = stage_copy(b, b->tst, src, bytes, 1, 0, &stg))) return e;
    k32_scatter_interior<S><<<std::min<unsigned>(nblk(n, 256), 1024), 256, 0, b->stream>>>(d, dst, (const S*)stg, d.Nx, d.Ny, d.Nz);
    k32_bind_own<<<1, 32, 0, b->stream>>>(b->F, member, nullptr, nullptr, nullptr, dst);
    BK(cudaGetLastError(), "scatter temp");
    return stage_done(b, b->tst);
}

extern "C" {

pi_status pi_batch_set_temp(pi_batch* b, int32_t member, const double* temp) { return set_temp_any<double>(b, member, temp); }
pi_status pi_batch_set_temp_f32(pi_batch* b, int32_t member, const float* temp) { return set_temp_any<float>(b, member, temp); }

pi_status pi_batch_set_flux_bc(pi_batch* b, int32_t member, int32_t tracer, int32_t face, int32_t kind,
                               const double* values, int64_t nt) {
    pi_status e = check_mem(b, member, "pi_set_flux_bc");
    if (e) return e;
    if (tracer < 0 || tracer >= PI_NTRACERS || face < 0 || face > 5 || kind < 0 || kind > 3)
        return bfail(b, PI_ERR_ARG, "pi_set_flux_bc: bad argument");
    MemberHost& h = b->mh[member];
    const HostGrid& g = h.g;
    size_t n1 = face <= PI_EAST ? g.Ny : g.Nx, n2 = face <= PI_NORTH ? g.Nz : g.Ny;
    size_t n = kind == PI_BC_CONST ? 1 : kind == PI_BC_ARRAY2D ? n1 * n2 : kind == PI_BC_ARRAY3D ? n1 * n2 * (size_t)std::max<int64_t>(nt, 0) : 0;
    if (kind == PI_BC_ARRAY3D && nt < 1) return bfail(b, PI_ERR_SHAPE, "BC: time-dependent flux needs nt >= 1");
    if (n && !values) return bfail(b, PI_ERR_ARG, "pi_set_flux_bc: NULL values");
    HostBC& hb = h.bcs[tracer][face];
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    free_graphs(b);                     // the tracer kernels depend on whether any member has a flux BC
    if (hb.v) { cudaFree(hb.v); hb.v = nullptr; }
    hb.kind = kind; hb.nt = nt;
    if (n) {
        std::vector<float> tmp(n);
        for (size_t q = 0; q < n; ++q) tmp[q] = (float)values[q];
        BK(cudaMalloc(&hb.v, n * sizeof(float)), "bc values");
        BK(cudaMemcpyAsync(hb.v, tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice, b->stream), "upload bc");
    }
    FluxBC32& d = b->bch[(size_t)b->mdh[member].bc_off + tracer * 6 + face];
    d.kind = kind; d.nt = nt; d.v = hb.v; d.n1 = (int)n1; d.n2 = (int)n2;
    int any = 0;
    for (int q = 0; q < PI_NTRACERS * 6; ++q) if (b->bch[(size_t)b->mdh[member].bc_off + q].kind) any = 1;
    b->mdh[member].any_bc = any;
    BK(cudaMemcpyAsync(b->bcs, b->bch.data(), b->bch.size() * sizeof(FluxBC32), cudaMemcpyHostToDevice, b->stream), "upload bcs");
    BK(cudaMemcpyAsync(b->md + member, &b->mdh[member], sizeof(MemberDev), cudaMemcpyHostToDevice, b->stream), "upload member");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

pi_status pi_batch_set_series(pi_batch* b, int32_t member,
                              const double* u, const double* v, const double* w, int64_t nvel, double dT_vel,
                              const double* parf, int64_t npar, double dT_PAR,
                              const double* temp, int64_t ntemp, double dT_temp, int32_t time_offset) {
    pi_status e = check_mem(b, member, "pi_batch_set_series");
    if (e) return e;
    const int has_vel = u != nullptr;
    if (!parf || !temp || npar < 1 || ntemp < 1 || (has_vel && (!v || !w || nvel < 1)))
        return bfail(b, PI_ERR_ARG, "pi_batch_set_series: PARF and temp series are required; u, v, w together");
    if (!(dT_PAR > 0) || !(dT_temp > 0) || (has_vel && !(dT_vel > 0))) return bfail(b, PI_ERR_ARG, "pi_batch_set_series: intervals must be positive");
    if ((e = pi_batch_clear_series(b, member))) return e;
    MemberHost& h = b->mh[member];
    const HostGrid& g = h.g;
    const MemberDev& d = b->mdh[member];
    cudaStream_t s = b->stream;
    MemberSeries& se = b->serh[member];
    if (has_vel) {
        BK(cudaMalloc(&h.ser_vel, (size_t)nvel * 3 * g.G * sizeof(float)), "velocity series");
        int ex = g.topo[0] == PI_BOUNDED, ey = g.topo[1] == PI_BOUNDED, ez = g.topo[2] == PI_BOUNDED;
        size_t nu = (size_t)(g.Nx + ex) * g.Ny * g.Nz, nv = (size_t)g.Nx * (g.Ny + ey) * g.Nz, nw = (size_t)g.Nx * g.Ny * (g.Nz + ez);
        for (int64_t t = 0; t < nvel; ++t) {
            float* base = h.ser_vel + (size_t)t * 3 * g.G;
            if ((e = vel_copy32(b, member, u + t * nu, v + t * nv, w + t * nw, base, base + g.G, base + 2 * g.G))) return e;
        }
    }
    const long long nf = (long long)g.Nx * g.Ny;
    BK(cudaMalloc(&h.ser_parf, (size_t)npar * nf * sizeof(float)), "PARF series");
    for (int64_t t = 0; t < npar; ++t) {
        BK(cudaMemcpyAsync(b->stage, parf + t * nf, nf * sizeof(double), cudaMemcpyDefault, s), "upload PARF");
        k32_d2f<<<std::min<unsigned>(nblk(nf, 256), 1024), 256, 0, s>>>(h.ser_parf + t * nf, b->stage, nf);
        BK(cudaStreamSynchronize(s), "synchronize");
    }
    const long long nt3 = (long long)g.Nx * g.Ny * g.Nz;
    BK(cudaMalloc(&h.ser_temp, (size_t)ntemp * g.G * sizeof(float)), "temperature series");
    BK(cudaMemsetAsync(h.ser_temp, 0, (size_t)ntemp * g.G * sizeof(float), s), "clear temperature series");
    for (int64_t t = 0; t < ntemp; ++t) {
        BK(cudaMemcpyAsync(b->stage, temp + t * nt3, nt3 * sizeof(double), cudaMemcpyDefault, s), "upload temp");
        k32_scatter_interior<double><<<std::min<unsigned>(nblk(nt3, 256), 1024), 256, 0, s>>>(d, h.ser_temp + t * g.G, b->stage, g.Nx, g.Ny, g.Nz);
        BK(cudaStreamSynchronize(s), "synchronize");
    }
    BK(cudaGetLastError(), "upload series");
    se.vel = h.ser_vel; se.nvel = has_vel ? nvel : 0; se.dT_vel = has_vel ? dT_vel : 1.0;
    se.parf = h.ser_parf; se.npar = npar; se.dT_PAR = dT_PAR;
    se.temp = h.ser_temp; se.ntemp = ntemp; se.dT_temp = dT_temp;
    se.has_series = 1; se.has_vel = has_vel; se.time_offset = time_offset;
    BK(cudaMemcpyAsync(b->S + member, &se, sizeof se, cudaMemcpyHostToDevice, s), "upload series table");
    BK(cudaStreamSynchronize(s), "synchronize");
    if (has_vel) { b->vel1_buf[member] = -1; b->vel1_pending[member] = 0; }   // vel₁ comes from the series
    return PI_OK;
}

pi_status pi_batch_clear_series(pi_batch* b, int32_t member) {
    pi_status e = check_mem(b, member, "pi_batch_clear_series");
    if (e) return e;
    MemberHost& h = b->mh[member];
    MemberSeries& se = b->serh[member];
    if (!se.has_series) return PI_OK;
    MemberForcing f;
    if ((e = read_forcing(b, member, f))) return e;
    const long long G = h.g.G;
    cudaStream_t s = b->stream;
    // keep the bound snapshots as the member's own fields
    auto in_series = [&](const float* p) {
        return h.ser_vel && p >= h.ser_vel && p < h.ser_vel + (size_t)se.nvel * 3 * G;
    };
    const bool v1s = in_series(f.vel1[0]), v0s = in_series(f.vel0[0]);
    if (v1s) {
        for (int c = 0; c < 3; ++c) BK(cudaMemcpyAsync(velown(b, member, 1, c), f.vel1[c], G * sizeof(float), cudaMemcpyDeviceToDevice, s), "keep velocity");
        if (v0s && f.vel0[0] == f.vel1[0]) for (int c = 0; c < 3; ++c) f.vel0[c] = velown(b, member, 1, c);
        for (int c = 0; c < 3; ++c) f.vel1[c] = velown(b, member, 1, c);
    }
    if (in_series(f.vel0[0])) {
        for (int c = 0; c < 3; ++c) BK(cudaMemcpyAsync(velown(b, member, 0, c), f.vel0[c], G * sizeof(float), cudaMemcpyDeviceToDevice, s), "keep velocity");
        for (int c = 0; c < 3; ++c) f.vel0[c] = velown(b, member, 0, c);
    }
    if (h.ser_temp && f.temp >= h.ser_temp && f.temp < h.ser_temp + (size_t)se.ntemp * G) {
        BK(cudaMemcpyAsync(b->tempown + b->mdh[member].cell_off, f.temp, G * sizeof(float), cudaMemcpyDeviceToDevice, s), "keep temperature");
        f.temp = b->tempown + b->mdh[member].cell_off;
    }
    if ((e = write_forcing(b, member, f))) return e;
    auto own_of = [&](const float* p) { return p == velown(b, member, 0, 0) ? 0 : p == velown(b, member, 1, 0) ? 1 : -1; };
    b->vel1_buf[member] = own_of(f.vel1[0]);
    b->vel0_buf[member] = own_of(f.vel0[0]);
    b->vel1_pending[member] = 0;
    free_series(h);
    float* keep[3] = { se.velh_buf[0], se.velh_buf[1], se.velh_buf[2] };
    se = MemberSeries{};
    for (int c = 0; c < 3; ++c) se.velh_buf[c] = keep[c];
    se.dT_vel = se.dT_PAR = se.dT_temp = 1.0;
    BK(cudaMemcpyAsync(b->S + member, &se, sizeof se, cudaMemcpyHostToDevice, s), "upload series table");
    BK(cudaStreamSynchronize(s), "synchronize");
    return PI_OK;
}

pi_status pi_batch_set_time_offset(pi_batch* b, int32_t member, int32_t time_offset) {
    pi_status e = check_mem(b, member, "pi_batch_set_time_offset");
    if (e) return e;
    b->serh[member].time_offset = time_offset;
    BK(cudaMemcpyAsync(b->S + member, &b->serh[member], sizeof(MemberSeries), cudaMemcpyHostToDevice, b->stream), "upload series table");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

pi_status pi_batch_synchronize(pi_batch* b) {
    if (!b) return bfail(b, PI_ERR_ARG, "pi_batch_synchronize: NULL batch");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return check_errors(b);
}

pi_status pi_batch_step(pi_batch* b, double dT, int64_t nsteps, int32_t sync) {
    return pi_batch_step_from(b, dT, 1, nsteps, sync);
}

pi_status pi_batch_step_from(pi_batch* b, double dT, int64_t first, int64_t nsteps, int32_t sync) {
    if (!b) return bfail(b, PI_ERR_ARG, "pi_batch_step: NULL batch");
    if (!(dT > 0) || nsteps < 0 || first < 1) return bfail(b, PI_ERR_ARG, "pi_batch_step: ΔT must be positive, nsteps >= 0 and first >= 1");
    pi_status e = build_tables(b);
    if (e) return e;
    bool any3d = false;
    for (const auto& h : b->mh)
        for (int n = 0; n < PI_NTRACERS; ++n) for (int f = 0; f < 6; ++f) any3d = any3d || h.bcs[n][f].kind == PI_BC_ARRAY3D;
    if (any3d) {
        // getbc(bc, i, j, t) of a time-dependent flux reads bc[i, j, iteration] (boundary_conditions.jl:44-52)
        int64_t it = 0;
        if ((e = pi_batch_get_time(b, &it, nullptr))) return e;
        for (const auto& h : b->mh)
            for (int n = 0; n < PI_NTRACERS; ++n)
                for (int f = 0; f < 6; ++f)
                    if (h.bcs[n][f].kind == PI_BC_ARRAY3D && h.bcs[n][f].nt < it + nsteps)
                        return bfail(b, PI_ERR_SHAPE, "BoundsError: time-dependent flux boundary condition has " +
                                                          std::to_string(h.bcs[n][f].nt) + " snapshots, step " +
                                                          std::to_string(it + nsteps) + " needs more");
    }
    b->last_dT = dT;
    // the step index within the update! call, for the time_offset series indexing
    b->call_step0 = first - 1;
    BK(cudaMemcpyAsync(&b->st->call_step, &b->call_step0, sizeof(int64_t), cudaMemcpyHostToDevice, b->stream), "set call step");
    if (b->profiling || !b->use_graph) {
        for (int64_t i = 0; i < nsteps; ++i) {
            if ((e = maybe_sort(b))) return e;
            if ((e = enqueue_step(b, dT, b->cur))) return e;
            b->cur ^= 1;
            after_step(b);
            b->tracers_dirty = false;
        }
    } else {
        if (b->graph_dT != dT || !b->gexec[0][0]) { if ((e = capture_graphs(b, dT))) return e; }
        for (int64_t i = 0; i < nsteps; ++i) {
            if ((e = maybe_sort(b))) return e;
            if (b->tracers_dirty) {
                // the step after a tracer upload maps the halo rows itself (two-kernel path)
                if ((e = enqueue_step(b, dT, b->cur))) return e;
                b->tracers_dirty = false;
            } else {
                BK(cudaGraphLaunch(b->gexec[b->cur][b->pcur], b->stream), "graph launch");
            }
            b->cur ^= 1;
            after_step(b);
        }
    }
    if (sync) return pi_batch_synchronize(b);
    return PI_OK;
}

pi_status pi_batch_get_time(pi_batch* b, int64_t* iteration, double* t) {
    if (!b) return bfail(b, PI_ERR_ARG, "pi_get_time: NULL batch");
    StepState hs{};
    BK(cudaMemcpyAsync(&hs, b->st, sizeof hs, cudaMemcpyDeviceToHost, b->stream), "read step state");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    if (iteration) *iteration = hs.iteration;
    if (t) *t = hs.t;
    return PI_OK;
}

pi_status pi_batch_set_time(pi_batch* b, int64_t iteration, double t) {
    if (!b) return bfail(b, PI_ERR_ARG, "pi_set_time: NULL batch");
    StepState hs{};
    BK(cudaMemcpyAsync(&hs, b->st, sizeof hs, cudaMemcpyDeviceToHost, b->stream), "read step state");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    hs.iteration = iteration; hs.t = t;
    BK(cudaMemcpyAsync(b->st, &hs, sizeof hs, cudaMemcpyHostToDevice, b->stream), "write step state");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

pi_status pi_batch_count_active(pi_batch* b, int32_t member, int32_t sp, int64_t* n) {
    if (!b || !n || member < -1 || member >= b->nm || sp < -1 || sp >= b->nsp) return bfail(b, PI_ERR_ARG, "pi_count_active: bad argument");
    long long first, count;
    if (member < 0) { first = 0; count = b->Stot; }
    else {
        const MemberDev& d = b->mdh[member];
        first = d.slot_off + (sp < 0 ? 0 : (long long)sp * d.C);
        count = sp < 0 ? (long long)b->nsp * d.C : d.C;
    }
    unsigned long long h = 0;
    BK(cudaMemsetAsync(b->scratch, 0, sizeof h, b->stream), "zero count");
    k32_count_active<<<std::max(1u, std::min<unsigned>(nblk(count, 256), 148 * 4)), 256, 0, b->stream>>>(b->P.flags + first, count, b->scratch);
    BK(cudaGetLastError(), "k32_count_active");
    BK(cudaMemcpyAsync(&h, b->scratch, sizeof h, cudaMemcpyDeviceToHost, b->stream), "download count");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    *n = (int64_t)h;
    return PI_OK;
}

pi_status pi_batch_count_active_async(pi_batch* b, int32_t member, int32_t sp, int64_t* out) {
    if (!b || !out || member < -1 || member >= b->nm || sp < -1 || sp >= b->nsp) return bfail(b, PI_ERR_ARG, "pi_count_active_async: bad argument");
    long long first, count;
    if (member < 0) { first = 0; count = b->Stot; }
    else {
        const MemberDev& d = b->mdh[member];
        first = d.slot_off + (sp < 0 ? 0 : (long long)sp * d.C);
        count = sp < 0 ? (long long)b->nsp * d.C : d.C;
    }
    // stream-ordered: the slot is cleared, counted and copied before the next call clears it
    unsigned long long* slot = b->scratch + 1;
    BK(cudaMemsetAsync(slot, 0, sizeof *slot, b->stream), "zero count");
    k32_count_active<<<std::max(1u, std::min<unsigned>(nblk(count, 256), 148 * 4)), 256, 0, b->stream>>>(b->P.flags + first, count, slot);
    BK(cudaGetLastError(), "k32_count_active");
    BK(cudaMemcpyAsync(out, slot, sizeof *slot, cudaMemcpyDeviceToHost, b->stream), "download count");
    return PI_OK;
}

pi_status pi_batch_set_diags(pi_batch* b, uint32_t tracer_mask, uint32_t proc_mask) {
    if (!b || tracer_mask >> PI_NTRACERS || proc_mask >> PI_NPROC) return bfail(b, PI_ERR_ARG, "pi_set_diags: bad argument");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    pi_status e;
    if (tracer_mask && !b->diag_tr && (e = balloc(b, &b->diag_tr, (size_t)PI_NTRACERS * b->Gtot, "tracer diagnostics"))) return e;
    if (proc_mask && !b->diag_proc && (e = balloc(b, &b->diag_proc, (size_t)b->nsp * PI_NPROC * b->Gtot, "process diagnostics"))) return e;
    if (b->diag_tr) BK(cudaMemsetAsync(b->diag_tr, 0, (size_t)PI_NTRACERS * b->Gtot * sizeof(float), b->stream), "clear diagnostics");
    if (b->diag_proc) BK(cudaMemsetAsync(b->diag_proc, 0, (size_t)b->nsp * PI_NPROC * b->Gtot * 8, b->stream), "clear diagnostics");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    b->tr_mask = tracer_mask; b->proc_mask = proc_mask;
    free_graphs(b);                     // the captured steps read the masks
    return PI_OK;
}

pi_status pi_batch_get_diag(pi_batch* b, int32_t member, int32_t kind, int32_t sp, double* out) {
    pi_status e = check_mem(b, member, "pi_get_diag");
    if (e) return e;
    if (!out) return bfail(b, PI_ERR_ARG, "pi_get_diag: bad argument");
    const MemberDev& d = b->mdh[member];
    const long long G = d.G;
    const unsigned grid = std::min<unsigned>(nblk(G, 256), 1024);
    if (kind == PI_DIAG_PAR) k32_f2d<<<grid, 256, 0, b->stream>>>(b->stage, b->diag_par + d.cell_off, G);
    else if (kind >= PI_DIAG_TRACER && kind < PI_DIAG_TRACER + PI_NTRACERS) {
        if (!(b->tr_mask >> (kind - PI_DIAG_TRACER) & 1u)) return bfail(b, PI_ERR_ARG, "pi_get_diag: tracer diagnostic not enabled");
        k32_f2d<<<grid, 256, 0, b->stream>>>(b->stage, b->diag_tr + (long long)(kind - PI_DIAG_TRACER) * b->Gtot + d.cell_off, G);
    } else if (kind >= PI_DIAG_PROC && kind < PI_DIAG_PROC + PI_NPROC) {
        const int q = kind - PI_DIAG_PROC;
        if (sp < 0 || sp >= b->nsp || !(b->proc_mask >> q & 1u))
            return bfail(b, PI_ERR_ARG, "pi_get_diag: process diagnostic not enabled or bad species");
        k32_fx2d<<<grid, 256, 0, b->stream>>>(b->stage, b->diag_proc + ((long long)sp * PI_NPROC + q) * b->Gtot + d.cell_off, G,
                                              proc_unit(d, q));
    } else {
        if (sp < 0 || sp >= b->nsp || kind < PI_DIAG_NUM || kind > PI_DIAG_DVID) return bfail(b, PI_ERR_ARG, "pi_get_diag: bad kind/species");
        k32_u2d<<<grid, 256, 0, b->stream>>>(b->stage, b->dcnt + ((long long)sp * 4 + (kind - PI_DIAG_NUM)) * b->Gtot + d.cell_off, G);
    }
    BK(cudaGetLastError(), "convert diag");
    BK(cudaMemcpyAsync(out, b->stage, G * sizeof(double), cudaMemcpyDeviceToHost, b->stream), "download diag");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

pi_status pi_batch_check_finite(pi_batch* b, int32_t member) {
    pi_status e = check_mem(b, member, "pi_check_finite");
    if (e) return e;
    const MemberDev& d = b->mdh[member];
    unsigned long long* dq = b->scratch;
    const unsigned long long none = ~0ull;
    unsigned long long q = none;
    for (int n = 0; n < PI_NTRACERS; ++n) {
        BK(cudaMemcpyAsync(dq, &none, sizeof none, cudaMemcpyHostToDevice, b->stream), "check finite");
        k32_first_nonfinite<<<std::min<unsigned>(nblk(d.G, 256), 148 * 4), 256, 0, b->stream>>>(
            b->trbuf[b->cur] + (long long)n * b->Gtot + d.cell_off, d.G, dq);
        BK(cudaGetLastError(), "check finite");
        BK(cudaMemcpyAsync(&q, dq, sizeof q, cudaMemcpyDeviceToHost, b->stream), "check finite");
        BK(cudaStreamSynchronize(b->stream), "synchronize");
        if (q != none) {
            const long long c = (long long)q;
            const long long i = c % d.Gx + 1, j = (c / d.Gx) % d.Gy + 1, k = c / ((long long)d.Gx * d.Gy) + 1;
            return bfail(b, PI_ERR_NAN, "NaN or Inf in tracer " + std::string(tracer_name(n)) + " at (" + std::to_string(i) +
                                            ", " + std::to_string(j) + ", " + std::to_string(k) + ")");
        }
    }
    for (int s = 0; s < b->nsp; ++s) {
        BK(cudaMemcpyAsync(dq, &none, sizeof none, cudaMemcpyHostToDevice, b->stream), "check finite");
        k32_first_nonfinite_inds<<<std::min<unsigned>(nblk(d.C, 256), 148 * 2), 256, 0, b->stream>>>(b->P, d.slot_off + s * d.C, d.C, dq);
        BK(cudaGetLastError(), "check finite");
        BK(cudaMemcpyAsync(&q, dq, sizeof q, cudaMemcpyDeviceToHost, b->stream), "check finite");
        BK(cudaStreamSynchronize(b->stream), "synchronize");
        if (q != none)
            return bfail(b, PI_ERR_NAN, "NaN or Inf in an attribute of individual " + std::to_string(q + 1) + " of species " + std::to_string(s + 1));
    }
    return PI_OK;
}

pi_status pi_batch_reset_diags(pi_batch* b) {
    if (!b) return bfail(b, PI_ERR_ARG, "pi_reset_diags: NULL batch");
    BK(cudaMemsetAsync(b->diag_par, 0, b->Gtot * sizeof(float), b->stream), "reset diags");
    BK(cudaMemsetAsync(b->dcnt, 0, (size_t)b->nsp * 4 * b->Gtot * sizeof(uint32_t), b->stream), "reset diags");
    if (b->diag_tr) BK(cudaMemsetAsync(b->diag_tr, 0, (size_t)PI_NTRACERS * b->Gtot * sizeof(float), b->stream), "reset diags");
    if (b->diag_proc) BK(cudaMemsetAsync(b->diag_proc, 0, (size_t)b->nsp * PI_NPROC * b->Gtot * 8, b->stream), "reset diags");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    return PI_OK;
}

pi_status pi_batch_budget(pi_batch* b, int32_t member, double out[6]) {
    pi_status e = check_mem(b, member, "pi_batch_budget");
    if (e) return e;
    if (!out) return bfail(b, PI_ERR_ARG, "pi_batch_budget: NULL out");
    const MemberDev& d = b->mdh[member];
    const int nb = 512;
    std::vector<double> h(3 * nb);
    k32_budget_cells<<<nb, 256, 0, b->stream>>>(d, b->trbuf[b->cur], b->dzF, b->Gtot, b->partial);
    BK(cudaGetLastError(), "k32_budget_cells");
    BK(cudaMemcpyAsync(h.data(), b->partial, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, b->stream), "download budget");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    for (int r = 0; r < 3; ++r) { double s = 0.0; for (int q = 0; q < nb; ++q) s += h[q * 3 + r]; out[r] = s; }
    k32_budget_inds<<<nb, 256, 0, b->stream>>>(d, b->nsp, b->sp + (size_t)member * b->nsp, b->P, b->partial);
    BK(cudaGetLastError(), "k32_budget_inds");
    BK(cudaMemcpyAsync(h.data(), b->partial, 3 * nb * sizeof(double), cudaMemcpyDeviceToHost, b->stream), "download budget");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    for (int r = 0; r < 3; ++r) { double s = 0.0; for (int q = 0; q < nb; ++q) s += h[q * 3 + r]; out[3 + r] = s; }
    return PI_OK;
}

pi_status pi_batch_guard_stats(pi_batch* b, int64_t* recomputed, int64_t* changed) {
    if (!b) return bfail(b, PI_ERR_ARG, "pi_batch_guard_stats: NULL batch");
    unsigned long long h[2] = {0, 0};
    BK(cudaMemcpyAsync(h, b->guard, sizeof h, cudaMemcpyDeviceToHost, b->stream), "read guard counts");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    if (recomputed) *recomputed = (int64_t)h[0];
    if (changed) *changed = (int64_t)h[1];
    return PI_OK;
}

pi_status pi_selftest_bounded_wait(int64_t limit_ns, int32_t* gave_up, int64_t* waited_ns) {
    if (limit_ns <= 0 || limit_ns > 2000000000LL || !gave_up || !waited_ns) return PI_ERR_ARG;
    int* d = nullptr;
    if (cudaMalloc(&d, 16) != cudaSuccess) return PI_ERR_NOMEM;
    k32_wait_selftest<<<1, 32>>>((unsigned long long)limit_ns, d, (unsigned long long*)(d + 2));
    int h[4] = {0, 0, 0, 0};
    cudaError_t e = cudaMemcpy(h, d, 16, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return PI_ERR_CUDA;
    *gave_up = h[0];
    unsigned long long w = 0;
    memcpy(&w, h + 2, sizeof w);
    *waited_ns = (int64_t)w;
    return PI_OK;
}

pi_status pi_batch_set_option(pi_batch* b, const char* name, int32_t value) {
    if (!b || !name) return bfail(b, PI_ERR_ARG, "pi_batch_set_option: NULL argument");
    struct Opt { const char* name; int Tuning::*field; std::vector<int> values; };
    static const Opt opts[] = {
        { "move_block", &Tuning::bs_move, {128, 256} },
        { "move_fit", &Tuning::occ_move, {2, 3, 4} },
        { "move_blocks_per_sm", &Tuning::persist_move, {0, 2, 4, 8} },
        { "physiology_block", &Tuning::bs_phys, {128, 256} },
        { "physiology_fit", &Tuning::occ_phys, {2, 3, 4} },
        { "physiology_blocks_per_sm", &Tuning::persist_phys, {0, 2, 4, 8} },
        { "xy_rows", &Tuning::ty, {4, 8, 16, 28} },
        { "z_levels", &Tuning::lz, {8, 16, 32, 64} },
        { "par_warps", &Tuning::wpb_par, {1, 2, 4, 8} },
        { "tracer_fused", &Tuning::fused, {0, 1} },
        { "tracer_fused_levels", &Tuning::lz_fused, {8, 16, 32, 64} },
        { "xy_beside_particles", &Tuning::concurrent, {0, 1} },
    };
    for (const Opt& o : opts) {
        if (strcmp(o.name, name)) continue;
        if (std::find(o.values.begin(), o.values.end(), (int)value) == o.values.end())
            return bfail(b, PI_ERR_ARG, std::string("pi_batch_set_option: value not allowed for ") + name);
        b->tune.*o.field = value;
        free_graphs(b);
        return PI_OK;
    }
    return bfail(b, PI_ERR_ARG, std::string("pi_batch_set_option: unknown option ") + name);
}

pi_status pi_batch_set_tracer_kernel(pi_batch* b, int32_t fused, int32_t levels) {
    if (!b || (fused != 0 && fused != 1) || (levels != 8 && levels != 16 && levels != 32 && levels != 64))
        return bfail(b, PI_ERR_ARG, "pi_batch_set_tracer_kernel: fused must be 0 or 1 and levels 8, 16, 32 or 64");
    b->tune.fused = fused;
    b->tune.lz_fused = levels;
    free_graphs(b);
    return PI_OK;
}

pi_status pi_batch_set_sort_interval(pi_batch* b, int32_t steps) {
    if (!b || steps < 0) return bfail(b, PI_ERR_ARG, "pi_batch_set_sort_interval: bad argument");
    b->sort_interval = steps;
    b->need_sort = steps > 0;           // a new cycle starts with a sort before the next step
    return PI_OK;
}

pi_status pi_batch_get_stream(pi_batch* b, void** stream) {
    if (!b || !stream) return bfail(b, PI_ERR_ARG, "pi_get_stream: NULL argument");
    *stream = (void*)b->stream;
    return PI_OK;
}

pi_status pi_batch_profile_enable(pi_batch* b, int32_t on) {
    if (!b) return bfail(b, PI_ERR_ARG, "pi_profile_enable: NULL batch");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    drain(b);
    b->prof_names.clear(); b->prof_count.clear(); b->prof_ms.clear();
    b->profiling = on ? 1 : 0;
    return PI_OK;
}

pi_status pi_batch_profile_read(pi_batch* b, int32_t max, char* names, size_t names_len,
                                int64_t* launches, double* ms, int32_t* n) {
    if (!b || !n) return bfail(b, PI_ERR_ARG, "pi_profile_read: NULL argument");
    BK(cudaStreamSynchronize(b->stream), "synchronize");
    drain(b);
    int32_t k = (int32_t)b->prof_names.size();
    *n = k;
    size_t off = 0;
    for (int32_t q = 0; q < k && q < max; ++q) {
        if (launches) launches[q] = b->prof_count[q];
        if (ms) ms[q] = b->prof_ms[q];
        if (names) {
            const std::string& nm = b->prof_names[q];
            if (off + nm.size() + 1 <= names_len) { memcpy(names + off, nm.c_str(), nm.size() + 1); off += nm.size() + 1; }
        }
    }
    return PI_OK;
}

// Times `k` eager steps per candidate with per-kernel events and keeps, for each knob, the value
// whose kernel ran fastest. Knobs are tuned one after another (coordinate descent).
pi_status pi_batch_autotune(pi_batch* b, double dT, int32_t k, char* report, size_t report_len) {
    if (!b || !(dT > 0) || k < 1) return bfail(b, PI_ERR_ARG, "pi_batch_autotune: bad argument");
    const int was = b->profiling;
    std::string rep;
    // average time per step of the kernels named (a name, or several separated by '|'; "step": the
    // whole step, start to end on the batch stream)
    cudaEvent_t st0 = take_event(b), st1 = take_event(b);
    auto kernel_ms = [&](const char* name, double& out) -> pi_status {
        pi_status e;
        b->profiling = 1;
        b->prof_names.clear(); b->prof_count.clear(); b->prof_ms.clear();
        b->last_dT = dT;
        if ((e = build_tables(b))) return e;
        BK(cudaEventRecord(st0, b->stream), "tuning event");
        for (int i = 0; i < k; ++i) {
            if ((e = maybe_sort(b))) return e;
            if ((e = enqueue_step(b, dT, b->cur))) return e;
            b->cur ^= 1;
            after_step(b);
            b->tracers_dirty = false;
        }
        BK(cudaEventRecord(st1, b->stream), "tuning event");
        BK(cudaStreamSynchronize(b->stream), "synchronize");
        drain(b);
        if ((e = check_errors(b))) return e;
        out = 0.0;
        if (!strcmp(name, "step")) {
            float ms = 0.f;
            BK(cudaEventElapsedTime(&ms, st0, st1), "tuning event");
            out = ms / k;
            return PI_OK;
        }
        const std::string names = std::string("|") + name + "|";
        for (size_t q = 0; q < b->prof_names.size(); ++q)
            if (names.find("|" + b->prof_names[q] + "|") != std::string::npos) out += b->prof_ms[q] / k;
        return PI_OK;
    };
    struct Knob { const char* kernel; int* field; std::vector<int> values; const char* label; int threads_per_value; };
    Tuning& t = b->tune;
    std::vector<Knob> knobs = {
        { "k32_move", &t.occ_move, {2, 3, 4}, "move register fit (blocks of 256 per SM)", 0 },
        { "k32_move", &t.bs_move, {128, 256, 512, 1024}, "move block", 1 },
        { "k32_move", &t.persist_move, {0, 2, 4, 8}, "move blocks/SM (0 = one tile per block)", 0 },
        { "k32_physiology", &t.occ_phys, {2, 3, 4}, "physiology register fit (blocks of 256 per SM)", 0 },
        { "k32_physiology", &t.bs_phys, {128, 256, 512, 1024}, "physiology block", 1 },
        { "k32_physiology", &t.persist_phys, {0, 2, 4, 8}, "physiology blocks/SM (0 = one tile per block)", 0 },
        { "k32_assign", &t.bs_assign, {128, 256, 512, 1024}, "assign block", 1 },
        { "k32_xy", &t.ty, {4, 8, 16, 28}, "x-y tracer tile rows", 0 },
        { "k32_ztail", &t.lz, {8, 16, 32, 64}, "z levels per thread", 0 },
        { "k32_par", &t.wpb_par, {1, 2, 4, 8}, "par warps/block", 32 },
    };
    // the largest block each kernel can be launched with (registers per thread)
    auto max_threads = [](const char* kernel) -> int {
        cudaFuncAttributes fa{};
        const void* f = nullptr;
        if (!strcmp(kernel, "k32_move")) f = (const void*)k32_move<2>;
        else if (!strcmp(kernel, "k32_physiology")) f = (const void*)k32_physiology<2>;
        else if (!strcmp(kernel, "k32_assign")) f = (const void*)k32_assign;
        else if (!strcmp(kernel, "k32_par")) f = (const void*)k32_par;
        if (!f || cudaFuncGetAttributes(&fa, f) != cudaSuccess) return 256;
        return fa.maxThreadsPerBlock;
    };
    free_graphs(b);
    // the knobs of the two-kernel tracer path are tuned on that path
    const int fused0 = t.fused;
    t.fused = 0;
    for (auto& kb : knobs) {
        int best = *kb.field;
        double best_ms = 1e300;
        const int lim = max_threads(kb.kernel);
        for (int v : kb.values) {
            if (kb.threads_per_value && v * kb.threads_per_value > lim) continue;
            *kb.field = v;
            double ms = 0.0;
            pi_status e = kernel_ms(kb.kernel, ms);
            if (e) { b->profiling = was; return e; }
            if (ms > 0.0 && ms < best_ms) { best_ms = ms; best = v; }
        }
        *kb.field = best;
        char line[160];
        snprintf(line, sizeof line, "%s = %d (%.4f ms)\n", kb.label, best, best_ms);
        rep += line;
    }
    // tracer path: k32_tracer (levels per block tuned) against k32_xy + k32_ztail + halo fill
    double two = 0.0;
    pi_status e0 = kernel_ms("k32_xy|k32_ztail|k32_halo", two);
    if (e0) { b->profiling = was; return e0; }
    t.fused = 1;
    int best_lz = t.lz_fused;
    double fused_ms = 1e300;
    for (int v : {8, 16, 32, 64}) {
        t.lz_fused = v;
        double ms = 0.0;
        if ((e0 = kernel_ms("k32_tracer", ms))) { b->profiling = was; return e0; }
        if (ms > 0.0 && ms < fused_ms) { fused_ms = ms; best_lz = v; }
    }
    t.lz_fused = best_lz;
    t.fused = (fused_ms < two) ? 1 : (fused_ms < 1e300 ? 0 : fused0);
    // with the x-y/z kernels: k32_xy beside the particle kernels or after them (whole step timed)
    if (!t.fused) {
        double best_ms = 1e300;
        int best = t.concurrent;
        for (int v : {0, 1}) {
            t.concurrent = v;
            double ms = 0.0;
            if ((e0 = kernel_ms("step", ms))) { b->profiling = was; return e0; }
            if (ms > 0.0 && ms < best_ms) { best_ms = ms; best = v; }
        }
        t.concurrent = best;
        char line[160];
        snprintf(line, sizeof line, "x-y kernel beside the particle kernels = %d (%.4f ms per step)\n", best, best_ms);
        rep += line;
    }
    {
        char line[200];
        snprintf(line, sizeof line, "tracer path = %s (fused %.4f ms at %d levels per block, two-kernel %.4f ms)\n",
                 t.fused ? "k32_tracer" : "k32_xy + k32_ztail", fused_ms < 1e300 ? fused_ms : 0.0, best_lz, two);
        rep += line;
    }
    b->profiling = was;
    b->prof_names.clear(); b->prof_count.clear(); b->prof_ms.clear();
    b->event_pool.push_back(st0);
    b->event_pool.push_back(st1);
    pi_status e = build_tables(b);
    if (e) return e;
    if (report && report_len) {
        size_t n = std::min(report_len - 1, rep.size());
        memcpy(report, rep.c_str(), n);
        report[n] = 0;
    }
    return PI_OK;
}

}  // extern "C"
