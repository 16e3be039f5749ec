// FP32 form: declarations shared by the FP32 kernels and their host orchestration.
//
// A batch is a set of independent members (each with its own grid, individuals, tracers, forcing
// and seed) that step together: every phase of the step is one launch over all members. A single
// FP32 model is a batch of one member.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pib200.h"
#include "../../include/pi_numerics.h"

// Individual flag byte (carried between steps): ac and the three decisions of get_probability!.
#define F32_AC   1u
#define F32_GRAZ 2u
#define F32_MORT 4u
#define F32_DVID 8u
// Status byte: ac at cell-lookup time in this step, and "the find_inds! cell differs from the
// cell of the position" (daughters in their birth step, uploaded states).
#define F32_ST_AC0   1u
#define F32_ST_STALE 2u

// Device error word bits.
#define F32_ERR_DOMAIN   1u
#define F32_ERR_CAPACITY 2u
#define F32_ERR_FORCING  4u
#define F32_ERR_LISTS    8u     // a division list entry outside its segment (access skipped)
#define F32_ERR_TIMEOUT  16u    // a bounded wait for staged data gave up

// Slots are processed in tiles of this many consecutive slots of one (member, species) segment.
#define F32_TILE 1024

// Per-member description used by the kernels.
struct MemberDev {
    int Nx, Ny, Nz, Hx, Hy, Hz, Gx, Gy, Gz;
    int tx, ty, tz;
    int all_water;
    int any_bc;
    float dx, dy;
    float rdx, rdy;         // 1/dx, 1/dy
    int cbx, cby;           // bit widths of ci and cj in an interior cell code
    int hbx, hby;           // bit widths of xi and yi in a find_inds! (halo) cell code
    long long cell_off;     // first cell of the member's halo-padded grid in the batch cell space
    long long G;            // (Nx+2Hx)(Ny+2Hy)(Nz+2Hz)
    long long col_off;      // first of the member's Nx*Ny surface columns
    long long slot_off;     // first slot of species 0; species s starts at slot_off + s*C
    long long C;            // capacity per species
    int dz_off;             // first of the member's Gz levels in dzF/dzC
    int bc_off;             // first of the member's 14*6 flux boundary conditions
    long long woff;         // first word of species 0 in the logical-slot bitmaps
    long long wps;          // bitmap words per species (32 per tile of F32_TILE slots)
    long long bin_off;      // first cell-sort bin of species 0 (Nx*Ny*Nz + tiles bins per species)
    uint64_t seed;
    double fx_unit;         // mmol per fixed-point unit of the particle→grid mass sums
    double chl_unit;        // mg Chl per fixed-point unit of the Chl sums
    double fx_inv;          // 1 / fx_unit
    double chl_inv;         // 1 / chl_unit
};

// Cell codes: three indices in bit fields of one int32 (a, b, c from the low bits up, widths of a
// and b given), so that unpacking takes shifts and masks.
__host__ __device__ inline int32_t f32_pack(int a, int b, int c, int ba, int bb) {
    return (int32_t)((unsigned)a | ((unsigned)b << ba) | ((unsigned)c << (ba + bb)));
}
__host__ __device__ inline void f32_unpack(int32_t code, int ba, int bb, int& a, int& b, int& c) {
    const unsigned u = (unsigned)code;
    a = (int)(u & ((1u << ba) - 1u));
    b = (int)((u >> ba) & ((1u << bb) - 1u));
    c = (int)(u >> (ba + bb));
}
// bits needed for the values 0..v
inline int f32_bits(long long v) { int b = 1; while ((1LL << b) <= v) ++b; return b; }

// Forcing of a member for the current step.
struct MemberForcing {
    const float* vel0[3];   // halo-padded velocity of the previous step
    const float* vel1[3];   // halo-padded velocity of this step
    const float* velh[3];   // (vel0 + vel1) / 2, or vel1 itself when vel0 and vel1 are the same field
    const float* temp;      // halo-padded temperature
};

// Forcing time series resident on the device (PlanktonSimulation's arrays), or none.
struct MemberSeries {
    const float* vel;       // nvel snapshots of 3 halo-padded fields (u, v, w), G each
    long long nvel;
    double dT_vel;
    const float* parf;      // npar snapshots of Nx*Ny
    long long npar;
    double dT_PAR;
    const float* temp;      // ntemp halo-padded snapshots
    long long ntemp;
    double dT_temp;
    int has_series;
    int has_vel;
    int time_offset;        // bit 0 vel, bit 1 PAR, bit 2 temp: index by the step within the call
    float* velh_buf[3];     // scratch for vel½ (member-local fields)
};

// Step counters on the device (graph replay needs no host argument).
struct StepState {
    int64_t iteration;      // model.iteration
    double t;               // model.t
    int64_t call_step;      // steps taken in the current update! call (time_offset indexing)
    int64_t err_iter;       // iteration at which a capacity error occurred
    int32_t err_member;     // member of that error
    int32_t pad;
};

// Individuals of all members and species.
//
// Storage order. Each (member, species) segment of `capacity` slots is stored in a physical order
// that a periodic counting sort keeps grouped by cell, so that neighbouring threads read
// neighbouring velocity corners and add into neighbouring cell sums. Every slot keeps its logical
// slot number (the reference's array index), which keys its random draws and orders the division
// bookkeeping, so no result depends on the physical order. Arrays below are indexed by physical
// position unless stated.
struct IndDev32 {
    int32_t* cell;          // interior cell of the position: ci + (Nx+1)(cj + (Ny+1) ck); -1 inactive
    int32_t* scell;         // find_inds! cell (xi + (Gx+1)(yi + (Gy+1) zi)) when F32_ST_STALE
    float *ox, *oy, *oz;    // in-cell offsets, in [0, 1)
    float *Bm, *Cq, *Nq, *Pq, *Chl, *age, *gen;
    uint8_t* flags;
    uint8_t* stat;
    int32_t* lslot;         // logical slot (within the segment) held at this physical position
    // indexed by logical slot (shared by both physical buffers)
    int32_t* phys;          // physical position (within the segment) of each logical slot
    uint32_t* freebits;     // bit set: the logical slot is inactive (MemberDev::woff layout)
    uint32_t* dvbits;       // bit set: the logical slot divides in this step
};

struct SpeciesDev32 {
    float Nsuper, Cquota, Chl2Cint, alpha, Phi, Topt, Tmax, Ea;
    float PCmax, VDOCmax, VNO3max, VNH4max, VPO4max;
    float KsatDOC, KsatNH4, KsatNO3, KsatPO4, Cqmax, Nqmax, Pqmax;
    float Chl2N, R_NC, R_PC, k_mtb, respir, grz_P, dvid_P, dvid_reg, dvid_reg2;
    float mort_P, mort_reg, grazFracC, grazFracN, grazFracP, mortFracC, mortFracN, mortFracP;
    int dvid_type;
    float OGT_rate;         // exp(-Ea / (R (Topt + 273.15))), a constant of the species
};

// Float64 parameters of the decision probabilities, for the guard band of k32_physiology.
struct SpeciesDec64 {
    double grz_P, mort_P, mort_reg, dvid_P, dvid_reg, dvid_reg2, CqNs;   // CqNs = Cquota·Nsuper
    int dvid_type;
};

struct BgcDev32 {
    float kw, kc, kDOC, Nit, kDON, kDOP, kPOC, kPON, kPOP;
    float kappa_h, kappa_v, kappa_hP, kappa_vP;
    int shared_graz;
    float w_sink_org, w_sink_inorg, lambda_POC, lambda_min, kdiss, lambda_dust, lambda_Fe, ligand, DFeFrac;
};

struct FluxBC32 {
    int kind;
    int n1, n2;
    long long nt;
    const float* v;
};

// Per-cell fixed-point accumulators of the particle→grid sums (zeroed as they are consumed).
enum { ACC_DIC = 0, ACC_NH4, ACC_NO3, ACC_PO4, ACC_DOC, ACC_DON, ACC_DOP, ACC_POC, ACC_PON, ACC_POP, ACC_N };
