// Internal declarations shared by the host orchestration (pib200.cu) and the device kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pib200.h"
#include "../../include/pi_numerics.h"

// Float32 literals of the reference that appear inside Float64 arithmetic (see the kernels that
// use them for the reference line each comes from).
#define F_1em30 ((double)1.0e-30f)
#define F_RGAS  ((double)8.3145f)
#define F_T0    ((double)273.15f)
#define F_4em2  ((double)4.0e-2f)
#define F_1em4  ((double)1.0e-4f)
#define F_1em2  ((double)1.0e-2f)
#define F_1em1  ((double)1.0e-1f)
#define F_5em2  ((double)0.05f)
#define F_CHL   ((double)893.49f)      // mg Chl per mmol (MacroMolecularMode)
#define F_2em3  ((double)2.0e-3f)
#define F_1em3  ((double)1.0e-3f)
#define F_1em5  ((double)1.0e-5f)
#define F_1em6  ((double)1.0e-6f)
#define F_0p99  ((double)0.99f)
#define F_THMAX ((double)1.0e20f)
#define F_1em20 ((double)1.0e-20f)

// physiology modes of an FP64 model
#define MODE_QUOTA  0
#define MODE_CARBON 1
#define MODE_MACRO  2
#define MODE_IRON   3

// process diagnostics of the largest mode (MacroMolecularMode): sizes of the per-species buffers
#define PI_MAXPROC PI_NIPROC     // the most processes of any mode (IronEnergyMode's 32)

// Device error word bits (sticky until pi_synchronize reads and clears them).
#define PI_DEVERR_DOMAIN   1u
#define PI_DEVERR_CAPACITY 2u
#define PI_DEVERR_ABIO     4u   // with CAPACITY: the overflow was of abiotic particle slots
#define PI_DEVERR_MAXPTC   8u   // with CAPACITY: a merge into a species without max_ptc

// Per-individual flag byte: ac plus the three 0/1 decisions carried to the next step.
#define FL_AC   1u
#define FL_GRAZ 2u
#define FL_MORT 4u
#define FL_DVID 8u

// Per-step status byte.
#define ST_AC0  1u   // active when cells were found (find_inds!/find_NPT! time)

// Grid description passed by value to kernels. Indices inside kernels are the reference's
// 1-based, halo-inclusive (i, j, k).
struct DGrid {
    int Nx, Ny, Nz, Hx, Hy, Hz, Gx, Gy, Gz;
    int tx, ty, tz;
    int all_water;
    double dx, dy;
    const double* dzF;     // Gz
    const double* dzC;     // Gz
    const uint8_t* lm;     // G
    long long G;
    // LatLonGrid metrics (lat_lon_grid.jl:1-45), null for a RectilinearGrid: dxC, dyC, dxF, dyF,
    // Az over the Gx·Gy columns, Ax, Ay, Vol over the G cells
    const double *mdxC, *mdyC, *mdxF, *mdyF, *mAz, *mAx, *mAy, *mVol;
};

__host__ __device__ __forceinline__ int gidx(const DGrid& g, int i, int j, int k) {
    return (i - 1) + g.Gx * ((j - 1) + g.Gy * (k - 1));
}

// Packed (xi, yi, zi) with 0 <= xi <= Gx etc.: xi + (Gx+1)*(yi + (Gy+1)*zi).
__host__ __device__ __forceinline__ int32_t pack_cell(const DGrid& g, int xi, int yi, int zi) {
    return xi + (g.Gx + 1) * (yi + (g.Gy + 1) * zi);
}
__host__ __device__ __forceinline__ void unpack_cell(const DGrid& g, int32_t c, int& xi, int& yi, int& zi) {
    xi = c % (g.Gx + 1);
    int r = c / (g.Gx + 1);
    yi = r % (g.Gy + 1);
    zi = r / (g.Gy + 1);
}

// Device pointers of one species (FP64 plain form).
struct SpcDev {
    double *x, *y, *z, *Sz, *Bm, *Cq, *Nq, *Pq, *Chl, *gen, *age;
    double* Bd;         // CarbonMode damaged biomass (NULL for QuotaMode)
    // MacroMolecularMode pools (NULL otherwise): protein, DNA, RNA, carbohydrate/lipid, N and P reserves
    double *PRO, *DNA, *RNA, *CH, *NST, *PST;
    double* ptc;        // abiotic particles held (every mode)
    // IronEnergyMode quotas, excess energy and time since sunset (NULL otherwise; CH above)
    double *qNO3, *qNH4, *qP, *qFe, *qFePS, *qFeNR, *qFeNF, *exEn, *tdark;
    uint8_t* flags;
    int32_t* cell;      // packed (xi, yi, zi)
    uint8_t* stat;      // ST_* bits of the current step
};

// One abiotic species (Abiotic/particle_generation.jl:2-5): positions, activity and the packed
// find_inds! cell of `capacity` slots.
struct AbioDev {
    double *x, *y, *z;
    uint8_t* ac;
    int32_t* cell;
};

struct SpcParams {      // pi_quota_params on the device
    pi_quota_params p;
};

struct FluxBCDev {
    int kind;
    int n1, n2;
    long long nt;
    const double* v;
};

// Per-step work arrays shared by the kernels.
struct StepBufs {
    uint32_t* cnt;          // G+1 counts of active individuals per cell
    uint32_t* off;          // G+1 exclusive prefix of cnt
    uint32_t* key;          // nsp*C cell key (G-linear) per individual, sentinel when inactive
    uint32_t* key_sorted;   // nsp*C
    uint32_t* gid_sorted;   // nsp*C: gid = sp*C + slot sorted by (cell, gid)
    int32_t* pos;           // nsp*C: position of gid in gid_sorted (valid when ST_AC0)
    double* contrib;        // 5 per entry: DIC, DOC, NH4, NO3, PO4 consumption
    double* loss;           // 6 per entry: DOC, DON, DOP, POC, PON, POP loss
    uint8_t* evk;           // per entry: 0 none, 1 grazing loss, 2 mortality loss
    unsigned long long* flag64;   // C: (is_div << 32) | is_free
    unsigned long long* rank64;   // C: exclusive prefix of flag64
    int32_t* divlist;       // C
    int32_t* freelist;      // C
    uint32_t* ndiv;         // 1
    uint32_t* err;          // device error word
    int64_t* err_iter;      // iteration at which a capacity error occurred
};
