// IronEnergyMode physiology in the FP64 plain form — IronEnergyMode/plankton_growth.jl:2-26,
// growth_kernels.jl:1-337, division_death_probability.jl:7-107, calc_consume! (consume_loss.jl:2-9).
// Every expression is in the reference's operation order (the library is built with -fmad=false).
#pragma once

#include "kernels_fp64.cuh"

namespace pib {

__device__ __forceinline__ double i_tempFunc(double T, const pi_iron_params& p) {      // growth_kernels.jl:12-17
    double k = jl_max(0.0, pi_exp(-p.Ea / (F_RGAS * (T + F_T0))));
    return jl_min(1.0, k / pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0))));
}
__device__ __forceinline__ double i_tempFunc_CF(double T, const pi_iron_params& p) {   // :2-9
    double x = T - p.Topt, xmax = p.Tmax - p.Topt;
    double k = pi_exp(-p.Ea / (F_RGAS * (T + F_T0))) * shape_dec(x, xmax, F_4em2, 4);
    k = jl_max(0.0, k);
    return jl_min(1.0, k / pi_exp(-p.Ea / (F_RGAS * (p.Topt + F_T0))));
}

// Every slot is updated: the light reaction, the iron allocation and the dark clock carry no ac,
// so the state of an inactive slot keeps changing as in the reference, from zero light,
// temperature and nutrients unless it was active when they were gathered (find_NPT!, with the
// change of PAR since the previous step).
__global__ void k_physiology_iron(DGrid g, SpcDev P, pi_iron_params p, long long C, int s,
                                  double dT, double t, uint64_t seed, uint32_t iter, int shared_graz,
                                  const double* __restrict__ NH4f, const double* __restrict__ NO3f,
                                  const double* __restrict__ PO4f, const double* __restrict__ DFef,
                                  const double* __restrict__ par, const double* __restrict__ par0,
                                  const double* __restrict__ temp, const uint32_t* __restrict__ off,
                                  const uint32_t* __restrict__ gid_sorted, const int32_t* __restrict__ pos,
                                  double* __restrict__ contrib, double* __restrict__ d_num,
                                  double* __restrict__ procv, const uint32_t* err) {
    long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= C) return;
    if (*err & PI_DEVERR_CAPACITY) return;
    const int ac = P.flags[slot] & FL_AC;
    const int ac0 = P.stat[slot] & ST_AC0;
    double NH4 = 0.0, NO3 = 0.0, PO4 = 0.0, DFe = 0.0, parv = 0.0, dpar = 0.0, T = 0.0, pop = 0.0;
    if (ac0) {                                         // find_NPT! (utils.jl:14-25), × ac at gathering
        int xi, yi, zi;
        unpack_cell(g, P.cell[slot], xi, yi, zi);
        const int c = gidx(g, xi, yi, zi);
        NH4 = jl_max(0.0, NH4f[c]); NO3 = jl_max(0.0, NO3f[c]); PO4 = jl_max(0.0, PO4f[c]); DFe = jl_max(0.0, DFef[c]);
        parv = par[c]; dpar = par[c] - par0[c]; T = temp[c];
        if (shared_graz) {
            pop = (double)(off[c + 1] - off[c]);
        } else {
            uint32_t n = 0;
            for (uint32_t q = off[c]; q < off[c + 1]; ++q) n += (gid_sorted[q] / (uint32_t)C) == (uint32_t)s;
            pop = (double)n;
        }
    }
    const double nfx = p.is_croc + p.is_tric;
    const double Bm = P.Bm[slot], Sz = P.Sz[slot], Chl = P.Chl[slot], tdark = P.tdark[slot];
    double CH = P.CH[slot], qNH4 = P.qNH4[slot], qNO3 = P.qNO3[slot], qP = P.qP[slot], qFe = P.qFe[slot];
    const double qFePS = P.qFePS[slot], qFeNR = P.qFeNR[slot], qFeNF = P.qFeNF[slot];
    // calc_trs_uptake_kernel! (growth_kernels.jl:56-66) with calc_NH4/NO3/P/Fe_uptake (:20-53)
    double reg = shape_dec(qNH4 / jl_max(F_1em30, Bm + CH), p.qNH4max, F_1em4, 2);
    double VNH4 = jl_mulb(p.VNH4max * reg * NH4 / jl_max(F_1em30, NH4 + p.KsatNH4) * i_tempFunc(T, p) * Bm, ac);
    VNH4 = jl_min(VNH4, NH4 / dT / jl_max(1.0, pop)) * p.is_nr;
    reg = shape_dec(qNO3 / jl_max(F_1em30, Bm + CH), p.qNO3max, F_1em4, 2);
    double VNO3 = jl_mulb(p.VNO3max * reg * NO3 / jl_max(F_1em30, NO3 + p.KsatNO3) * i_tempFunc(T, p) * Bm, ac);
    VNO3 = jl_min(VNO3, NO3 / dT / jl_max(1.0, pop)) * p.is_nr;
    reg = shape_dec((qP + Bm * p.R_PC) / jl_max(F_1em30, Bm + CH), p.qPmax, F_1em4, 2);
    double VPO4 = jl_mulb(p.VPO4max * reg * PO4 / jl_max(F_1em30, PO4 + p.KsatPO4) * i_tempFunc(T, p) * Bm, ac);
    VPO4 = jl_min(VPO4, PO4 / dT / jl_max(1.0, pop));
    reg = shape_dec((qFe + qFePS + qFeNF + qFeNR) / jl_max(F_1em30, Bm + CH), p.qFemax, F_1em4, 2);
    const double SA = p.SA * pi_pow(Sz, (double)(2.0f / 3.0f));
    double VFe = jl_mulb(p.KSAFe * SA * DFe * reg * p.Nsuper * i_tempFunc(T, p), ac);
    VFe = jl_min(VFe, DFe / dT / jl_max(1.0, pop));
    // update_state_1_kernel! (:73-79)
    qP += VPO4 * dT; qNO3 += VNO3 * dT; qNH4 += VNH4 * dT; qFe += VFe * dT;
    // calc_PS (:87-93)
    const double aI = parv * p.alpha * Chl / jl_max(F_1em30, Bm);
    const double Qfe_ps = qFePS / jl_max(F_1em30, Bm + CH);
    const double PS = p.PCmax * (1.0 - pi_exp(-aI)) * Bm * (Qfe_ps / jl_max(F_1em30, Qfe_ps + p.KfePS));
    // calc_respir (:106-111)
    double RS = jl_mulb(CH * p.k_rs * i_tempFunc(T, p), ac);
    RS = jl_min(RS, CH / dT);
    double ERS = jl_mulb(RS * p.e_rs, ac);
    // calc_CF (:125-131)
    reg = shape_dec(CH / jl_max(F_1em30, Bm + CH), p.CHmax, F_1em4, 2);
    double CF = jl_mulb(p.k_cf * reg * i_tempFunc_CF(T, p) * Bm, ac);
    double ECF = jl_mulb(CF * p.e_cf, ac);
    // calc_NR (:145-155) and calc_NF (:167-176), both regulated by the same NH4 quota
    reg = shape_dec(qNH4 / jl_max(F_1em30, Bm + CH), p.qNH4max, F_1em4, 2);
    const double Qfe_NR = qFeNR / jl_max(F_1em30, Bm + CH);
    double NR = jl_mulb(p.k_nr * reg * qNO3 * (Qfe_NR / jl_max(F_1em30, Qfe_NR + p.KfeNR)) * i_tempFunc(T, p), ac);
    NR = jl_min(NR, qNO3 / dT);
    double ENR = jl_mulb(NR * p.e_nr, ac);
    NR = NR * p.is_nr; ENR = ENR * p.is_nr;
    const double Qfe_NF = qFeNF / jl_max(F_1em30, Bm + CH);
    double NF = jl_mulb(p.k_nf * reg * (Qfe_NF / jl_max(F_1em30, Qfe_NF + p.KfeNF)) * i_tempFunc(T, p) * Bm, ac);
    double ENF = jl_mulb(NF * p.e_nf, ac);
    NF = NF * nfx; ENF = ENF * nfx;
    // energy_alloc (:190-197), energy_allocation_kernel! (:198-206)
    const double ECFt = jl_min(PS, ECF);
    const double ENFt = jl_min(ENF, PS + ERS - ECFt) * nfx;
    const double ENRt = jl_min(ENR, PS + ERS - ECFt) * p.is_nr;
    const double ERSt = jl_min(ERS, jl_max(0.0, ECFt + ENFt + ENRt - PS));
    const double exEn = jl_max(0.0, PS - ECFt - ENFt - ENRt);
    ERS = ERSt; ECF = ECFt; ENF = ENFt; ENR = ENRt;
    RS = ERS / p.e_rs; CF = ECF / p.e_cf; NF = ENF / p.e_nf; NR = ENR / p.e_nr;
    // update_state_2_kernel! (:213-219)
    CH += (CF - RS) * dT;
    qNO3 += -NR * dT;
    qNH4 += NR * dT;
    qNH4 += NF * dT;
    // calc_ρChl_kernel! (:227-231), calc_BS_kernel! (:239-243)
    const double rChl = jl_mulb(jl_mulb(p.Chl2N / jl_max(F_1em30, parv * p.alpha * Chl / Bm), jl_isless(F_1em1, parv)), ac);
    const double BS = jl_mulb(jl_min(jl_min(CH, qNH4 / p.R_NC), qP / p.R_PC) * p.k_mtb, ac);
    // iron_alloc (:251-283): Bool·Bool is a Bool, Bool + Bool an Int
    const int pos_dpar = jl_isless(0.0, dpar), neg_dpar = jl_isless(dpar, 0.0), dark = jl_isequal(0.0, parv);
    const int light = jl_isless(0.0, parv), early = jl_isless(tdark, p.NF_clock), late = jl_isless(p.NF_clock, tdark);
    double ST2PS = jl_mulb(p.k_Fe_ST2PS * qFe, pos_dpar);
    double PS2ST = p.k_Fe_PS2ST * qFePS * (double)(neg_dpar + dark);
    double ST2NR = jl_mulb(jl_mulb(p.k_Fe_ST2NR * qFe, dark), early) * p.is_nr;
    double NR2ST = p.k_Fe_NR2ST * qFeNR * (double)((dark & late) + light) * p.is_nr;
    const double ST2NF_cr = jl_mulb(jl_mulb(p.k_Fe_ST2NF * qFe, dark), early);
    const double NF2ST_cr = p.k_Fe_NF2ST * qFeNF * (double)((dark & late) + light);
    const double ST2NF_tr = jl_mulb(p.k_Fe_ST2NF * qFe, pos_dpar);
    const double NF2ST_tr = p.k_Fe_NF2ST * qFeNF * (double)(neg_dpar + dark);
    double ST2NF = ST2NF_cr * p.is_croc + ST2NF_tr * p.is_tric;
    double NF2ST = NF2ST_cr * p.is_croc + NF2ST_tr * p.is_tric;
    ST2PS = jl_min(ST2PS, qFe / dT);
    PS2ST = jl_min(PS2ST, qFePS / dT);
    ST2NR = jl_min(ST2NR, qFe / dT - ST2PS);
    NR2ST = jl_min(NR2ST, qFeNR / dT);
    ST2NF = jl_min(ST2NF, qFe / dT - ST2PS);
    NF2ST = jl_min(NF2ST, qFeNF / dT);
    // update_biomass_kernel! (:296-312), update_cellsize_kernel! (:322-325), update_tdark_kernel! (:333-337)
    const double Bm1 = Bm + dT * BS;
    CH -= dT * BS;
    qNH4 -= dT * BS * p.R_NC;
    qP -= dT * BS * p.R_PC;
    const double Chl1 = Chl + dT * BS * p.R_NC * rChl;
    const double age = P.age[slot] + jl_mulb(dT / 3600.0, ac);
    const double qFe1 = qFe + dT * (PS2ST - ST2PS + NR2ST - ST2NR + NF2ST - ST2NF);
    const double qFePS1 = qFePS + dT * (ST2PS - PS2ST);
    const double qFeNR1 = qFeNR + dT * (ST2NR - NR2ST);
    const double qFeNF1 = qFeNF + dT * (ST2NF - NF2ST);
    const double Sz1 = Bm1 / (p.Cquota * p.Nsuper);
    const double tdark1 = tdark * (1.0 - (double)light) + jl_mulb(dT, dark);
    // calc_graz_quadratic!, calc_mort!, calc_dvid!, get_probability! (division_death_probability.jl)
    const double graz = jl_mulb(pop * p.grz_P, ac);
    const double mort = jl_mulb(p.mort_P * shape_dec(Sz1, p.mort_reg, F_1em5, 4), ac);
    double dv;
    const int ty = (int)p.dvid_type;
    if (ty == 1) dv = p.dvid_P * shape_inc(Sz1, p.dvid_reg, F_2em3, 2);
    else if (ty == 2) dv = p.dvid_P * shape_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg, F_1em5, 4);
    else dv = p.dvid_P * shape_inc(Sz1, p.dvid_reg, F_1em3, 4) * shape_inc(fmod(t, 86400.0) / 3600.0, p.dvid_reg2, F_1em5, 4);
    const double dvid = jl_mulb(dv, ac);
    double r0, r1, r2;
    pi_draw3(seed, iter, (uint32_t)s, PI_DRAW_DECISION, (uint32_t)slot, &r0, &r1, &r2);
    const int dg = jl_isless(r0, graz * dT) && ac;
    const int dm = jl_isless(r1, mort * dT) && ac;
    const int dd = jl_isless(r2, dvid * dT) && ac;
    P.Bm[slot] = Bm1; P.CH[slot] = CH; P.qNH4[slot] = qNH4; P.qNO3[slot] = qNO3; P.qP[slot] = qP;
    P.Chl[slot] = Chl1; P.age[slot] = age; P.qFe[slot] = qFe1; P.qFePS[slot] = qFePS1; P.qFeNR[slot] = qFeNR1;
    P.qFeNF[slot] = qFeNF1; P.Sz[slot] = Sz1; P.tdark[slot] = tdark1; P.exEn[slot] = exEn;
    P.flags[slot] = (uint8_t)((ac ? FL_AC : 0) | (dg ? FL_GRAZ : 0) | (dm ? FL_MORT : 0) | (dd ? FL_DVID : 0));
    // calc_consume_kernel! (consume_loss.jl:2-9): DIC, NH4, NO3, PO4, DFe per binned individual
    if (ac0) {
        double* K = contrib + (long long)pos[(long long)s * C + slot] * 5;
        K[0] = jl_mulb((RS - PS) * dT, ac);
        K[1] = jl_mulb(-VNH4 * dT, ac);
        K[2] = jl_mulb(-VNO3 * dT, ac);
        K[3] = jl_mulb(-VPO4 * dT, ac);
        K[4] = jl_mulb(-VFe * dT, ac);
    }
    // diags_spcs! (Diagnostics/diagnostics_kernels.jl:22-23) in PI_IPROC_* order
    if (procv) {
        const double v[PI_NIPROC] = { PS, CF, ECF, RS, ERS, NR, ENR, NF, ENF, BS, VNH4, VNO3, VPO4, VFe,
                                      PS2ST, ST2PS, NR2ST, ST2NR, NF2ST, ST2NF, Bm1, exEn, CH, qNO3, qNH4, qP,
                                      qFe1, qFePS1, qFeNR1, qFeNF1, Chl1, tdark1 };
        for (int q = 0; q < PI_NIPROC; ++q) procv[(long long)q * C + slot] = v[q];
    }
    if (ac) {
        int xi, yi, zi;
        unpack_cell(g, P.cell[slot], xi, yi, zi);
        atomicAdd(&d_num[gidx(g, xi, yi, zi)], 1.0);
    }
}

// Individuals' C (Bm + CH), N (Bm·R_NC + qNO3 + qNH4) and P (Bm·R_PC + qP): block partials.
__global__ void k_budget_inds_iron(SpcDev P, long long C, double R_NC, double R_PC, double* __restrict__ part) {
    double c = 0.0, n = 0.0, q = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < C; i += (long long)gridDim.x * blockDim.x)
        if (P.flags[i] & FL_AC) {
            c += P.Bm[i] + P.CH[i];
            n += P.Bm[i] * R_NC + P.qNO3[i] + P.qNH4[i];
            q += P.Bm[i] * R_PC + P.qP[i];
        }
    __shared__ double sh[3][256];
    sh[0][threadIdx.x] = c; sh[1][threadIdx.x] = n; sh[2][threadIdx.x] = q;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int r = 0; r < 3; ++r) sh[r][threadIdx.x] += sh[r][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) for (int r = 0; r < 3; ++r) part[blockIdx.x * 3 + r] = sh[r][0];
}

}  // namespace pib
