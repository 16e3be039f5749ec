/*
 * pi_numerics.h — numeric primitives shared bit-for-bit by the host and the device.
 *
 * The model time step of PlanktonIndividuals.jl is restated twice in this project: once as the
 * CUDA kernels of libpib200 and once as the CPU oracle used by the tests. Both must produce the
 * same IEEE-754 double bits, so every primitive whose result is not fixed by IEEE-754 itself
 * (exp, integer powers, the random draws) and every Julia semantic that differs from C's
 * (min/max, isless, mod, Bool * Float) is defined here once, with plain IEEE operations only.
 * Compile the host with -ffp-contract=off and the device with -fmad=false so no multiply-add is
 * contracted behind the code's back.
 *
 *  - Random draws: Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel
 *    random numbers: as easy as 1, 2, 3", SC'11). The reference fills C-length arrays with
 *    rand!(rng_type(arch), ·) (src/Individuals/Advection/particle_diffusion.jl:18-20,
 *    src/Individuals/Plankton/division_death_probability.jl:97-99); here the draw for one slot is
 *    a pure function of (seed, iteration, species, purpose, slot), so both sides see the same
 *    numbers. Each value is a 24-bit integer times 2^-24, exact in float and double.
 *  - pi_exp: Cody–Waite reduction x = k ln2 + r (W. J. Cody and W. Waite, Software Manual for the
 *    Elementary Functions, 1980) with ln2 split into a 32-bit head and a tail, then the degree-14
 *    Taylor polynomial of e^r (|r| <= ln2/2, truncation error < 3e-18) in Horner form, then an
 *    exact scaling by 2^k. Coefficients are 1/n! rounded to double. Reference `exp` is Julia
 *    1.12.2 Base.Math (not vendored); ULP-level agreement with it is not pinned.
 *  - pi_pow_int: Julia 1.12 Base.Math `^(x::Float64, n)` for small integer n takes the
 *    compensated power-by-squaring path (`pow_body`: Dekker two-product with an error term carried
 *    beside each square, one fused multiply-add at the end). The reference raises to 4.0f0 and
 *    2.0f0 in its shape functions (src/Individuals/utils.jl:109-137); this restates that method.
 *  - pi_log: x = m·2^e by frexp (exact) with m in [√½, √2), then log x = e·ln2 + 2·atanh(s),
 *    s = (m − 1)/(m + 1), the atanh by its odd Taylor series through s^25 (|s| < 0.1716, truncation
 *    < 1e-20) in Horner form, ln2 split as in pi_exp. pi_pow(x, y) = pi_exp(y·pi_log(x)) for x >= 0,
 *    for the reference's non-integer powers (Sz^(2/3), IronEnergyMode/growth_kernels.jl:48);
 *    agreement with Julia's correctly rounded pow is to a few ulp and not pinned.
 *  - Julia semantics: `min`/`max` propagate NaN and order -0.0 < 0.0; `isless` orders NaN last;
 *    `x * b::Bool` is `ifelse(b, x, copysign(0, x))`; `mod(x, 1)` is `rem` moved into [0, 1).
 */
#ifndef PI_NUMERICS_H
#define PI_NUMERICS_H

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define PI_HD __host__ __device__ __forceinline__
#else
#define PI_HD static inline
#endif

/* ------------------------------------------------------------------------------------------ */
/* Julia floating-point semantics                                                               */
/* ------------------------------------------------------------------------------------------ */

PI_HD int pi_isnan(double x) { return x != x; }

PI_HD int pi_signbit(double x) {
    union { double d; uint64_t u; } v; v.d = x; return (int)(v.u >> 63);
}

/* Julia Base: max(x, y) = isnan(x)|isnan(y) ? x - y : (signbit(x - y) ? y : x) */
PI_HD double jl_max(double x, double y) {
    double d = x - y;
    if (pi_isnan(x) || pi_isnan(y)) return d;
    return pi_signbit(d) ? y : x;
}

/* Julia Base: min(x, y) = isnan(x)|isnan(y) ? x - y : (signbit(x - y) ? x : y) */
PI_HD double jl_min(double x, double y) {
    double d = x - y;
    if (pi_isnan(x) || pi_isnan(y)) return d;
    return pi_signbit(d) ? x : y;
}

/* Julia isless on floats: total order -Inf < ... < -0.0 < 0.0 < ... < Inf < NaN. */
/* isequal(x, y): NaN equals NaN, -0.0 differs from 0.0 */
PI_HD int jl_isequal(double x, double y) {
    if (x != x || y != y) return (x != x) && (y != y);
    return x == y && signbit(x) == signbit(y);
}

PI_HD int jl_isless(double x, double y) {
    if (pi_isnan(x)) return 0;
    if (pi_isnan(y)) return 1;
    if (x == y) return pi_signbit(x) && !pi_signbit(y);
    return x < y;
}

/* Julia x * b for x::Float64, b::Bool: ifelse(b, x, copysign(0.0, x)). */
PI_HD double jl_mulb(double x, int b) { return b ? x : copysign(0.0, x); }

/* Julia mod(x, 1.0): r = rem(x, 1); r == 0 ? copysign(r, 1) : (r < 0 ? r + 1 : r).
 * rem(x, 1) is computed as x - trunc(x): exact for finite x (Sterbenz: trunc(x) is within a factor
 * of two of x when |x| >= 1, and 0 otherwise), NaN for infinite or NaN x, like fmod. */
PI_HD double jl_mod1(double x) {
    double r = x - trunc(x);
    if (r == 0.0) return 0.0;
    if ((r > 0.0) != (1.0 > 0.0)) return r + 1.0;
    return r;
}

/* Julia unsafe_trunc(Int, x) for finite x within range; NaN maps to 0 (the reference's value is
 * unspecified there, and the callers flag it as an out-of-domain position). */
PI_HD int64_t jl_trunc(double x) {
    if (pi_isnan(x)) return 0;
    if (x >= 9.2e18) return (int64_t)9.2e18;
    if (x <= -9.2e18) return -(int64_t)9.2e18;
    return (int64_t)x;
}

/* ------------------------------------------------------------------------------------------ */
/* exp                                                                                          */
/* ------------------------------------------------------------------------------------------ */

PI_HD double pi_pow2i(int k) {
    /* 2^k for k in [-1022, 1023], built from the exponent field. */
    union { uint64_t u; double d; } v;
    v.u = (uint64_t)(k + 1023) << 52;
    return v.d;
}

PI_HD double pi_exp(double x) {
    if (pi_isnan(x)) return x;
    if (x > 0x1.62e42fefa39efp+9) return INFINITY;   /* > ln(DBL_MAX) */
    if (x < -0x1.74910d52d3052p+9) return 0.0;       /* < ln(2^-1075)  */
    const double inv_ln2 = 0x1.71547652b82fep+0;
    const double ln2_hi  = 0x1.62e42fee00000p-1;     /* ln 2, 32 significant bits */
    const double ln2_lo  = 0x1.a39ef35793c76p-33;    /* ln 2 - ln2_hi              */
    const double shifter = 0x1.8p52;                 /* round-to-nearest-even via 1.5*2^52 */
    double kd = (x * inv_ln2 + shifter) - shifter;
    double r = (x - kd * ln2_hi) - kd * ln2_lo;
    double p = 0x1.93974a8c07c9dp-37;                /* 1/14! */
    p = p * r + 0x1.6124613a86d09p-33;               /* 1/13! */
    p = p * r + 0x1.1eed8eff8d898p-29;               /* 1/12! */
    p = p * r + 0x1.ae64567f544e4p-26;               /* 1/11! */
    p = p * r + 0x1.27e4fb7789f5cp-22;               /* 1/10! */
    p = p * r + 0x1.71de3a556c734p-19;               /* 1/9!  */
    p = p * r + 0x1.a01a01a01a01ap-16;               /* 1/8!  */
    p = p * r + 0x1.a01a01a01a01ap-13;               /* 1/7!  */
    p = p * r + 0x1.6c16c16c16c17p-10;               /* 1/6!  */
    p = p * r + 0x1.1111111111111p-7;                /* 1/5!  */
    p = p * r + 0x1.5555555555555p-5;                /* 1/4!  */
    p = p * r + 0x1.5555555555555p-3;                /* 1/3!  */
    p = p * r + 0.5;                                 /* 1/2!  */
    p = p * r + 1.0;
    p = p * r + 1.0;
    int k = (int)kd;
    if (k > 1023) { p = p * 0x1p1023; k -= 1023; }
    if (k < -1022) { p = p * 0x1p-1022; k += 1022; }
    return p * pi_pow2i(k);
}

PI_HD double pi_log(double x) {
    if (pi_isnan(x) || x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (x == INFINITY) return x;
    int e = 0;
    double m = frexp(x, &e);                          /* x = m·2^e, m in [0.5, 1) */
    if (m < 0x1.6a09e667f3bcdp-1) { m = m * 2.0; e -= 1; }
    const double ln2_hi = 0x1.62e42fee00000p-1, ln2_lo = 0x1.a39ef35793c76p-33;
    double f = m - 1.0, s = f / (2.0 + f), z = s * s;
    double t = 1.0 / 25.0;
    t = t * z + 1.0 / 23.0; t = t * z + 1.0 / 21.0; t = t * z + 1.0 / 19.0; t = t * z + 1.0 / 17.0;
    t = t * z + 1.0 / 15.0; t = t * z + 1.0 / 13.0; t = t * z + 1.0 / 11.0; t = t * z + 1.0 / 9.0;
    t = t * z + 1.0 / 7.0; t = t * z + 1.0 / 5.0; t = t * z + 1.0 / 3.0;
    double lm = 2.0 * s + 2.0 * s * (z * t);
    double ed = (double)e;
    return ed * ln2_hi + (lm + ed * ln2_lo);
}

PI_HD double pi_pow(double x, double y) {
    if (x == 0.0) return y > 0.0 ? 0.0 : (y == 0.0 ? 1.0 : INFINITY);
    return pi_exp(y * pi_log(x));
}

/* ------------------------------------------------------------------------------------------ */
/* Integer powers with Julia's compensated power-by-squaring                                    */
/* ------------------------------------------------------------------------------------------ */

PI_HD double pi_fma(double a, double b, double c) { return fma(a, b, c); }

/* x^n for 1 <= n <= 4, as Julia's pow_body(x, n): square-and-multiply on (value, error) pairs. */
PI_HD double pi_pow_int(double x, int n) {
    if (n == 3) return x * x * x;
    double y = 1.0, ynlo = 0.0, xnlo = 0.0;
    while (n > 1) {
        if (n & 1) {
            double err = pi_fma(y, xnlo, x * ynlo);
            double hi = x * y;
            double lo = pi_fma(x, y, -hi);
            y = hi; ynlo = lo + err;
        }
        double err = x * 2.0 * xnlo;
        double hi = x * x;
        double lo = pi_fma(x, x, -hi);
        x = hi; xnlo = lo + err;
        n >>= 1;
    }
    double err = pi_fma(y, xnlo, x * ynlo);
    int fin = !pi_isnan(x - x) && !pi_isnan(err - err);
    return fin ? pi_fma(x, y, err) : x * y;
}

/* ------------------------------------------------------------------------------------------ */
/* Philox4x32-10 counter-based draws                                                            */
/* ------------------------------------------------------------------------------------------ */

PI_HD uint32_t pi_mulhilo32(uint32_t a, uint32_t b, uint32_t* hi) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    return (uint32_t)p;
}

PI_HD void pi_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, hi1;
        uint32_t lo0 = pi_mulhilo32(0xD2511F53u, c0, &hi0);
        uint32_t lo1 = pi_mulhilo32(0xCD9E8D57u, c2, &hi1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        if (r < 9) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Draw purposes: one Philox block gives the three draws of one call site for one slot. */
enum { PI_DRAW_DIFFUSION = 0,   /* rnd.x, rnd.y, rnd.z of particle_diffusion!          */
       PI_DRAW_DECISION  = 1,   /* rnd.x, rnd.y, rnd.z of get_probability! (graz, mort, dvid) */
       PI_DRAW_ABIO_DIFFUSION = 2,   /* particle_diffusion! of abiotic species `species`     */
       PI_DRAW_ABIO_BC   = 3,   /* rnd_3d of particles_from_bcs! (abiotic species, cell)    */
       PI_DRAW_RELEASE   = 4 }; /* rnd.x of get_release_probability! (release pair, slot)   */

/* Three uniforms in [0, 1) on the 2^-24 lattice for (seed, iteration, species, purpose, slot). */
PI_HD void pi_draw3(uint64_t seed, uint32_t iteration, uint32_t species, uint32_t purpose,
                    uint32_t slot, double* r0, double* r1, double* r2) {
    uint32_t ctr[4] = { slot, iteration, (species & 0xFFFFu) | (purpose << 16), 0x706c6b74u };
    uint32_t key[2] = { (uint32_t)seed, (uint32_t)(seed >> 32) };
    uint32_t o[4];
    pi_philox4x32_10(ctr, key, o);
    const double s = 0x1p-24;
    *r0 = (double)(o[0] >> 8) * s;
    *r1 = (double)(o[1] >> 8) * s;
    *r2 = (double)(o[2] >> 8) * s;
}

#endif /* PI_NUMERICS_H */
