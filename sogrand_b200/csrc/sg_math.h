/* sg_math.h -- the decoder's own binary64 exp, log and JacLog.
 *
 * The SOGRAND decoder (SOGRAND_C/cubic_decoder_final.c) calls libm exp/log
 * about once per tested error pattern.  Its hard decisions, guess counts and
 * iteration counts do not depend on the last bit of those results, but its
 * soft values do.  So that the CUDA kernel and a CPU restatement can be
 * compared bit for bit, both evaluate exp and log with the routines below,
 * which use only IEEE-754 add, multiply, fused multiply-add and bit
 * manipulation: the same source gives the same bits on x86-64 and on sm_100a.
 *
 * Methods (published, restated here in own code):
 *  - exp: Tang's table-driven method (ACM TOMS 15(2), 1989) with a 128-entry
 *    table of 2^(j/128) held as H_j*(1+t_j), Cody-Waite reduction
 *    r = x - k*ln2/128 in two parts, and the Taylor series of e^r to r^7.
 *  - log: x = 2^e * z with z in [0.6875, 1.375) taken from the bit pattern,
 *    a 128-entry table of reciprocals c_j, r = z*c_j - 1 formed exactly in
 *    double-double (TwoProduct by FMA), log(x) = e*ln2 - log(c_j) + log1p(r)
 *    with the Taylor series of log1p to r^9 and a double-double sum.
 * Accuracy (measured against mpmath by tests/test_math.py): both below
 * 0.51 ulp over the decoder's argument ranges; subnormal exp results may be
 * off by one subnormal ulp (double rounding), which the decoder never uses.
 *
 * Tables live in sg_mathtab.h (generated by gen_mathtab.py).  Device code
 * passes pointers to shared-memory copies so that divergent lanes index
 * them without constant-cache serialisation.
 *
 * This translation unit must be compiled without floating-point contraction
 * (-ffp-contract=off on the host, -fmad=false on the device): every fused
 * multiply-add below is explicit.
 */
#pragma once
#include <stdint.h>
#include "sg_mathtab.h"

#if defined(__CUDACC__)
#define SG_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#define SG_HD static inline
#endif

#define SG_EXP_TAB_LEN 256 /* 128 x {H_j, t_j} */
#define SG_LOG_TAB_LEN 384 /* 128 x {c_j, hi, lo} */

SG_HD uint64_t sg_bits(double x)
{
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    memcpy(&b, &x, 8);
    return b;
#endif
}

SG_HD double sg_from_bits(uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, 8);
    return x;
#endif
}

SG_HD double sg_fma(double a, double b, double c)
{
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

/* 2^e for e in [-1022, 1023], exactly. */
SG_HD double sg_pow2i(int e)
{
    return sg_from_bits((uint64_t)(int64_t)(e + 1023) << 52);
}

/* exp(x), round-to-nearest result within ~0.505 ulp.
 * tab: SG_EXP_TAB_LEN doubles, {H_j, t_j} interleaved. */
SG_HD double sg_exp(double x, const double* tab)
{
    if (!(x <= 709.782712893384)) /* NaN or overflow */
        return x != x ? x : sg_from_bits(0x7ff0000000000000ULL);
    if (x < -745.1332191019412)
        return 0.0;
    double z = x * SG_EXP_INV_LN2_N;
    double kd = z + SG_EXP_SHIFT;
    int k = (int)(uint32_t)sg_bits(kd); /* round(z), two's complement in the low word */
    kd = kd - SG_EXP_SHIFT;
    double r = sg_fma(-kd, SG_EXP_LN2_N_HI, x); /* exact */
    r = sg_fma(-kd, SG_EXP_LN2_N_LO, r);
    int j = k & 127;
    int e = k >> 7; /* floor(k / 128) */
    double H = tab[2 * j];
    double t = tab[2 * j + 1];
    double r2 = r * r;
    double p = sg_fma(r, SG_EXP_C7, SG_EXP_C6);
    p = sg_fma(r, p, SG_EXP_C5);
    p = sg_fma(r, p, SG_EXP_C4);
    p = sg_fma(r, p, SG_EXP_C3);
    p = sg_fma(r, p, SG_EXP_C2);
    p = p * r2;                   /* e^r - 1 - r */
    double u = sg_fma(t, r, t);   /* t * (1 + r) */
    double tmp = r + (u + p);     /* (1 + t) e^r - 1 */
    if (e >= -1021 && e <= 1022) {
        double S = sg_from_bits(sg_bits(H) + ((uint64_t)(int64_t)e << 52));
        return sg_fma(S, tmp, S);
    }
    /* Near overflow or underflow: scale in two exact steps.  A subnormal
     * result is rounded twice. */
    int e1 = e > 0 ? e - 64 : e + 64;
    double S = sg_from_bits(sg_bits(H) + ((uint64_t)(int64_t)e1 << 52));
    double y = sg_fma(S, tmp, S);
    return e > 0 ? y * 0x1p64 : y * 0x1p-64;
}

/* exp(x) for x <= 0, bit-identical to sg_exp: the same operations without
 * the range checks that cannot fire for arguments above -707.5 (the guess
 * loop's exp(-PM), PM >= 0). */
SG_HD double sg_exp_neg(double x, const double* tab)
{
    if (x < -707.5)
        return sg_exp(x, tab);
    double z = x * SG_EXP_INV_LN2_N;
    double kd = z + SG_EXP_SHIFT;
    int k = (int)(uint32_t)sg_bits(kd);
    kd = kd - SG_EXP_SHIFT;
    double r = sg_fma(-kd, SG_EXP_LN2_N_HI, x);
    r = sg_fma(-kd, SG_EXP_LN2_N_LO, r);
    int j = k & 127;
    int e = k >> 7;
#if defined(__CUDA_ARCH__)
    const double2 Ht = reinterpret_cast<const double2*>(tab)[j];
    const double H = Ht.x, t = Ht.y;
#else
    const double H = tab[2 * j], t = tab[2 * j + 1];
#endif
    double r2 = r * r;
    double p = sg_fma(r, SG_EXP_C7, SG_EXP_C6);
    p = sg_fma(r, p, SG_EXP_C5);
    p = sg_fma(r, p, SG_EXP_C4);
    p = sg_fma(r, p, SG_EXP_C3);
    p = sg_fma(r, p, SG_EXP_C2);
    p = p * r2;
    double u = sg_fma(t, r, t);
    double tmp = r + (u + p);
    double S = sg_from_bits(sg_bits(H) + ((uint64_t)(int64_t)e << 52));
    return sg_fma(S, tmp, S);
}

/* TwoSum: s + err == a + b exactly. */
SG_HD double sg_two_sum(double a, double b, double* err)
{
    double s = a + b;
    double bb = s - a;
    *err = (a - (s - bb)) + (b - bb);
    return s;
}

/* log(x), round-to-nearest result within ~0.502 ulp.
 * tab: SG_LOG_TAB_LEN doubles, {c_j, hi(-log c_j), lo(-log c_j)}. */
SG_HD double sg_log(double x, const double* tab)
{
    uint64_t ix = sg_bits(x);
    int escale = 0;
    if (ix - 0x0010000000000000ULL >= 0x7ff0000000000000ULL - 0x0010000000000000ULL) {
        /* zero, subnormal, negative, inf or NaN */
        if (x == 0.0)
            return -1.0 / 0.0;
        if (x != x || x < 0.0)
            return (x - x) / (x - x); /* NaN */
        if (ix == 0x7ff0000000000000ULL)
            return x; /* +inf */
        x = x * 0x1p52; /* subnormal: normalise */
        ix = sg_bits(x);
        escale = -52;
    }
    uint64_t tmpb = ix - SG_LOG_OFF;
    int j = (int)((tmpb >> 45) & 127);
    int e = (int)((int64_t)tmpb >> 52) + escale;
    double zz = sg_from_bits(ix - (tmpb & (0xfffULL << 52)));
    double c = tab[3 * j];
    double lch = tab[3 * j + 1];
    double lcl = tab[3 * j + 2];
    /* r_hi + r_lo = z*c - 1 exactly */
    double pr = zz * c;
    double pe = sg_fma(zz, c, -pr);
    double pm1 = pr - 1.0; /* exact (Sterbenz) */
    double rh = pm1 + pe;
    double rl = pe - (rh - pm1); /* |pm1| >= |pe| unless pm1 == 0, where rl = 0 */
    double r2 = rh * rh;
    double q = sg_fma(rh, SG_LOG_C9, SG_LOG_C8);
    q = sg_fma(rh, q, SG_LOG_C7);
    q = sg_fma(rh, q, SG_LOG_C6);
    q = sg_fma(rh, q, SG_LOG_C5);
    q = sg_fma(rh, q, SG_LOG_C4);
    q = sg_fma(rh, q, SG_LOG_C3);
    q = sg_fma(rh, q, SG_LOG_C2);
    double poly = r2 * q; /* log1p(r) - r */
    double ed = (double)e;
    double a = ed * SG_LOG_LN2_HI; /* exact */
    double t1, t2;
    double s1 = sg_two_sum(a, lch, &t1);
    double s2 = sg_two_sum(s1, rh, &t2);
    double lo = ((t1 + t2) + (lcl + sg_fma(ed, SG_LOG_LN2_LO, rl))) + poly;
    return s2 + lo;
}

