/* sg_crmath.h -- correctly rounded binary64 exp and log.
 *
 * The reference decoder (SOGRAND_C/cubic_decoder_final.c) calls libm exp and
 * log about once per tested error pattern, and its guess counts depend on the
 * last bits of those results through the running P_notGuess subtraction.  A
 * correctly rounded exp/log (the double nearest to the exact value) is the
 * one libm behaviour that is defined independently of any implementation, so
 * the decoder uses these: it then equals, bit for bit, the reference source
 * compiled against any correctly rounded libm.
 *
 * Method: Ziv's strategy (A. Ziv, "Fast evaluation of elementary mathematical
 * functions with correctly rounded last bit", ACM TOMS 17(3), 1991), with the
 * table-driven reductions of sg_math.h (Tang, ACM TOMS 15(2), 1989):
 *   fast path  the result as a double-double yh + yl with a proven relative
 *              error bound; if yh + yl +- bound round to the same double, that
 *              double is the correctly rounded result;
 *   near 1     log(x) for |x - 1| < 2^-30 as r - r^2/2 (kept exact) plus a
 *              rounded tail, decided against the exact midpoints: arguments
 *              1 + m 2^-52 (JacLog of large |LLR|) have exact images within
 *              2^-105 of a midpoint;
 *   slow path  (rare) the same reduction evaluated in double-double
 *              arithmetic (Dekker/Knuth error-free transformations) to about
 *              2^-104, followed by the same test at 2^-101.  An argument whose
 *              exact image lies closer than that to a rounding boundary would
 *              still be ambiguous and is rounded from the slow-path value;
 *              such arguments occur with probability about 2^-48.
 * Error bounds (relative to the result; checked against mpmath and a
 * binary128 evaluation by tests/test_math.py): exp fast path 2^-67 (test at
 * 2^-65), log fast path 2^-64 (test at 2^-62), slow paths about 2^-104
 * (measured 2^-104.8 at worst; test at 2^-101).  Subnormal exp results are
 * rounded on their own 2^-1074 grid.
 *
 * Same source on the host (gcc -ffp-contract=off) and the device
 * (nvcc -fmad=false): every fused multiply-add is explicit, so both give the
 * same bits.  The tables are sg_math.h's (pointers to copies, shared memory
 * on the device); the extra constants are in sg_mathtab.h.
 */
#pragma once
#include "sg_math.h"

/* SG_CR_PROBE(kind): optional hook at slow-path entry (1 exp, 2 log), for
 * tests that count how often the slow paths run. */
#ifndef SG_CR_PROBE
#define SG_CR_PROBE(kind)
#endif

/* relative half-widths of the rounding tests (twice the proven error bounds) */
#define SG_CR_EPS_EXP 0x1p-65
#define SG_CR_EPS_LOG 0x1p-62
#define SG_CR_EPS_SLOW 0x1p-101

#if defined(__CUDACC__)
#define SG_NOINL __host__ __device__ __noinline__
#else
#define SG_NOINL static __attribute__((noinline))
#endif

typedef struct {
    double h, l;
} sg_dd;

SG_HD sg_dd sg_dd_mk(double h, double l)
{
    sg_dd r;
    r.h = h;
    r.l = l;
    return r;
}

/* s + *e == a + b exactly, given |a| >= |b| (or a == 0). */
SG_HD double sg_fast_two_sum(double a, double b, double* e)
{
    double s = a + b;
    *e = b - (s - a);
    return s;
}

/* Accurate double-double addition (both operands' low parts summed with
 * their own error terms). */
SG_HD sg_dd sg_dd_add(sg_dd a, sg_dd b)
{
    double s2, t2;
    double s1 = sg_two_sum(a.h, b.h, &s2);
    double t1 = sg_two_sum(a.l, b.l, &t2);
    s2 = s2 + t1;
    s1 = sg_fast_two_sum(s1, s2, &s2);
    s2 = s2 + t2;
    s1 = sg_fast_two_sum(s1, s2, &s2);
    return sg_dd_mk(s1, s2);
}

SG_HD sg_dd sg_dd_mul(sg_dd a, sg_dd b)
{
    double p = a.h * b.h;
    double e = sg_fma(a.h, b.h, -p);
    e = e + (a.h * b.l + a.l * b.h);
    p = sg_fast_two_sum(p, e, &e);
    return sg_dd_mk(p, e);
}

/* Correct rounding of yh + yl (|yl| <= ulp(yh)/2), known to relative error
 * below eps/2: returns 1 with *out = the correctly rounded value when
 * yh + yl +- eps*|yh| round alike, 0 otherwise (*out is then the rounding of
 * yh + yl + eps*|yh|). */
SG_HD int sg_cr_round(double yh, double yl, double eps, double* out)
{
    const double E = fabs(yh) * eps;
    const double a = yh + (yl + E);
    const double b = yh + (yl - E);
    *out = a;
    return a == b;
}

/* Correct rounding of V = y + ye + w, where y + ye is exact with |ye| <=
 * ulp(y)/2 (the output of a TwoSum), y normal and nonzero, and w is known
 * to within Ew with |w| far below ulp(y): V is compared with the midpoints
 * between y and its neighbours exactly, so that a V within a fraction of
 * ulp(ye) of a midpoint is still decided.  Returns 1 with *out when the
 * comparison is decided, 0 otherwise. */
SG_HD int sg_cr_round3(double y, double ye, double w, double Ew, double* out)
{
    const double a = fabs(y);
    const double f = y < 0 ? -ye : ye, g = y < 0 ? -w : w; /* in magnitude space */
    const double a_up = sg_from_bits(sg_bits(a) + 1), a_dn = sg_from_bits(sg_bits(a) - 1);
    const double hu_up = (a_up - a) * 0.5, hu_dn = (a - a_dn) * 0.5;
    /* f - hu_up and f + hu_dn are exact whenever they are small (Sterbenz);
     * otherwise they exceed ulp(y)/4 in magnitude and g cannot change
     * their sign */
    const double d_up = (f - hu_up) + g, d_dn = (f + hu_dn) + g;
    double r;
    if (d_up > Ew)
        r = a_up;
    else if (d_dn < -Ew)
        r = a_dn;
    else if (d_up < -Ew && d_dn > Ew)
        r = a;
    else
        return 0;
    *out = y < 0 ? -r : r;
    return 1;
}

/* The same as sg_cr_round for the value (yh + yl) * 2^e, e <= -1022 (yh in
 * (0.99, 2)): rounded on the subnormal grid 2^-1074, which below 2^-1021 is
 * also the grid of the normal numbers.  force: round the approximation
 * itself. */
SG_HD int sg_cr_round_sub(double yh, double yl, int e, double eps, int force, double* out)
{
    const double sc = sg_pow2i(e + 1074); /* e + 1074 in [-2, 52] */
    const double zh = yh * sc, zl = yl * sc;
    const double m = zh < 0x1p52 ? (zh + 0x1p52) - 0x1p52 : zh; /* an integer nearest zh */
    const double d = (zh - m) + zl;                              /* zh - m is exact */
    const double E = force ? 0.0 : zh * eps;
    double n;
    if (fabs(d) < 0.5 - E)
        n = m;
    else if (d > 0.5 + E)
        n = m + 1.0;
    else if (d < -0.5 - E)
        n = m - 1.0;
    else if (force)
        n = d > 0 ? m + 1.0 : m; /* an exact tie cannot occur for exp */
    else
        return 0;
    *out = n * 0x1p-1074;
    return 1;
}

/* Argument reduction of exp: x = (128 e + j) ln2/128 + r, r = rh + rl to
 * 2^-110 absolute, |r| < 2^-8.5.  kd*C1 and kd*C2 are exact (|kd| < 2^18,
 * 35-bit constants) and x - kd*C1 is exact (Sterbenz). */
SG_HD void sg_exp_reduce(double x, double* rh, double* rl, int* j, int* e)
{
    const double kd0 = x * SG_EXP_INV_LN2_N + SG_EXP_SHIFT;
    const int k = (int)(uint32_t)sg_bits(kd0); /* round(x * 128/ln2) */
    const double kd = kd0 - SG_EXP_SHIFT;
    const double t1 = sg_fma(-kd, SG_CR_EXP_C1, x);
    double re;
    *rh = sg_two_sum(t1, -(kd * SG_CR_EXP_C2), &re);
    *rl = re - kd * SG_CR_EXP_C3;
    *j = k & 127;
    *e = k >> 7;
}

/* exp(x) / 2^e as a double-double to about 2^-104 (e and the reduction as
 * sg_exp_reduce): e^r and 2^(j/128) in double-double arithmetic. */
SG_HD sg_dd sg_exp_cr_dd(double x, const double* tab, int* e)
{
    double rh, rl;
    int j;
    sg_exp_reduce(x, &rh, &rl, &j, e);
    double rle;
    const double r0 = sg_two_sum(rh, rl, &rle);
    const sg_dd r = sg_dd_mk(r0, rle);
    /* 1/6! + r/7! + ... + r^5/11! in double: times r^6 < 2^-51 its rounding
     * stays below 2^-113 */
    double h = sg_fma(r0, SG_CR_EXP_F11, SG_CR_EXP_F10);
    h = sg_fma(r0, h, SG_CR_EXP_F9);
    h = sg_fma(r0, h, SG_CR_EXP_F8);
    h = sg_fma(r0, h, SG_CR_EXP_F7);
    h = sg_fma(r0, h, SG_CR_EXP_F6);
    sg_dd P = sg_dd_mk(h, 0.0);
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_EXP_F5_HI, SG_CR_EXP_F5_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_EXP_F4_HI, SG_CR_EXP_F4_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_EXP_F3_HI, SG_CR_EXP_F3_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_EXP_F2_HI, SG_CR_EXP_F2_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(1.0, 0.0));
    P = sg_dd_mul(P, r); /* e^r - 1 */
    const double H = tab[2 * j];
    const sg_dd T = sg_dd_mk(H, H * tab[2 * j + 1]); /* 2^(j/128) */
    return sg_dd_add(T, sg_dd_mul(T, P));
}

/* exp slow path: the double-double value, rounded. */
SG_NOINL double sg_exp_cr_slow(double x, const double* tab)
{
    SG_CR_PROBE(1);
    int e;
    const sg_dd R = sg_exp_cr_dd(x, tab, &e);
    double y;
    if (e >= -1021) {
        sg_cr_round(R.h, R.l, SG_CR_EPS_SLOW, &y); /* if ambiguous: rounded from R */
        return e <= 1023 ? y * sg_pow2i(e) : (y * sg_pow2i(e - 1)) * 2.0;
    }
    if (!sg_cr_round_sub(R.h, R.l, e, SG_CR_EPS_SLOW, 0, &y))
        sg_cr_round_sub(R.h, R.l, e, 0.0, 1, &y);
    return y;
}

/* Fast path of exp: 2^(j/128) e^r / 2^e = yh + yl to 2^-67 relative. */
SG_HD double sg_exp_cr_fast(double rh, double rl, int j, const double* tab, double* yl)
{
#if defined(__CUDA_ARCH__)
    const double2 Ht = reinterpret_cast<const double2*>(tab)[j];
    const double H = Ht.x, t = Ht.y;
#else
    const double H = tab[2 * j], t = tab[2 * j + 1];
#endif
    /* q = e^r - 1 - r to 2^-69.3 absolute (|r| < 2^-8.5) */
    const double r2 = rh * rh;
    double p = sg_fma(rh, SG_EXP_C7, SG_EXP_C6);
    p = sg_fma(rh, p, SG_EXP_C5);
    p = sg_fma(rh, p, SG_EXP_C4);
    p = sg_fma(rh, p, SG_EXP_C3);
    p = sg_fma(rh, p, SG_EXP_C2);
    const double q = sg_fma(r2, p, rh * rl);
    /* 2^(j/128) e^r = H (1 + t)(1 + rh + rl + q)
     *              = H + H rh + H ((rl + q) + t (1 + rh)) (+ below 2^-104) */
    const double ah = H * rh;
    const double al = sg_fma(H, rh, -ah);
    double se;
    const double s = sg_fast_two_sum(H, ah, &se);
    const double lo = se + (al + H * ((rl + q) + sg_fma(t, rh, t)));
    return sg_fast_two_sum(s, lo, yl);
}

/* Correctly rounded exp(x).  tab: the SG_EXP_TAB_LEN doubles {H_j, t_j} of
 * sg_math.h. */
SG_HD double sg_exp_cr(double x, const double* tab)
{
    if (!(x <= SG_CR_EXP_XMAX)) /* NaN or overflow */
        return x != x ? x : sg_from_bits(0x7ff0000000000000ULL);
    if (x < SG_CR_EXP_XMIN)
        return 0.0;
    double rh, rl, yl, y;
    int j, e;
    sg_exp_reduce(x, &rh, &rl, &j, &e);
    const double yh = sg_exp_cr_fast(rh, rl, j, tab, &yl);
    if (e >= -1021) {
        if (sg_cr_round(yh, yl, SG_CR_EPS_EXP, &y))
            return e <= 1023 ? y * sg_pow2i(e) : (y * sg_pow2i(e - 1)) * 2.0;
    } else if (sg_cr_round_sub(yh, yl, e, SG_CR_EPS_EXP, 0, &y)) {
        return y;
    }
    return sg_exp_cr_slow(x, tab);
}

/* sg_exp_cr for x in [-707.5, 0] (the guess loop's exp(-PM), PM >= 0),
 * where the result is normal: the same operations without the range checks
 * and the subnormal rounding. */
SG_HD double sg_exp_cr_neg(double x, const double* tab)
{
    if (x < -707.5)
        return sg_exp_cr(x, tab);
    double rh, rl, yl, y;
    int j, e;
    sg_exp_reduce(x, &rh, &rl, &j, &e);
    const double yh = sg_exp_cr_fast(rh, rl, j, tab, &yl);
    if (sg_cr_round(yh, yl, SG_CR_EPS_EXP, &y))
        return y * sg_pow2i(e);
    return sg_exp_cr_slow(x, tab);
}

/* Argument reduction of log: x = 2^e z, z in [0.6875, 1.375) in
 * subinterval j; r = z c_j - 1 = rh + rl exactly, |r| < 2^-7.  x must be
 * positive and finite. */
SG_HD void sg_log_reduce(double x, const double* tab, double* rh, double* rl, int* e, int* j)
{
    uint64_t ix = sg_bits(x);
    int escale = 0;
    if (ix < 0x0010000000000000ULL) { /* subnormal: normalise */
        x = x * 0x1p52;
        ix = sg_bits(x);
        escale = -52;
    }
    const uint64_t tmpb = ix - SG_LOG_OFF;
    *j = (int)((tmpb >> 45) & 127);
    *e = (int)((int64_t)tmpb >> 52) + escale;
    const double zz = sg_from_bits(ix - (tmpb & (0xfffULL << 52)));
    const double c = tab[3 * *j];
    const double pr = zz * c;
    const double pe = sg_fma(zz, c, -pr);
    const double pm1 = pr - 1.0; /* exact (Sterbenz) */
    *rh = pm1 + pe;
    *rl = pe - (*rh - pm1);
}

/* log(x) as a double-double to about 2^-104 (x positive and finite):
 * log1p(r), e ln2 and -log(c_j) in double-double arithmetic. */
SG_HD sg_dd sg_log_cr_dd(double x, const double* tab)
{
    double rh, rl;
    int e, j;
    sg_log_reduce(x, tab, &rh, &rl, &e, &j);
    const double lch = tab[3 * j + 1], lcl = tab[3 * j + 2];
    double rle;
    const double r0 = sg_two_sum(rh, rl, &rle);
    const sg_dd r = sg_dd_mk(r0, rle);
    /* -1/10 + r/11 - ... + r^7/17 in double: relative to log1p(r) these
     * terms are below r^9/10 < 2^-66, so their rounding stays below 2^-119;
     * the terms up to r^9 in double-double */
    double h = sg_fma(r0, SG_CR_LOG_G17, SG_CR_LOG_G16);
    h = sg_fma(r0, h, SG_CR_LOG_G15);
    h = sg_fma(r0, h, SG_CR_LOG_G14);
    h = sg_fma(r0, h, SG_CR_LOG_G13);
    h = sg_fma(r0, h, SG_CR_LOG_G12);
    h = sg_fma(r0, h, SG_CR_LOG_G11);
    h = sg_fma(r0, h, SG_CR_LOG_G10);
    sg_dd P = sg_dd_mk(h, 0.0);
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G9_HI, SG_CR_LOG_G9_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G8_HI, SG_CR_LOG_G8_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G7_HI, SG_CR_LOG_G7_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G6_HI, SG_CR_LOG_G6_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G5_HI, SG_CR_LOG_G5_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G4_HI, SG_CR_LOG_G4_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G3_HI, SG_CR_LOG_G3_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(SG_CR_LOG_G2_HI, SG_CR_LOG_G2_LO));
    P = sg_dd_add(sg_dd_mul(P, r), sg_dd_mk(1.0, 0.0));
    P = sg_dd_mul(P, r); /* log1p(r) */
    const double ed = (double)e;
    const double a = ed * SG_LOG_LN2_HI; /* exact */
    const double b = ed * SG_LOG_LN2_LO;
    const double be = sg_fma(ed, SG_LOG_LN2_LO, -b);
    sg_dd E = sg_dd_add(sg_dd_mk(a, 0.0), sg_dd_mk(b, be + ed * SG_CR_LOG_LN2_LO2));
    E = sg_dd_add(E, sg_dd_mk(lch, lcl));
    return sg_dd_add(E, P);
}

/* log slow path: the double-double value, rounded. */
SG_NOINL double sg_log_cr_slow(double x, const double* tab)
{
    SG_CR_PROBE(2);
    const sg_dd R = sg_log_cr_dd(x, tab);
    double y;
    sg_cr_round(R.h, R.l, SG_CR_EPS_SLOW, &y); /* if ambiguous: rounded from R */
    return y;
}

/* Correctly rounded log(x).  tab: the SG_LOG_TAB_LEN doubles
 * {c_j, hi(-log c_j), lo(-log c_j)} of sg_math.h. */
SG_HD double sg_log_cr(double x, const double* tab)
{
    const uint64_t ix = sg_bits(x);
    if (ix - 0x0010000000000000ULL >= 0x7ff0000000000000ULL - 0x0010000000000000ULL) {
        /* zero, subnormal, negative, inf or NaN */
        if (x == 0.0)
            return -1.0 / 0.0;
        if (x != x || x < 0.0)
            return (x - x) / (x - x); /* NaN */
        if (ix == 0x7ff0000000000000ULL)
            return x; /* +inf */
    }
    double rh, rl;
    int e, j;
    sg_log_reduce(x, tab, &rh, &rl, &e, &j);
    const double lch = tab[3 * j + 1];
    const double lcl = tab[3 * j + 2];
    double y, yl;
    if (e == 0 && tab[3 * j] == 1.0 && fabs(rh) < 0x1p-30) {
        /* x within 2^-30 of 1: r = x - 1 exactly, and log(x) = r - r^2/2 +
         * t with t = r^3/3 - r^4/4 (next term below 2^-120 relative).  The
         * first two terms are kept exact (h + u + ue) and only t is
         * rounded, so the rounding test below uses the actual error, not a
         * relative bound. */
        if (rh == 0.0)
            return 0.0; /* log(1) */
        const double s = rh * rh;
        const double se = sg_fma(rh, rh, -s);
        double he, ue, y1e;
        const double h = sg_two_sum(rh, -0.5 * s, &he);
        const double u = sg_two_sum(he, -0.5 * se, &ue);
        const double t = (rh * s) * sg_fma(-0.25, rh, SG_CR_LOG_G3);
        const double y1 = sg_two_sum(h, u, &y1e);
        const double w = ue + t;
        /* w: rounding (2^-53), t's own error (< 2^-50 relative) and the
         * truncation (< 2^-120 of the result), doubled */
        const double Ew = fabs(w) * 0x1p-52 + fabs(t) * 0x1p-49 + fabs(y1) * 0x1p-119;
        if (sg_cr_round3(y1, y1e, w, Ew, &y))
            return y;
        return sg_log_cr_slow(x, tab);
    }
    /* log1p(r) = rh - rh^2/2 + [rl (1 - rh) + rh^3 (1/3 - rh/4 + ... - rh^8/11)],
     * rh^2 = s + se exactly */
    const double s = rh * rh;
    const double se = sg_fma(rh, rh, -s);
    double he;
    const double h = sg_two_sum(rh, -0.5 * s, &he);
    double p = sg_fma(rh, SG_CR_LOG_G11, SG_CR_LOG_G10);
    p = sg_fma(rh, p, SG_CR_LOG_G9);
    p = sg_fma(rh, p, SG_CR_LOG_G8);
    p = sg_fma(rh, p, SG_CR_LOG_G7);
    p = sg_fma(rh, p, SG_CR_LOG_G6);
    p = sg_fma(rh, p, SG_CR_LOG_G5);
    p = sg_fma(rh, p, SG_CR_LOG_G4);
    p = sg_fma(rh, p, SG_CR_LOG_G3);
    const double lo1 = he + (-0.5 * se + (sg_fma(-rl, rh, rl) + (s * rh) * p));
    /* + e ln2 - log(c) */
    const double ed = (double)e;
    const double a = ed * SG_LOG_LN2_HI; /* exact */
    double t1, t2;
    const double s1 = sg_two_sum(a, lch, &t1);
    const double s2 = sg_two_sum(s1, h, &t2);
    const double lo = ((t1 + t2) + (lcl + ed * SG_LOG_LN2_LO)) + lo1;
    const double yh = sg_fast_two_sum(s2, lo, &yl);
    if (sg_cr_round(yh, yl, SG_CR_EPS_LOG, &y))
        return y;
    return sg_log_cr_slow(x, tab);
}
