/* crq.h -- correctly rounded exp and log for the CPU checkers.
 *
 * TEST INFRASTRUCTURE ONLY.  x87 extended precision first (glibc's expl and
 * logl, about 2^-62 relative error); when that result lies within 2^-60 of
 * the midpoint between two doubles, binary128 (libquadmath's expq/logq,
 * about 2^-112) rounded once to double.  Independent of the decoder's own
 * correctly rounded routines (sogrand_b200/csrc/sg_crmath.h), which the
 * tests check against it.  Host-only; link with -lquadmath -lm.
 */
#pragma once
#include <math.h>
#include <quadmath.h>

static double crq_round(long double y, double x, int is_exp)
{
    double d = (double)y; /* round to nearest */
    if (!(d == d) || d == 0.0 || d > 1.7976931348623157e308 || d < -1.7976931348623157e308)
        return d;
    long double diff = y - (long double)d;
    double nb = nextafter(d, diff > 0 ? INFINITY : -INFINITY);
    long double half = fabsl((long double)nb - (long double)d) / 2;
    if (fabsl(fabsl(diff) - half) > ldexpl(fabsl(y), -60))
        return d;
    __float128 q = is_exp ? expq((__float128)x) : logq((__float128)x);
    return (double)q;
}

static inline double crq_exp(double x)
{
    if (!(x <= 709.782712893384))
        return x != x ? x : INFINITY;
    if (x < -745.2)
        return 0.0;
    return crq_round(expl((long double)x), x, 1);
}

static inline double crq_log(double x)
{
    if (x == 0.0)
        return -INFINITY;
    if (!(x > 0.0))
        return NAN;
    if (x > 1.7976931348623157e308)
        return x;
    return crq_round(logl((long double)x), x, 0);
}
