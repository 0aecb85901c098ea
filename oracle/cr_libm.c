/* cr_libm.c -- the correctly rounded exp and log of crq.h under the names
 * sgcr_exp / sgcr_log.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the unmodified
 * reference decoder with cr_libm.h force-included, which binds its exp and
 * log calls to these, giving the reference as it behaves under a correctly
 * rounded libm (oracle/_ref/libsgref_cr.so).  Every other libm function the
 * reference calls (pow, sqrt, round, ceil, floor, fabs, fmax, fmin) is exact
 * in glibc for the arguments it passes. */
#include "crq.h"

double sgcr_exp(double x) { return crq_exp(x); }
double sgcr_log(double x) { return crq_log(x); }
