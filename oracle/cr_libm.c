/* cr_libm.c -- correctly rounded exp and log under the names sgcr_exp /
 * sgcr_log, for the reference built against a correctly rounded libm.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the unmodified
 * reference decoder with cr_libm.h force-included, which binds its exp and
 * log calls to these, giving the reference as it behaves under a correctly
 * rounded libm (oracle/_ref/libsgref_cr.so).  A correctly rounded function
 * is unique, so any correct implementation gives the same bits; these use
 * the decoder's routines (sogrand_b200/csrc/sg_crmath.h), which
 * tests/test_math.py checks against the independent binary128 evaluation
 * of crq.h and against mpmath (crq.h itself is too slow for the hundreds of
 * millions of calls a fixture set makes).  Every other libm function the
 * reference calls (pow, sqrt, round, ceil, floor, fabs, fmax, fmin) is
 * exact in glibc for the arguments it passes. */
#include "../sogrand_b200/csrc/sg_crmath.h"

static const double k_etab[SG_EXP_TAB_LEN] = SG_EXP_TAB_INIT;
static const double k_ltab[SG_LOG_TAB_LEN] = SG_LOG_TAB_INIT;

double sgcr_exp(double x) { return sg_exp_cr(x, k_etab); }
double sgcr_log(double x) { return sg_log_cr(x, k_ltab); }
