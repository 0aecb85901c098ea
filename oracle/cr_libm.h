/* cr_libm.h -- force-included (gcc -include) ahead of the unmodified
 * reference source: after <math.h> has declared libm, every later use of
 * exp and log in the source names the correctly rounded routines of
 * cr_libm.c instead.  TEST INFRASTRUCTURE ONLY. */
#include <math.h>
double sgcr_exp(double x);
double sgcr_log(double x);
#define exp sgcr_exp
#define log sgcr_log
