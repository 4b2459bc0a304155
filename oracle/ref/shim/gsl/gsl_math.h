/* ORACLE build shim (test infrastructure only): the GSL math helpers used by
 * the md.error reference sources.  x^n by binary exponentiation. */
#ifndef ORACLE_GSL_MATH_SHIM_H
#define ORACLE_GSL_MATH_SHIM_H
#include <math.h>
static inline double gsl_pow_int(double x, int n) {
  unsigned un;
  if (n < 0) { x = 1.0 / x; un = (unsigned)(-n); } else un = (unsigned)n;
  double v = 1.0;
  do { if (un & 1) v *= x; un >>= 1; x *= x; } while (un);
  return v;
}
static inline double gsl_pow_2(const double x) { return x * x; }
static inline double gsl_pow_3(const double x) { return x * x * x; }
static inline double gsl_pow_4(const double x) { double x2 = x * x; return x2 * x2; }
static inline double gsl_pow_5(const double x) { double x2 = x * x; return x2 * x2 * x; }
static inline double gsl_pow_6(const double x) { double x2 = x * x; return x2 * x2 * x2; }
#endif
