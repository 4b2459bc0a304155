/* ORACLE build shim (test infrastructure only): gsl_sf_bessel_sequence_Jnu_e
 * for the two orders the reference uses (nu = 1/2, 5/2), evaluated from the
 * closed forms J_{1/2}(x) = sqrt(2/(pi x)) sin x and
 * J_{5/2}(x) = sqrt(2/(pi x)) ((3/x^2 - 1) sin x - 3 cos x / x).
 * On entry v[] holds the arguments, on exit the values. */
#ifndef ORACLE_GSL_SF_BESSEL_SHIM_H
#define ORACLE_GSL_SF_BESSEL_SHIM_H
#include <math.h>
#define GSL_PREC_APPROX 2
static inline int gsl_sf_bessel_sequence_Jnu_e(double nu, int mode, size_t size, double* v) {
  (void)mode;
  for (size_t i = 0; i < size; ++i) {
    double x = v[i];
    if (x == 0) { v[i] = 0; continue; }
    double s = sqrt(2.0 / (M_PI * x));
    if (nu == 0.5) v[i] = s * sin(x);
    else if (nu == 2.5) v[i] = s * ((3.0 / (x * x) - 1.0) * sin(x) - 3.0 * cos(x) / x);
    else return 1;
  }
  return 0;
}
#endif
