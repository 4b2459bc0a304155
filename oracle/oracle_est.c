/*
 * ORACLE -- test infrastructure only.  CPU FP64 restatement of the a-priori
 * Ewald / SPME error estimates (rectangular box), the checker of the GPU sums.
 * RE = longRange.hetero/profile.test/template/tools/real.error:
 *  - ElectrostaticInteraction::errorEstimatePME (version 3)  RE/src/ElectrostaticInteraction.cpp:349-401
 *  - ElectrostaticInteraction_rec_BSpline::errorEstimate    RE/src/EleRecBSpline.cpp:154-206
 *  - EleEcalculator tables (produce4Item)                   RE/src/EleEcalculator.cpp:100-220
 */
#include <math.h>

/* real-space and Ewald-truncation estimates; c2 = sum q^2 */
void orc_error_estimate_pme(const double box[3], const int K[3], double beta, double rcut, double c2,
                            int natom, double* err_dir, double* err_rec) {
  const double V = box[0] * box[1] * box[2];
  *err_dir = 2 * sqrt(c2 / (double)natom) * sqrt(c2 / rcut / V) * exp(-beta * beta * rcut * rcut);
  double sum = 0;
  for (int m0 = -K[0]; m0 <= K[0]; ++m0)
    for (int m1 = -K[1]; m1 <= K[1]; ++m1)
      for (int m2 = -K[2]; m2 <= K[2]; ++m2) {
        if (m0 >= -K[0] / 2 && m0 <= K[0] / 2 && m1 >= -K[1] / 2 && m1 <= K[1] / 2 &&
            m2 >= -K[2] / 2 && m2 <= K[2] / 2)
          continue;
        double mx = m0 / box[0], my = m1 / box[1], mz = m2 / box[2];
        double mm = mx * mx + my * my + mz * mz;
        sum += exp(-2 * M_PI * M_PI / beta / beta * mm) / mm;
      }
  *err_rec = sqrt(sum / (double)natom) * 2 * c2 / V;
}

static double ipow(int n, double x) {
  double v = 1;
  for (int i = 0; i < n; ++i) v *= x;
  return v;
}

static double terms(double x, int n, int first, int last, int mode) {
  /* mode 0: sum over l of 1/(x+2 pi l)^n + 1/(x-2 pi l)^n, l = first..last
     mode 1: sum l (1/(x+2 pi l)^n - 1/(x-2 pi l)^n);  mode 2: sum l^2 (...+...) */
  double s = 0;
  for (int l = first; l <= last; ++l) {
    double a = 1. / ipow(n, x + 2 * M_PI * l), b = 1. / ipow(n, x - 2 * M_PI * l);
    if (l == 0) { s += 1. / ipow(n, x); continue; }
    if (mode == 0) s += a + b;
    else if (mode == 1) s += (a - b) * l;
    else s += (a + b) * l * l;
  }
  return s;
}

/* produce4Item: e1 = -S6/D, e2 = (S6^2 + S6(2n))/D^2 with S6 the |l| = 1..5
   aliasing sum and D the |l| <= 7 sum */
void orc_ecal_e1e2(double x, int n, double* e1, double* e2) {
  if (x == 0) { *e1 = *e2 = 0; return; }
  double s6 = terms(x, n, 1, 5, 0);
  double de = terms(x, n, 0, 7, 0);
  *e1 = -s6 / de;
  *e2 = (s6 * s6 + terms(x, 2 * n, 1, 5, 0)) / (de * de);
}

/* homogeneous ik-SPME interpolation error estimate */
double orc_error_estimate_spme_ik(const double box[3], const int K[3], int n, double beta, double c2,
                                  int natom) {
  const double V = box[0] * box[1] * box[2];
  double sum = 0;
  for (int m0 = -K[0] / 2; m0 < K[0] / 2; ++m0)
    for (int m1 = -K[1] / 2; m1 < K[1] / 2; ++m1)
      for (int m2 = -K[2] / 2; m2 < K[2] / 2; ++m2) {
        if (!m0 && !m1 && !m2) continue;
        double mx = m0 / box[0], my = m1 / box[1], mz = m2 / box[2];
        double mm = mx * mx + my * my + mz * mz;
        double e1[3], e2[3];
        orc_ecal_e1e2(2 * M_PI * m0 / (double)K[0], n, &e1[0], &e2[0]);
        orc_ecal_e1e2(2 * M_PI * m1 / (double)K[1], n, &e1[1], &e2[1]);
        orc_ecal_e1e2(2 * M_PI * m2 / (double)K[2], n, &e1[2], &e2[2]);
        double ees = e2[0] + e2[1] + e2[2] + 2 * e1[0] * e1[1] + 2 * e1[0] * e1[2] + 2 * e1[1] * e1[2];
        double s = e1[0] + e1[1] + e1[2];
        double expp = exp(-2 * M_PI * M_PI / beta / beta * mm) / mm * 2 / V * 2 / V;
        sum += 2 * expp * (ees + s * s);
      }
  sum *= c2 * c2 / (double)natom;
  return sqrt(sum);
}
