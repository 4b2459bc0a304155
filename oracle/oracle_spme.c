/*
 * ORACLE -- test infrastructure only.  CPU FP64 restatement of the md.error
 * reciprocal / real-space electrostatics, used as the checker of the GPU SPME
 * chain.  Rectangular boxes.
 *
 * Follows (RE = longRange.hetero/profile.test/template/tools/real.error):
 *  - cardinal B-spline M_n and its derivative     RE/include/Polynominal.h:172-720
 *  - calB |b(m)|^2                                 RE/src/EleRecBSpline.cpp:729-796
 *  - calPsiFPhiF (ik) / FBSpline calPsiFPhiF       RE/src/EleRecBSpline.cpp:799-877,
 *                                                  RE/src/EleRecFBSpline.cpp:1146-1195
 *  - calQ spread, ik gather, energy                RE/src/EleRecBSpline.cpp:393-619
 *  - analytic-differentiation gather               RE/src/EleRecFBSpline.cpp:771-907
 *  - exact reciprocal Ewald sum                    RE/src/EleRecES.cpp:49-144
 *  - real-space pair term and self energy          RE/src/EleDir.cpp:43-61,
 *                                                  RE/src/ElectrostaticInteraction.cpp:219-222
 * B-spline weights use the standard recursion M_k(u) = (u M_{k-1}(u) +
 * (k-u) M_{k-1}(u-1))/(k-1) (Essmann et al., J. Chem. Phys. 103, 8577 (1995)).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_dft3d(const int n[3], double* data, int sign);

/* M_n(f + j), j = 0..n-1, and derivatives, for f in [0,1) */
void orc_bspline_weights(int n, double f, double* w, double* dw) {
  double m[16];
  memset(m, 0, sizeof(m));
  m[0] = f; m[1] = 1.0 - f;                 /* order 2: M2(f) = f, M2(f+1) = 1-f */
  for (int k = 3; k <= n; ++k) {
    if (k == n && dw) {                     /* M_n' (f+j) = M_{n-1}(f+j) - M_{n-1}(f+j-1) */
      for (int j = 0; j < n; ++j) dw[j] = (j < n - 1 ? m[j] : 0.0) - (j > 0 ? m[j - 1] : 0.0);
    }
    double t[16];
    for (int j = 0; j < k; ++j) {
      double u = f + j;
      double a = (j < k - 1) ? m[j] : 0.0;
      double b = (j > 0) ? m[j - 1] : 0.0;
      t[j] = (u * a + (k - u) * b) / (k - 1);
    }
    for (int j = 0; j < k; ++j) m[j] = t[j];
  }
  if (n == 2 && dw) { dw[0] = 1.0; dw[1] = -1.0; }
  for (int j = 0; j < n; ++j) w[j] = m[j];
}

/* cardinal B-spline value M_n(x) on [0, n] */
double orc_bspline(int n, double x) {
  if (x <= 0 || x >= n) return 0.0;
  double f = x - floor(x);
  int j = (int)floor(x);
  double w[16];
  orc_bspline_weights(n, f, w, NULL);
  return w[j];
}

/* |b_d(m)|^2 of calB */
void orc_spme_bmod(int n, int K, double* b) {
  for (int m = 0; m < K; ++m) {
    double re = 0, im = 0;
    for (int k = 0; k < n - 1; ++k) {
      double s = orc_bspline(n, k + 1.0);
      re += s * cos(2 * M_PI * m * k / (double)K);
      im += s * sin(2 * M_PI * m * k / (double)K);
    }
    b[m] = 1.0 / (re * re + im * im);
  }
}

static int wrapi(int k, int K) { return k < 0 ? k + K : (k >= K ? k - K : k); }

/* Q = sum_i q_i prod_d M_n(u_d - k_d), u_d = K_d x_d / L_d (calQ) */
void orc_spme_spread(int natom, const double* pos, const double* q, const double box[3], const int K[3],
                     int n, double* Q) {
  memset(Q, 0, sizeof(double) * (size_t)K[0] * K[1] * K[2]);
  for (int i = 0; i < natom; ++i) {
    double w[3][16];
    int base[3];
    for (int d = 0; d < 3; ++d) {
      double u = K[d] * pos[3 * i + d] / box[d];
      u -= floor(u / K[d]) * K[d];
      base[d] = (int)floor(u);
      orc_bspline_weights(n, u - base[d], w[d], NULL);
    }
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b)
        for (int c = 0; c < n; ++c) {
          int i0 = wrapi(base[0] - a, K[0]), i1 = wrapi(base[1] - b, K[1]), i2 = wrapi(base[2] - c, K[2]);
          Q[i2 + (size_t)K[2] * (i1 + (size_t)K[1] * i0)] += q[i] * w[0][a] * w[1][b] * w[2][c];
        }
  }
}

/* ik or analytic SPME: reciprocal energy and forces (method 0 ik, 1 analytic) */
double orc_spme_rec(int natom, const double* pos, const double* q, const double box[3], const int K[3],
                    int n, double beta, int method, double* force) {
  const size_t size = (size_t)K[0] * K[1] * K[2];
  const double V = box[0] * box[1] * box[2];
  double* Q = (double*)malloc(sizeof(double) * size);
  orc_spme_spread(natom, pos, q, box, K, n, Q);
  double* b[3];
  for (int d = 0; d < 3; ++d) { b[d] = (double*)malloc(sizeof(double) * K[d]); orc_spme_bmod(n, K[d], b[d]); }
  double* QF = (double*)malloc(sizeof(double) * 2 * size);
  for (size_t t = 0; t < size; ++t) { QF[2 * t] = Q[t]; QF[2 * t + 1] = 0; }
  orc_dft3d(K, QF, -1);
  const int nconv = method == 0 ? 4 : 1;
  double* G[4];
  for (int c = 0; c < nconv; ++c) G[c] = (double*)malloc(sizeof(double) * 2 * size);
  const double scale = M_PI * M_PI / beta / beta;
  for (int i = 0; i < K[0]; ++i) {
    int ip = i <= K[0] / 2 ? i : i - K[0];
    for (int j = 0; j < K[1]; ++j) {
      int jp = j <= K[1] / 2 ? j : j - K[1];
      for (int k = 0; k < K[2]; ++k) {
        int kp = k <= K[2] / 2 ? k : k - K[2];
        size_t t = k + (size_t)K[2] * (j + (size_t)K[1] * i);
        double psi = 0, ph[3] = {0, 0, 0};
        if (ip || jp || kp) {
          double m[3] = {ip / box[0], jp / box[1], kp / box[2]};
          double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
          double expm = exp(-scale * mm) / mm * b[0][i] * b[1][j] * b[2][k];
          psi = (method == 0 ? 1. / (M_PI * V) : 1. / (2 * M_PI * V)) * expm * size;
          for (int d = 0; d < 3; ++d) ph[d] = -2. / V * expm * m[d] * size;
        }
        double qr = QF[2 * t], qi = QF[2 * t + 1];
        G[0][2 * t] = qr * psi; G[0][2 * t + 1] = qi * psi;
        if (method == 0)
          for (int d = 0; d < 3; ++d) { G[1 + d][2 * t] = -qi * ph[d]; G[1 + d][2 * t + 1] = qr * ph[d]; }
      }
    }
  }
  /* The reference multiplies on the r2c half spectrum (k2 <= K2/2) and runs a
     c2r transform, which takes the other half as the Hermitian image of the
     stored one: X(a,b,c) = conj X(-a,-b,K2-c) for c > K2/2.  On the x / y
     Nyquist planes the ik kernel is not Hermitian, so re-derive that half. */
  for (int c = 0; c < nconv; ++c)
    for (int i = 0; i < K[0]; ++i)
      for (int j = 0; j < K[1]; ++j)
        for (int k = K[2] / 2 + 1; k < K[2]; ++k) {
          size_t t = k + (size_t)K[2] * (j + (size_t)K[1] * i);
          size_t s = (K[2] - k) + (size_t)K[2] * (((K[1] - j) % K[1]) + (size_t)K[1] * ((K[0] - i) % K[0]));
          G[c][2 * t] = G[c][2 * s];
          G[c][2 * t + 1] = -G[c][2 * s + 1];
        }
  for (int c = 0; c < nconv; ++c) orc_dft3d(K, G[c], +1);
  double E = 0;
  for (size_t t = 0; t < size; ++t) E += Q[t] * G[0][2 * t] / size;
  if (method == 0) E *= 0.5;
  for (int at = 0; at < natom; ++at) {
    double w[3][16], dw[3][16];
    int base[3];
    for (int d = 0; d < 3; ++d) {
      double u = K[d] * pos[3 * at + d] / box[d];
      u -= floor(u / K[d]) * K[d];
      base[d] = (int)floor(u);
      orc_bspline_weights(n, u - base[d], w[d], dw[d]);
    }
    double f[3] = {0, 0, 0};
    for (int a = 0; a < n; ++a)
      for (int bb = 0; bb < n; ++bb)
        for (int c = 0; c < n; ++c) {
          size_t t = wrapi(base[2] - c, K[2]) + (size_t)K[2] * (wrapi(base[1] - bb, K[1]) + (size_t)K[1] * wrapi(base[0] - a, K[0]));
          if (method == 0) {
            double wt = w[0][a] * w[1][bb] * w[2][c];
            for (int d = 0; d < 3; ++d) f[d] += G[1 + d][2 * t] / size * wt;
          } else {
            double cv = G[0][2 * t] / size;
            f[0] += -cv * dw[0][a] * w[1][bb] * w[2][c] * K[0] / box[0];
            f[1] += -cv * w[0][a] * dw[1][bb] * w[2][c] * K[1] / box[1];
            f[2] += -cv * w[0][a] * w[1][bb] * dw[2][c] * K[2] / box[2];
          }
        }
    for (int d = 0; d < 3; ++d) force[3 * at + d] = (method == 0 ? 1.0 : 2.0) * q[at] * f[d];
  }
  for (int c = 0; c < nconv; ++c) free(G[c]);
  for (int d = 0; d < 3; ++d) free(b[d]);
  free(QF); free(Q);
  return E;
}

/* exact reciprocal Ewald sum over |m_d| <= K_d/2 (EleRecES) */
double orc_ewald_rec_exact(int natom, const double* pos, const double* q, const double box[3],
                           const int K[3], double beta, double* force) {
  const double V = box[0] * box[1] * box[2];
  double E = 0;
  memset(force, 0, sizeof(double) * 3 * natom);
  for (int m0 = -K[0] / 2; m0 <= K[0] / 2; ++m0)
    for (int m1 = -K[1] / 2; m1 <= K[1] / 2; ++m1)
      for (int m2 = -K[2] / 2; m2 <= K[2] / 2; ++m2) {
        if (!m0 && !m1 && !m2) continue;
        double m[3] = {m0 / box[0], m1 / box[1], m2 / box[2]};
        double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
        double ex = exp(-M_PI * M_PI * mm / beta / beta) / mm;
        double sr = 0, si = 0;
        for (int i = 0; i < natom; ++i) {
          double t = 2 * M_PI * (m[0] * pos[3 * i] + m[1] * pos[3 * i + 1] + m[2] * pos[3 * i + 2]);
          sr += q[i] * cos(t);
          si += q[i] * sin(t);
        }
        E += ex * (sr * sr + si * si);
        for (int i = 0; i < natom; ++i) {
          double t = 2 * M_PI * (m[0] * pos[3 * i] + m[1] * pos[3 * i + 1] + m[2] * pos[3 * i + 2]);
          double a = q[i] * cos(t), b = q[i] * sin(t);
          /* applyInteraction: sum0,sum1 use exp(-i t); coeff = (sum0 b + sum1 a) 2/V ex */
          double coeff = (sr * b - si * a) * 2. / V * ex;
          for (int d = 0; d < 3; ++d) force[3 * i + d] += coeff * m[d];
        }
      }
  return E / (2 * M_PI * V);
}

/* real-space Ewald with minimum image, all pairs (EleDir), and the self term */
double orc_ewald_dir(int natom, const double* pos, const double* q, const double box[3], double beta,
                     double rcut, double* force) {
  double E = 0;
  const double rc2 = rcut * rcut, spi = 1. / sqrt(M_PI);
  memset(force, 0, sizeof(double) * 3 * natom);
#pragma omp parallel for reduction(+ : E) schedule(dynamic, 16)
  for (int i = 0; i < natom; ++i) {
    double f[3] = {0, 0, 0};
    for (int j = 0; j < natom; ++j) {
      if (j == i) continue;
      double d[3];
      for (int k = 0; k < 3; ++k) {
        d[k] = pos[3 * i + k] - pos[3 * j + k];
        d[k] -= floor(d[k] / box[k] + 0.5) * box[k];
      }
      double rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (rr > rc2) continue;
      double r = sqrt(rr), qq = q[i] * q[j];
      double e = erfc(beta * r);
      double s = (e / r + 2 * beta * spi * exp(-beta * beta * rr)) / rr * qq;
      for (int k = 0; k < 3; ++k) f[k] += s * d[k];
      E += 0.5 * qq * e / r;
    }
    for (int k = 0; k < 3; ++k) force[3 * i + k] = f[k];
  }
  return E;
}

double orc_ewald_self(int natom, const double* q, double beta) {
  double s = 0;
  for (int i = 0; i < natom; ++i) s += q[i] * q[i];
  return -beta / sqrt(M_PI) * s;
}

/* Self-force correction of analytic-differentiation SPME (SelfCorr::calKernel
   and ::correction, RE/src/SelfCorr.cpp:99-220), rectangular box, |k| <= 3:
     c_d(k) = sum_m (e^{-pi^2 m^2/beta^2}/m^2 / (2 pi V)) (-2) g_d(m_d, k) (-4 pi k K_d / L_d)
     g_d(m, k) = (u + 2 pi k)^-n / sum_{l=-3..3} (u + 2 pi l)^-n,  u = 2 pi m / K_d
   (0 at the Nyquist index of an even K_d), then for k = 1..3
     F_id -= c_d(k) q_i^2 sin(2 pi k K_d x_id / L_d). */
static double ipow_d(double x, int n) {
  double r = 1;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

static double alias_sum(double u, int n) {
  double s = 1. / ipow_d(u, n), up = u, un = u;
  for (int l = 0; l < 3; ++l) {
    up += 2. * M_PI;
    un -= 2. * M_PI;
    s += 1. / ipow_d(up, n);
    s += 1. / ipow_d(un, n);
  }
  return s;
}

void orc_spme_selfcorr(int natom, const double* pos, const double* q, const double box[3], const int K[3],
                       int order, double beta, double* force) {
  const double V = box[0] * box[1] * box[2];
  const double scalor = 1. / (2. * M_PI * V);
  double c[3][4] = {{0}};
  for (int kk = 1; kk <= 3; ++kk) {
    for (int i0 = 0; i0 < K[0]; ++i0)
      for (int i1 = 0; i1 < K[1]; ++i1)
        for (int i2 = 0; i2 < K[2]; ++i2) {
          const int idx[3] = {i0, i1, i2};
          int p[3];
          for (int d = 0; d < 3; ++d) p[d] = idx[d] > (K[d] >> 1) ? idx[d] - K[d] : idx[d];
          const double m[3] = {p[0] / box[0], p[1] / box[1], p[2] / box[2]};
          const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
          if (m2 == 0) continue;
          const double t = M_PI / beta;
          const double fm = exp(-t * t * m2) / m2 * scalor;
          for (int d = 0; d < 3; ++d) {
            if (idx[d] == (K[d] >> 1) && (K[d] % 2 == 0)) continue;
            const double u = 2. * M_PI * p[d] / K[d];
            const double g = 1. / ipow_d(u + 2. * M_PI * kk, order) / alias_sum(u, order);
            c[d][kk] += (-2. * fm * g) * (-4.) * M_PI * kk * (double)K[d] / box[d];
          }
        }
  }
  for (int i = 0; i < natom; ++i)
    for (int kk = 1; kk <= 3; ++kk)
      for (int d = 0; d < 3; ++d)
        force[3 * i + d] -= c[d][kk] * q[i] * q[i] * sin(2. * M_PI * kk * K[d] / box[d] * pos[3 * i + d]);
}
