/* ORACLE -- test infrastructure only.  CPU restatement of the inhomogeneous
 * ik-SPME error estimate of ErrorEstimate_SPME_Ik (longRange.hetero/profile.test/
 * template/tools/analyze/src/ErrorEstimate_SPME_Ik.cpp:119-470), rectangular box,
 * on the grid of the density profile (the SPME mesh K):
 *   g(m)   = -4 pi f(m) m*,  f = e^{-pi^2 |m*|^2/beta^2} / |m*|^2 / (2 pi V)
 *   a_d(m, k) = (u_d + 2 pi k)^-n / sum_{l=-3..3} (u_d + 2 pi l)^-n,  u_d = 2 pi m_d / K_d
 *   k2b = sum_{k = +-1..+-4} sum_dir V/N |IFFT(i g a_dir(k))|^2
 *   k1  = i g 2 sum_{k, dir} a_dir(k)  (k-space kernel, times V)
 *   k2a = FFT(V/N |IFFT(k1 / V)|^2) + 2 FFT(k2b)
 *   e1_d = IFFT(k1_d FFT(rho1 V/N)) q/V,  e2 = IFFT(k2a FFT(rho2 V/N)) q^2/V
 *   error1 = sum_d e1_d^2 (real and imaginary parts apart), error2 = e2
 * with each component of g zeroed at the Nyquist index of an even K_d.
 * Transforms are unnormalised, sign -1 forward / +1 backward. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_dft3d(const int n[3], double* data, int sign);

static double ipw(double x, int n) {
  double r = 1;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

static double alias(double u, int n) {
  double s = 1. / ipw(u, n), up = u, un = u;
  for (int l = 0; l < 3; ++l) {
    up += 2. * M_PI;
    un -= 2. * M_PI;
    s += 1. / ipw(up, n);
    s += 1. / ipw(un, n);
  }
  return s;
}

static int cidx(int i, int K) { return i > (K >> 1) ? i - K : i; }

/* calError of both maps: e1_d = IFFT(k1_d FFT(rho1 V/N)) q/V, e2 = IFFT(k2a FFT(rho2 V/N)) q^2/V
 * (real parts scaled), error1 = sum_d e1_d^2 with real and imaginary parts apart; k1 [3][N]
 * and k2a [N] complex, interleaved */
static void errmap_apply(const int K[3], const double box[3], const double* k1, const double* k2a,
                         const double* rho1, const double* rho2, double charge, double* e1, double* e2) {
  const long N = (long)K[0] * K[1] * K[2];
  const double V = box[0] * box[1] * box[2];
  double* r1 = (double*)calloc(2 * N, sizeof(double));
  double* r2 = (double*)calloc(2 * N, sizeof(double));
  for (long i = 0; i < N; ++i) {
    r1[2 * i] = rho1[i] * V / (double)N;
    r2[2 * i] = rho2[i] * V / (double)N;
  }
  orc_dft3d(K, r1, -1);
  orc_dft3d(K, r2, -1);
  double* ex = (double*)calloc(8 * N, sizeof(double)); /* e1x, e1y, e1z, e2 */
  for (long i = 0; i < N; ++i) {
    for (int d = 0; d < 3; ++d) {
      const double ar = k1[2 * (d * N + i)], ai = k1[2 * (d * N + i) + 1];
      ex[2 * (d * N + i)] = r1[2 * i] * ar - r1[2 * i + 1] * ai;
      ex[2 * (d * N + i) + 1] = r1[2 * i] * ai + r1[2 * i + 1] * ar;
    }
    ex[2 * (3 * N + i)] = r2[2 * i] * k2a[2 * i] - r2[2 * i + 1] * k2a[2 * i + 1];
    ex[2 * (3 * N + i) + 1] = r2[2 * i] * k2a[2 * i + 1] + r2[2 * i + 1] * k2a[2 * i];
  }
  for (int d = 0; d < 4; ++d) orc_dft3d(K, ex + 2 * d * N, +1);
  for (long i = 0; i < N; ++i) {
    double s0 = 0, s1 = 0;
    for (int d = 0; d < 3; ++d) {
      const double re = ex[2 * (d * N + i)] * charge / V, im = ex[2 * (d * N + i) + 1];
      s0 += re * re;
      s1 += im * im;
    }
    e1[2 * i] = s0;
    e1[2 * i + 1] = s1;
    e2[2 * i] = ex[2 * (3 * N + i)] * charge * charge / V;
    e2[2 * i + 1] = ex[2 * (3 * N + i) + 1];
  }
  free(r1); free(r2); free(ex);
}

void orc_spme_ik_errmap(const int K[3], const double box[3], double beta, int order, const double* rho1,
                        const double* rho2, double charge, double* e1, double* e2) {
  const long N = (long)K[0] * K[1] * K[2];
  const double V = box[0] * box[1] * box[2];
  const double scal = 1. / (2. * M_PI * V);
  double* g = (double*)calloc(3 * N, sizeof(double));
  double* k1 = (double*)calloc(6 * N, sizeof(double));    /* 3 complex grids, kept k-space kernel */
  double* w = (double*)calloc(6 * N, sizeof(double));     /* 3 complex work grids */
  double* k2a = (double*)calloc(2 * N, sizeof(double));
  double* k2b = (double*)calloc(2 * N, sizeof(double));
  int even[3];
  for (int d = 0; d < 3; ++d) even[d] = (K[d] % 2 == 0);
  for (int i0 = 0; i0 < K[0]; ++i0)
    for (int i1 = 0; i1 < K[1]; ++i1)
      for (int i2 = 0; i2 < K[2]; ++i2) {
        const long idx = i2 + (long)K[2] * (i1 + (long)K[1] * i0);
        const double m[3] = {cidx(i0, K[0]) / box[0], cidx(i1, K[1]) / box[1], cidx(i2, K[2]) / box[2]};
        const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
        if (m2 == 0) continue;
        const double t = M_PI / beta, fm = exp(-t * t * m2) / m2 * scal;
        for (int d = 0; d < 3; ++d) g[d * N + idx] = -4. * M_PI * fm * m[d];
      }
  /* aliasing sums of the six k and three directions */
  for (int k = -4; k <= 4; ++k) {
    if (k == 0) continue;
    for (int dir = 0; dir < 3; ++dir) {
      memset(w, 0, sizeof(double) * 6 * N);
      for (int i0 = 0; i0 < K[0]; ++i0)
        for (int i1 = 0; i1 < K[1]; ++i1)
          for (int i2 = 0; i2 < K[2]; ++i2) {
            const long idx = i2 + (long)K[2] * (i1 + (long)K[1] * i0);
            if (idx == 0) continue;
            const int ii[3] = {i0, i1, i2};
            const double u = 2. * M_PI * cidx(ii[dir], K[dir]) / K[dir];
            const double a = 1. / ipw(u + 2. * M_PI * k, order) * (1. / alias(u, order));
            for (int d = 0; d < 3; ++d) {
              double v = g[d * N + idx] * a;
              if (even[d] && ii[d] == (K[d] >> 1)) v = 0.;
              w[2 * (d * N + idx) + 1] = v;
            }
          }
      for (int d = 0; d < 3; ++d) orc_dft3d(K, w + 2 * d * N, +1);
      for (long i = 0; i < N; ++i) {
        double s = 0;
        for (int d = 0; d < 3; ++d) {
          const double re = w[2 * (d * N + i)], im = w[2 * (d * N + i) + 1];
          s += re * re + im * im;
        }
        k2b[2 * i] += s * V / (double)N;
      }
    }
  }
  /* the summed kernel */
  memset(w, 0, sizeof(double) * 6 * N);
  for (int i0 = 0; i0 < K[0]; ++i0)
    for (int i1 = 0; i1 < K[1]; ++i1)
      for (int i2 = 0; i2 < K[2]; ++i2) {
        const long idx = i2 + (long)K[2] * (i1 + (long)K[1] * i0);
        if (idx == 0) continue;
        const int ii[3] = {i0, i1, i2};
        double u[3], fen[3];
        for (int d = 0; d < 3; ++d) {
          u[d] = 2. * M_PI * cidx(ii[d], K[d]) / K[d];
          fen[d] = 1. / alias(u[d], order);
        }
        double sum = 0.;
        for (int k = -4; k <= 4; ++k) {
          if (k == 0) continue;
          for (int d = 0; d < 3; ++d) sum += 1. / ipw(u[d] + 2. * M_PI * k, order) * fen[d];
        }
        for (int d = 0; d < 3; ++d) {
          double v = g[d * N + idx] * sum * 2.;
          if (even[d] && ii[d] == (K[d] >> 1)) v = 0.;
          w[2 * (d * N + idx) + 1] = v;
          k1[2 * (d * N + idx) + 1] = v * V;
        }
      }
  for (int d = 0; d < 3; ++d) orc_dft3d(K, w + 2 * d * N, +1);
  for (long i = 0; i < N; ++i) {
    double s = 0;
    for (int d = 0; d < 3; ++d) {
      const double re = w[2 * (d * N + i)], im = w[2 * (d * N + i) + 1];
      s += re * re + im * im;
    }
    k2a[2 * i] = s * V / (double)N;
  }
  orc_dft3d(K, k2a, -1);
  orc_dft3d(K, k2b, -1);
  for (long i = 0; i < 2 * N; ++i) k2a[i] += 2. * k2b[i];
  errmap_apply(K, box, k1, k2a, rho1, rho2, charge, e1, e2);
  free(g); free(k1); free(w); free(k2a); free(k2b);
}


/* ------------------------------------------------------------ real space
 * ErrorEstimate_dir::makeS1k / makeS2k / calError (analyze/src/ErrorEstimate_dir.cpp:
 * 124-331), rectangular box:
 *   s1k(k) = 2/k int_rc^30 r f(r)^2 sin(2 pi k r) dr  (k != 0),  4 pi int_rc^30 r^2 f^2 dr (k = 0),
 *     f(r) = (2 beta/sqrt(pi) e^{-beta^2 r^2} + erfc(beta r)/r) / r
 *   s2k_d(k) = i k_d [2 pi / k int_rc^30 -2 erfc(beta r) sin(2 pi k r) dr
 *              + 2 pi rc erfc(beta rc) (2 cos(e)/e - 2 sin(e)/e^2) / k],  e = 2 pi k rc
 * with the integrals of the analyze tools' Integral1D (src/Integral1D.cpp:60-232):
 * Gauss-4 boxes (nodes sqrt((3 -+ 2 sqrt(1.2))/7), weights (18 +- sqrt 30)/36),
 * the range split into 10 boxes of tol/10, a box bisected while
 * |coarse - (left + right)| >= 255 tol (children tol/2) and while its width is at
 * least 1e-13 of the initial box; tol = 1e-20.  Then the calError above with
 * k1 = s2k, k2a = s1k. */
typedef struct { int kind; double k, beta; } DirFn;

static double dir_f(const DirFn* f, double r) {
  if (f->kind == 2) return -2. * erfc(f->beta * r) * sin(2. * M_PI * f->k * r);
  const double betar = f->beta * r, ri = 1. / r;
  const double fr = (2. * f->beta / sqrt(M_PI) * exp(-betar * betar) + erfc(betar) * ri) * ri;
  if (f->kind == 0) return r * fr * fr * sin(2. * M_PI * f->k * r);
  return r * r * fr * fr;
}

static double dir_coarse(const DirFn* f, double xlo, double xup) {
  const double hx = xup - xlo;
  const double v0 = sqrt((3 - 2 * sqrt(1.2)) / 7.), v1 = sqrt((3 + 2 * sqrt(1.2)) / 7.);
  const double x0 = 0.5 * (xup - xlo) * (-v1) + 0.5 * (xup + xlo);
  const double x1 = 0.5 * (xup - xlo) * (-v0) + 0.5 * (xup + xlo);
  const double x2 = 0.5 * (xup - xlo) * (+v0) + 0.5 * (xup + xlo);
  const double x3 = 0.5 * (xup - xlo) * (+v1) + 0.5 * (xup + xlo);
  const double w0 = (18 + sqrt(30.)) / 36., w1 = (18 - sqrt(30.)) / 36.;
  return 0.5 * hx * (w1 * (dir_f(f, x0) + dir_f(f, x3)) + w0 * (dir_f(f, x1) + dir_f(f, x2)));
}

static double dir_box(const DirFn* f, double xlo, double xup, double tol, double coarse, double ghx) {
  const double hhx = 0.5 * (xup - xlo);
  const double c0 = dir_coarse(f, xlo, xlo + hhx), c1 = dir_coarse(f, xlo + hhx, xup);
  double value = c0 + c1;
  if (fabs(coarse - value) < tol * 255) return value;
  if (hhx * 2 < 1e-13 * ghx) return value;
  value = 0;
  value += dir_box(f, xlo, xlo + hhx, tol * 0.5, c0, ghx);
  value += dir_box(f, xlo + hhx, xup, tol * 0.5, c1, ghx);
  return value;
}

static double dir_int(int kind, double k, double beta, double xlo, double xup, double tol, int init_nx) {
  DirFn f = {kind, k, beta};
  const double hx = (xup - xlo) / (double)init_nx, nxi = 1. / (double)init_nx;
  double value = 0;
  for (int i = 0; i < init_nx; i++) {
    const double x = xlo + i * hx;
    value += dir_box(&f, x, x + hx, tol * nxi, dir_coarse(&f, x, x + hx), hx);
  }
  return value;
}

void orc_dir_errmap(const int K[3], const double box[3], double beta, double rcut, const double* rho1,
                    const double* rho2, double charge, double* e1, double* e2) {
  const long N = (long)K[0] * K[1] * K[2];
  double* k1 = (double*)calloc(6 * N, sizeof(double));
  double* k2a = (double*)calloc(2 * N, sizeof(double));
#pragma omp parallel for schedule(dynamic, 4)
  for (int ix = -K[0] / 2; ix < K[0] - K[0] / 2; ++ix) {
    const int lx = ix < 0 ? ix + K[0] : ix;
    for (int iy = -K[1] / 2; iy < K[1] - K[1] / 2; ++iy) {
      const int ly = iy < 0 ? iy + K[1] : iy;
      for (int iz = -K[2] / 2; iz < K[2] - K[2] / 2; ++iz) {
        const int lz = iz < 0 ? iz + K[2] : iz;
        const long p = lz + (long)K[2] * (ly + (long)K[1] * lx);
        /* makeS1k */
        const double k1m = sqrt(ix * ix / (box[0] * box[0]) + iy * iy / (box[1] * box[1]) + iz * iz / (box[2] * box[2]));
        if (k1m != 0) k2a[2 * p] = 2. / k1m * dir_int(0, k1m, beta, rcut, 30, 1e-20, 10);
        else k2a[2 * p] = 4. * M_PI * dir_int(1, k1m, beta, rcut, 30, 1e-20, 10);
        /* makeS2k */
        const double kx = ix / box[0], ky = iy / box[1], kz = iz / box[2];
        const double k = sqrt(kx * kx + ky * ky + kz * kz);
        if (k != 0) {
          const double an = dir_int(2, k, beta, rcut, 30, 1e-20, 10) / k;
          const double e = 2. * M_PI * k * rcut;
          double size = 2. * M_PI * rcut * erfc(beta * rcut) * (2. * cos(e) / e - 2. * sin(e) / (e * e));
          size /= k;
          const double kk[3] = {kx, ky, kz};
          for (int d = 0; d < 3; ++d) {
            double v = 2 * M_PI * kk[d] * an;
            v += size * kk[d];
            k1[2 * (d * N + p) + 1] = v;
          }
        }
      }
    }
  }
  errmap_apply(K, box, k1, k2a, rho1, rho2, charge, e1, e2);
  free(k1); free(k2a);
}


/* ------------------------------------------------- analytic differentiation
 * ErrorEstimate_SPME_Ana::reinit / calKernel / calError (analyze/src/
 * ErrorEstimate_SPME_Ana.cpp:140-745), rectangular box, alias images
 * 0 < |k| <= 2 (global_half_N_k_sum = 2):
 *   F_d(m, k) = -2 f(m) a_d(m, k)   (0 at the Nyquist index of an even K_d)
 *   A*_dd     = L_e L_f / V,  c_d(k) = 2 pi k K_d A*_dd
 *   self      = sum_{k, d} c_d(k)^2 (sum_m F_d(m, k))^2
 *   k2b       = sum_{k, dir} V/N (|IFFT(w)|^2 + |IFFT(w + i c_dir(k) F_dir(k) e_dir)|^2),
 *               w = i g a_dir(k)
 *   k1        = V i g 2 sum_{k, dir} a_dir(k),  k2a = FFT(V/N |IFFT(k1 / V)|^2) + FFT(k2b)
 * then calError as for the ik map.  fconv (nullable) receives
 * FConvRho1_d(k) = IFFT(FFT(rho1 V/N) V F_d(k)) / V as [4 (k = -2,-1,1,2)][3][N][2]. */
static double ana_astar(const double box[3], int d) {
  const double V = box[0] * (box[1] * box[2]);
  if (d == 0) return (box[1] * box[2]) * (1. / V);
  if (d == 1) return (box[0] * box[2]) * (1. / V);
  return (box[0] * box[1]) * (1. / V);
}

static double ana_F(const int K[3], int order, double fm, const int ii[3], int d, int k) {
  if (K[d] % 2 == 0 && ii[d] == (K[d] >> 1)) return 0.;
  const double u = 2. * M_PI * cidx(ii[d], K[d]) / K[d];
  double fen = 1. / ipw(u + 2. * M_PI * k, order);
  fen /= alias(u, order);
  return -2. * fm * fen;
}

void orc_spme_ana_errmap(const int K[3], const double box[3], double beta, int order, const double* rho1,
                         const double* rho2, double charge, double* e1, double* e2, double* self_out,
                         double* fconv) {
  const int KC = 2;
  const long N = (long)K[0] * K[1] * K[2];
  const double V = box[0] * box[1] * box[2];
  const double scal = 1. / (2. * M_PI * V);
  double* g = (double*)calloc(3 * N, sizeof(double));
  double* f = (double*)calloc(N, sizeof(double));
  double* k1 = (double*)calloc(6 * N, sizeof(double));
  double* w = (double*)calloc(6 * N, sizeof(double));
  double* k2a = (double*)calloc(2 * N, sizeof(double));
  double* k2b = (double*)calloc(2 * N, sizeof(double));
  int even[3];
  for (int d = 0; d < 3; ++d) even[d] = (K[d] % 2 == 0);
  for (long idx = 0; idx < N; ++idx) {
    const int ii[3] = {(int)(idx / ((long)K[1] * K[2])), (int)((idx / K[2]) % K[1]), (int)(idx % K[2])};
    const double m[3] = {cidx(ii[0], K[0]) / box[0], cidx(ii[1], K[1]) / box[1], cidx(ii[2], K[2]) / box[2]};
    const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
    if (m2 == 0) continue;
    const double t = M_PI / beta;
    f[idx] = exp(-t * t * m2) / m2 * scal;
    for (int d = 0; d < 3; ++d) g[d * N + idx] = -4. * M_PI * f[idx] * m[d];
  }
  /* self-force error: sequential sums over the grid, as calKernel takes them */
  double self = 0.;
  for (int k = -KC; k <= KC; ++k) {
    if (k == 0) continue;
    for (int d = 0; d < 3; ++d) {
      double s = 0.;
      for (long idx = 0; idx < N; ++idx) {
        const int ii[3] = {(int)(idx / ((long)K[1] * K[2])), (int)((idx / K[2]) % K[1]), (int)(idx % K[2])};
        s += ana_F(K, order, f[idx], ii, d, k);
      }
      const double a = ana_astar(box, d);
      self += 4. * M_PI * M_PI * k * k * K[d] * K[d] * a * a * s * s;
    }
  }
  *self_out = self;
  /* second moment of the aliased force kernels */
  for (int k = -KC; k <= KC; ++k) {
    if (k == 0) continue;
    for (int dir = 0; dir < 3; ++dir) {
      memset(w, 0, sizeof(double) * 6 * N);
      double* wd = (double*)calloc(2 * N, sizeof(double)); /* component dir with the derivative term */
      for (long idx = 1; idx < N; ++idx) {
        const int ii[3] = {(int)(idx / ((long)K[1] * K[2])), (int)((idx / K[2]) % K[1]), (int)(idx % K[2])};
        const double u = 2. * M_PI * cidx(ii[dir], K[dir]) / K[dir];
        const double a = 1. / ipw(u + 2. * M_PI * k, order) * (1. / alias(u, order));
        for (int d = 0; d < 3; ++d) {
          double v = g[d * N + idx] * a;
          if (even[d] && ii[d] == (K[d] >> 1)) v = 0.;
          w[2 * (d * N + idx) + 1] = v;
        }
      }
      for (long idx = 0; idx < N; ++idx) {
        const int ii[3] = {(int)(idx / ((long)K[1] * K[2])), (int)((idx / K[2]) % K[1]), (int)(idx % K[2])};
        wd[2 * idx + 1] = w[2 * (dir * N + idx) + 1] +
                          2. * M_PI * (double)k * K[dir] * ana_astar(box, dir) * ana_F(K, order, f[idx], ii, dir, k);
      }
      for (int d = 0; d < 3; ++d) orc_dft3d(K, w + 2 * d * N, +1);
      orc_dft3d(K, wd, +1);
      for (int pass = 0; pass < 2; ++pass)
        for (long i = 0; i < N; ++i) {
          double s = 0;
          for (int d = 0; d < 3; ++d) {
            const double* src = (pass == 1 && d == dir) ? wd + 2 * i : w + 2 * (d * N + i);
            s += src[0] * src[0] + src[1] * src[1];
          }
          k2b[2 * i] += s * V / (double)N;
        }
      free(wd);
    }
  }
  /* the summed kernel */
  memset(w, 0, sizeof(double) * 6 * N);
  for (long idx = 1; idx < N; ++idx) {
    const int ii[3] = {(int)(idx / ((long)K[1] * K[2])), (int)((idx / K[2]) % K[1]), (int)(idx % K[2])};
    double u[3], fen[3];
    for (int d = 0; d < 3; ++d) {
      u[d] = 2. * M_PI * cidx(ii[d], K[d]) / K[d];
      fen[d] = 1. / alias(u[d], order);
    }
    double sum = 0.;
    for (int k = -KC; k <= KC; ++k) {
      if (k == 0) continue;
      for (int d = 0; d < 3; ++d) sum += 1. / ipw(u[d] + 2. * M_PI * k, order) * fen[d];
    }
    for (int d = 0; d < 3; ++d) {
      double v = g[d * N + idx] * sum * 2.;
      if (even[d] && ii[d] == (K[d] >> 1)) v = 0.;
      w[2 * (d * N + idx) + 1] = v;
      k1[2 * (d * N + idx) + 1] = v * V;
    }
  }
  for (int d = 0; d < 3; ++d) orc_dft3d(K, w + 2 * d * N, +1);
  for (long i = 0; i < N; ++i) {
    double s = 0;
    for (int d = 0; d < 3; ++d) {
      const double re = w[2 * (d * N + i)], im = w[2 * (d * N + i) + 1];
      s += re * re + im * im;
    }
    k2a[2 * i] = s * V / (double)N;
  }
  orc_dft3d(K, k2a, -1);
  orc_dft3d(K, k2b, -1);
  for (long i = 0; i < 2 * N; ++i) k2a[i] += k2b[i];
  errmap_apply(K, box, k1, k2a, rho1, rho2, charge, e1, e2);
  if (fconv) {
    double* r1 = (double*)calloc(2 * N, sizeof(double));
    for (long i = 0; i < N; ++i) r1[2 * i] = rho1[i] * V / (double)N;
    orc_dft3d(K, r1, -1);
    int slot = 0;
    for (int k = -KC; k <= KC; ++k) {
      if (k == 0) continue;
      for (int d = 0; d < 3; ++d) {
        double* o = fconv + 2 * N * (3 * slot + d);
        for (long idx = 0; idx < N; ++idx) {
          const int ii[3] = {(int)(idx / ((long)K[1] * K[2])), (int)((idx / K[2]) % K[1]), (int)(idx % K[2])};
          const double b = ana_F(K, order, f[idx], ii, d, k) * V;
          o[2 * idx] = r1[2 * idx] * b;
          o[2 * idx + 1] = r1[2 * idx + 1] * b;
        }
        orc_dft3d(K, o, +1);
        for (long i = 0; i < 2 * N; ++i) o[i] /= V;
      }
      ++slot;
    }
    free(r1);
  }
  free(g); free(f); free(k1); free(w); free(k2a); free(k2b);
}
