/*
 * ORACLE -- test infrastructure only.  CPU FP64 restatement of the adaptive
 * cutoff estimate (AdaptRCut), the density profile it consumes and the tail
 * pressure correction it feeds, used as the checker of the GPU versions.
 *
 * Follows (ENG = shortRange.inhomo/template/tools/simulation.hetero.cutoff):
 *  - DensityProfile_PiecewiseConst::reinit/deposite/calculate  ENG/src/DensityProfile.cu:27-99
 *  - Integral1D Gauss4 adaptive quadrature                     ENG/src/Integral1D.cu:164-232
 *  - AdaptRCut::makeS1k / makeS2k                              ENG/src/AdaptRCut.cu:265-416
 *  - AdaptRCut::calError / calRCutOnePoint / refineRCut         ENG/src/AdaptRCut.cu:182-508
 *  - PressureCorrection::makeKernel / correction                ENG/src/PressureCorrection.cu:175-340
 * FFTs: our own unnormalised complex DFT (sign -1 forward, +1 backward), the
 * FFTW convention the reference relies on.  The pressure-correction Bessel
 * functions J_{1/2}, J_{5/2} are evaluated in closed form instead of the
 * reference's interpolated GSL tables (that part is parity-unpinned).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ density profile */
/* bin counts: unsigned(L/refh), made odd (DensityProfile.cu:37-42) */
void orc_dp_bins(const double box[3], double refh, int n[3]) {
  for (int d = 0; d < 3; ++d) {
    unsigned v = (unsigned)(box[d] / refh);
    if ((v - (v / 2) * 2) == 0) v++;
    n[d] = (int)v;
  }
}

/* deposite: coord is binary32 (CoordType), the wrap and bin index in FP64 */
void orc_dp_deposit(int natom, const float* coord, const double box[3], const int n[3],
                    double* profile) {
  const double h[3] = {box[0] / n[0], box[1] / n[1], box[2] / n[2]};
  for (int i = 0; i < natom; ++i) {
    unsigned b[3];
    for (int d = 0; d < 3; ++d) {
      double tmp = coord[3 * i + d];
      if (coord[3 * i + d] >= box[d]) tmp -= box[d];
      else if (coord[3 * i + d] < 0) tmp += box[d];
      b[d] = (unsigned)(tmp / h[d]);
      if (b[d] >= (unsigned)n[d]) b[d] = n[d] - 1;
    }
    profile[b[2] + n[2] * (b[1] + n[1] * b[0])] += 1.;
  }
}

void orc_dp_calculate(const double box[3], const int n[3], int ndata, double* profile) {
  double dv = (box[0] / n[0]) * (box[1] / n[1]) * (box[2] / n[2]);
  long nele = (long)n[0] * n[1] * n[2];
  for (long i = 0; i < nele; ++i) profile[i] /= dv * ndata;
}

/* ------------------------------------------------------------ DFT */
static void dft_line(double* re, double* im, int n, int stride, int sign, double* wr, double* wi,
                     double* tr, double* ti) {
  for (int k = 0; k < n; ++k) {
    double sr = 0, si = 0;
    for (int j = 0; j < n; ++j) {
      int m = (int)(((long)j * k) % n);
      double c = wr[m], s = sign * wi[m];
      double xr = re[(long)j * stride], xi = im[(long)j * stride];
      sr += xr * c - xi * s;
      si += xr * s + xi * c;
    }
    tr[k] = sr;
    ti[k] = si;
  }
  for (int k = 0; k < n; ++k) {
    re[(long)k * stride] = tr[k];
    im[(long)k * stride] = ti[k];
  }
}

/* in-place 3D DFT of interleaved complex data[n0][n1][n2][2] */
void orc_dft3d(const int n[3], double* data, int sign) {
  long nele = (long)n[0] * n[1] * n[2];
  double* re = (double*)malloc(sizeof(double) * nele);
  double* im = (double*)malloc(sizeof(double) * nele);
  for (long i = 0; i < nele; ++i) { re[i] = data[2 * i]; im[i] = data[2 * i + 1]; }
  int nmax = n[0] > n[1] ? n[0] : n[1];
  nmax = nmax > n[2] ? nmax : n[2];
  double* wr = (double*)malloc(sizeof(double) * nmax);
  double* wi = (double*)malloc(sizeof(double) * nmax);
  double* tr = (double*)malloc(sizeof(double) * nmax);
  double* ti = (double*)malloc(sizeof(double) * nmax);
  for (int ax = 0; ax < 3; ++ax) {
    int len = n[ax];
    for (int m = 0; m < len; ++m) {
      wr[m] = cos(2.0 * M_PI * m / len);
      wi[m] = -sin(2.0 * M_PI * m / len);  /* sign applied per call */
    }
    long stride = ax == 2 ? 1 : (ax == 1 ? n[2] : (long)n[1] * n[2]);
    long o1 = ax == 0 ? n[1] : n[0], o2 = ax == 2 ? n[1] : n[2];
    for (long a = 0; a < o1; ++a)
      for (long b = 0; b < o2; ++b) {
        long base;
        if (ax == 0) base = b + n[2] * a;            /* a = iy, b = iz */
        else if (ax == 1) base = b + (long)n[1] * n[2] * a; /* a = ix, b = iz */
        else base = n[2] * (b + n[1] * a);          /* a = ix, b = iy */
        dft_line(re + base, im + base, len, (int)stride, -sign, wr, wi, tr, ti);
      }
  }
  for (long i = 0; i < nele; ++i) { data[2 * i] = re[i]; data[2 * i + 1] = im[i]; }
  free(re); free(im); free(wr); free(wi); free(tr); free(ti);
}

/* ------------------------------------------------------------ quadrature */
static double pow_int(double x, int nn) {
  /* x^n by binary exponentiation, negative n through 1/x */
  unsigned n;
  if (nn < 0) { x = 1.0 / x; n = (unsigned)(-nn); } else n = (unsigned)nn;
  double v = 1.0;
  do {
    if (n & 1) v *= x;
    n >>= 1;
    x *= x;
  } while (n);
  return v;
}

typedef struct { int kind; double k; } Fn;  /* kind 13: x^-13 sin(2 pi k x); 5: x^-5 ...; 1/25: bessel */

static double jhalf(double x) { return x == 0 ? 0 : sqrt(2.0 / (M_PI * x)) * sin(x); }
static double j5half(double x) {
  if (x == 0) return 0;
  return sqrt(2.0 / (M_PI * x)) * ((3.0 / (x * x) - 1.0) * sin(x) - 3.0 * cos(x) / x);
}

static double fn_eval(const Fn* f, double x) {
  switch (f->kind) {
    case 13: return pow_int(x, -13) * sin(2. * M_PI * f->k * x);
    case 5: return pow_int(x, -5) * sin(2. * M_PI * f->k * x);
    case 1: return (-24.) / (pow_int(x, 4) * sqrt(x)) * jhalf(2 * M_PI * f->k * x);
    default: return (-24.) / (pow_int(x, 4) * sqrt(x)) * j5half(2 * M_PI * f->k * x);
  }
}

static double g4_coarse(const Fn* f, double xlo, double xup) {
  const double v0 = sqrt((3 - 2 * sqrt(1.2)) / 7.), v1 = sqrt((3 + 2 * sqrt(1.2)) / 7.);
  const double w0 = (18 + sqrt(30.)) / 36., w1 = (18 - sqrt(30.)) / 36.;
  double x0 = 0.5 * (xup - xlo) * (-v1) + 0.5 * (xup + xlo);
  double x1 = 0.5 * (xup - xlo) * (-v0) + 0.5 * (xup + xlo);
  double x2 = 0.5 * (xup - xlo) * (+v0) + 0.5 * (xup + xlo);
  double x3 = 0.5 * (xup - xlo) * (+v1) + 0.5 * (xup + xlo);
  return 0.5 * (xup - xlo) * (w1 * (fn_eval(f, x0) + fn_eval(f, x3)) + w0 * (fn_eval(f, x1) + fn_eval(f, x2)));
}

static double g4_adapt(const Fn* f, double xlo, double xup, double tol, double coarse, double ghx) {
  double hhx = 0.5 * (xup - xlo);
  double c0 = g4_coarse(f, xlo, xlo + hhx), c1 = g4_coarse(f, xlo + hhx, xup);
  double value = c0 + c1;
  if (fabs(coarse - value) < tol * 255) return value;
  if (hhx * 2 < 1e-13 * ghx) return value;
  return g4_adapt(f, xlo, xlo + hhx, tol * 0.5, c0, ghx) + g4_adapt(f, xlo + hhx, xup, tol * 0.5, c1, ghx);
}

/* Integral1D::cal_int(Gauss4, f, xlo, xup, tol, init_nx = 1) */
double orc_gauss4(int kind, double k, double xlo, double xup, double tol) {
  Fn f = {kind, k};
  double c = g4_coarse(&f, xlo, xup);
  return g4_adapt(&f, xlo, xup, tol, c, xup - xlo);
}

/* ------------------------------------------------------------ AdaptRCut */
static int idx3(const int n[3], int x, int y, int z) { return z + n[2] * (y + n[1] * x); }

/* s1k: real parts [nrc][nele]; s2k{x,y,z}: imaginary parts [nrc][nele] */
void orc_arc_kernels(const double box[3], const int n[3], const double* rc, int nrc, double eps,
                     double sigma, double* s1k, double* s2kx, double* s2ky, double* s2kz) {
  long nele = (long)n[0] * n[1] * n[2];
  double pref = 16. * 36. * pow_int(sigma, 12) * eps;
  double pre = 8. * eps * pow_int(sigma, 6);
#pragma omp parallel for schedule(dynamic, 8)
  for (int ix = -n[0] / 2; ix < n[0] - n[0] / 2; ++ix) {
    int lx = ix < 0 ? ix + n[0] : ix;
    for (int iy = -n[1] / 2; iy < n[1] - n[1] / 2; ++iy) {
      int ly = iy < 0 ? iy + n[1] : iy;
      for (int iz = -n[2] / 2; iz < n[2] - n[2] / 2; ++iz) {
        int lz = iz < 0 ? iz + n[2] : iz;
        long p = idx3(n, lx, ly, lz);
        double kx = ix / box[0], ky = iy / box[1], kz = iz / box[2];
        double k1 = sqrt(ix * ix / (box[0] * box[0]) + iy * iy / (box[1] * box[1]) + iz * iz / (box[2] * box[2]));
        double k2 = sqrt(kx * kx + ky * ky + kz * kz);
        for (int c = nrc - 1; c >= 0; --c) {
          /* makeS1k */
          if (k1 != 0) {
            double an = (c == nrc - 1) ? orc_gauss4(13, k1, rc[nrc - 1], 30, 1e-12)
                                       : orc_gauss4(13, k1, rc[c], rc[c + 1], 1e-12);
            double v = 2. / k1 * pref * an;
            s1k[c * nele + p] = (c == nrc - 1) ? v : s1k[(c + 1) * nele + p] + v;
          } else {
            s1k[c * nele + p] = 4. * M_PI * pref / 11. * pow_int(rc[c], -11);
          }
          /* makeS2k, first loop */
          if (k2 != 0) {
            double an = ((c == nrc - 1) ? orc_gauss4(5, k2, rc[c], 30, 1e-16)
                                        : orc_gauss4(5, k2, rc[c], rc[c + 1], 1e-16)) * pre / k2;
            double bx = 2 * M_PI * kx * an, by = 2 * M_PI * ky * an, bz = 2 * M_PI * kz * an;
            if (c == nrc - 1) {
              s2kx[c * nele + p] = bx; s2ky[c * nele + p] = by; s2kz[c * nele + p] = bz;
            } else {
              s2kx[c * nele + p] = s2kx[(c + 1) * nele + p] + bx;
              s2ky[c * nele + p] = s2ky[(c + 1) * nele + p] + by;
              s2kz[c * nele + p] = s2kz[(c + 1) * nele + p] + bz;
            }
          }
        }
        /* makeS2k, second loop: boundary term at each rc */
        for (int c = nrc - 1; c >= 0; --c) {
          double r = rc[c];
          double rc6 = pow_int(r, 6);
          if (k2 != 0) {
            double e = 2. * M_PI * k2 * r;
            double size = -2. * M_PI * r * r * (4. * eps * pow_int(sigma, 6) / rc6) *
                          (2. * cos(e) / e - 2. * sin(e) / (e * e));
            size /= k2;
            s2kx[c * nele + p] += size * kx;
            s2ky[c * nele + p] += size * ky;
            s2kz[c * nele + p] += size * kz;
          } else {
            s2kx[c * nele + p] = s2ky[c * nele + p] = s2kz[c * nele + p] = 0.;
          }
        }
      }
    }
  }
}

/* calError: error[c][i] = sqrt(e1 + e2x^2 + e2y^2 + e2z^2) (real parts);
   also returns the transformed density rhok (scaled by V/nele) */
void orc_arc_error(const double box[3], const int n[3], int nrc, const double* s1k,
                   const double* s2kx, const double* s2ky, const double* s2kz, const double* rho,
                   double* error) {
  long nele = (long)n[0] * n[1] * n[2];
  double V = box[0] * box[1] * box[2];
  double* rk = (double*)malloc(sizeof(double) * 2 * nele);
  for (long i = 0; i < nele; ++i) { rk[2 * i] = rho[i]; rk[2 * i + 1] = 0; }
  orc_dft3d(n, rk, -1);
  for (long i = 0; i < 2 * nele; ++i) rk[i] *= V / nele;
  double* w[4];
  for (int t = 0; t < 4; ++t) w[t] = (double*)malloc(sizeof(double) * 2 * nele);
  for (int c = 0; c < nrc; ++c) {
    for (long i = 0; i < nele; ++i) {
      double ar = rk[2 * i], ai = rk[2 * i + 1];
      /* (a)(s1 + 0i) and (a)(0 + s2 i) */
      double s1 = s1k[c * nele + i];
      w[0][2 * i] = ar * s1; w[0][2 * i + 1] = ai * s1;
      const double* s2[3] = {s2kx, s2ky, s2kz};
      for (int d = 0; d < 3; ++d) {
        double b = s2[d][c * nele + i];
        w[1 + d][2 * i] = -ai * b;
        w[1 + d][2 * i + 1] = ar * b;
      }
    }
    for (int t = 0; t < 4; ++t) orc_dft3d(n, w[t], +1);
    for (long i = 0; i < nele; ++i) {
      double e1 = w[0][2 * i] / V, ex = w[1][2 * i] / V, ey = w[2][2 * i] / V, ez = w[3][2 * i] / V;
      error[c * nele + i] = sqrt(e1 + ex * ex + ey * ey + ez * ez);
    }
  }
  for (int t = 0; t < 4; ++t) free(w[t]);
  free(rk);
}

/* calRCut: bisection per bin; returns rcut, index, result_error */
void orc_arc_calrcut(int nrc, const double* rc, long nele, const double* error, double prec,
                     double* rcut, int* rcidx, double* rerr) {
  for (long i = 0; i < nele; ++i) {
    unsigned a = 0, b = nrc - 1;
    double ea = error[(long)a * nele + i], eb = error[(long)b * nele + i];
    if (ea - prec <= 0) { rcut[i] = rc[a]; rcidx[i] = a; rerr[i] = ea; }
    else if (eb - prec >= 0) { rcut[i] = rc[b]; rcidx[i] = b; rerr[i] = eb; }
    else {
      while (b - a > 1) {
        unsigned c = (a + b) / 2;
        double ec = error[(long)c * nele + i];
        if (ec > prec) { a = c; } else { b = c; eb = ec; }
      }
      rcut[i] = rc[b]; rcidx[i] = b; rerr[i] = eb;
    }
  }
}

/* refineRCut: max rc index over the periodic 27-bin neighbourhood */
void orc_arc_refine(const int n[3], const double* rc, long nele, const double* error, int* rcidx,
                    double* rcut, double* rerr) {
  int* bk = (int*)calloc(nele, sizeof(int));
  for (int x = 0; x < n[0]; ++x)
    for (int y = 0; y < n[1]; ++y)
      for (int z = 0; z < n[2]; ++z) {
        int i = idx3(n, x, y, z);
        for (int dx = -1; dx <= 1; ++dx)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
              int jx = (x + dx + n[0]) % n[0], jy = (y + dy + n[1]) % n[1], jz = (z + dz + n[2]) % n[2];
              int v = rcidx[idx3(n, jx, jy, jz)];
              if (v > bk[i]) bk[i] = v;
            }
      }
  for (long i = 0; i < nele; ++i) {
    rcidx[i] = bk[i];
    rcut[i] = rc[bk[i]];
    rerr[i] = error[(long)bk[i] * nele + i];
  }
  free(bk);
}

/* ------------------------------------------------------------ pressure correction */
void orc_pc_kernels(const double box[3], const int n[3], const double* rc, int nrc, double* kxx,
                    double* kyy, double* kzz) {
  long nele = (long)n[0] * n[1] * n[2];
  const double upper = 30.;
#pragma omp parallel for schedule(dynamic, 4)
  for (int ix = -n[0] / 2; ix < n[0] - n[0] / 2; ++ix) {
    int lx = ix < 0 ? ix + n[0] : ix;
    double kx = ix / box[0];
    for (int iy = -n[1] / 2; iy < n[1] - n[1] / 2; ++iy) {
      int ly = iy < 0 ? iy + n[1] : iy;
      double ky = iy / box[1];
      for (int iz = -n[2] / 2; iz < n[2] - n[2] / 2; ++iz) {
        int lz = iz < 0 ? iz + n[2] : iz;
        double kz = iz / box[2];
        long p = idx3(n, lx, ly, lz);
        double k = sqrt(kx * kx + ky * ky + kz * kz);
        for (int c = nrc - 1; c >= 0; --c) {
          if (k == 0) { kxx[c * nele + p] = kyy[c * nele + p] = kzz[c * nele + p] = 0; continue; }
          double phi = acos(kz / k), theta;
          if (phi == 0.) theta = 0.;
          else {
            double t = kx / (k * sin(phi));
            if (t > 1.) t = 1.;
            if (t < -1.) t = -1.;
            theta = acos(t);
            if (ky < 0) theta = 2. * M_PI - theta;
          }
          double sc = M_PI / sqrt(k), cp = cos(phi), sp = sin(phi);
          double hi = (c == nrc - 1) ? upper : rc[c + 1];
          double i1 = orc_gauss4(1, k, rc[c], hi, 1e-7);
          double i5 = orc_gauss4(25, k, rc[c], hi, 1e-7);
          double vx = sc * (2. / 3. * i1 + (-1. / 3. + cp * cp - sp * sp * cos(theta * 2)) * i5);
          double vy = sc * (2. / 3. * i1 + (-1. / 3. + cp * cp + sp * sp * cos(theta * 2)) * i5);
          double vz = sc * 4. / 3. * (0.5 * i1 + (0.5 - 1.5 * cp * cp) * i5);
          if (c == nrc - 1) { kxx[c * nele + p] = vx; kyy[c * nele + p] = vy; kzz[c * nele + p] = vz; }
          else {
            kxx[c * nele + p] = kxx[(c + 1) * nele + p] + vx;
            kyy[c * nele + p] = kyy[(c + 1) * nele + p] + vy;
            kzz[c * nele + p] = kzz[(c + 1) * nele + p] + vz;
          }
        }
      }
    }
  }
}

/* correction(): p_aa = sum_i 0.5 (K_aa[idx_i] * rho)(r_i) rho_i dv / V^2 (one call, from 0) */
void orc_pc_correction(const double box[3], const int n[3], int nrc, const double* kxx,
                       const double* kyy, const double* kzz, const double* rho, const int* rcidx,
                       double p[3]) {
  long nele = (long)n[0] * n[1] * n[2];
  double V = box[0] * box[1] * box[2];
  double dv = (box[0] / n[0]) * (box[1] / n[1]) * (box[2] / n[2]);
  double* rk = (double*)malloc(sizeof(double) * 2 * nele);
  for (long i = 0; i < nele; ++i) { rk[2 * i] = rho[i]; rk[2 * i + 1] = 0; }
  orc_dft3d(n, rk, -1);
  for (long i = 0; i < 2 * nele; ++i) rk[i] *= V / nele;
  double* w = (double*)malloc(sizeof(double) * 2 * nele);
  const double* K[3] = {kxx, kyy, kzz};
  p[0] = p[1] = p[2] = 0;
  double* conv = (double*)malloc(sizeof(double) * nrc * nele);
  for (int d = 0; d < 3; ++d) {
    for (int c = 0; c < nrc; ++c) {
      for (long i = 0; i < nele; ++i) {
        double kk = K[d][c * nele + i];
        w[2 * i] = rk[2 * i] * kk;
        w[2 * i + 1] = rk[2 * i + 1] * kk;
      }
      orc_dft3d(n, w, +1);
      for (long i = 0; i < nele; ++i) conv[c * nele + i] = w[2 * i];
    }
    double s = 0;
    for (long i = 0; i < nele; ++i) s += 0.5 * conv[(long)rcidx[i] * nele + i] * rho[i] / V * dv;
    p[d] = s / V;
  }
  free(conv); free(w); free(rk);
}
