/* ORACLE build shim (test infrastructure only): FFTW3-API subset over our
 * own FP64 transforms, so that the md.error reference sources (which call
 * FFTW) compile and run here.  Power-of-two lines use an iterative radix-2
 * FFT, other lengths a direct O(n^2) DFT.  All transforms are unnormalised. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "shim/fftw3.h"

struct orc_fftw_plan_s {
  int kind; /* 0 c2c, 1 r2c, 2 c2r */
  int n[3];
  int sign;
  void* in;
  void* out;
};

void* fftw_malloc(size_t n) { return malloc(n ? n : 1); }
void fftw_free(void* p) { free(p); }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void line_fft(double* re, double* im, int n, int sign, double* tr, double* ti) {
  if (is_pow2(n)) {
    /* bit-reversal permutation then butterflies */
    for (int i = 1, j = 0; i < n; ++i) {
      int bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) {
        double t = re[i]; re[i] = re[j]; re[j] = t;
        t = im[i]; im[i] = im[j]; im[j] = t;
      }
    }
    for (int len = 2; len <= n; len <<= 1) {
      for (int i = 0; i < n; i += len) {
        for (int k = 0; k < len / 2; ++k) {
          double ang = sign * 2.0 * M_PI * k / len;
          double wr = cos(ang), wi = sin(ang);
          int a = i + k, b = i + k + len / 2;
          double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
          re[b] = re[a] - xr; im[b] = im[a] - xi;
          re[a] += xr; im[a] += xi;
        }
      }
    }
    return;
  }
  for (int k = 0; k < n; ++k) {
    double sr = 0, si = 0;
    for (int j = 0; j < n; ++j) {
      long m = ((long)j * k) % n;
      double ang = sign * 2.0 * M_PI * (double)m / n;
      double c = cos(ang), s = sin(ang);
      sr += re[j] * c - im[j] * s;
      si += re[j] * s + im[j] * c;
    }
    tr[k] = sr; ti[k] = si;
  }
  memcpy(re, tr, sizeof(double) * n);
  memcpy(im, ti, sizeof(double) * n);
}

/* in-place 3D transform of split re/im arrays [n0][n1][n2] */
static void fft3(const int n[3], double* re, double* im, int sign) {
  int nmax = n[0] > n[1] ? n[0] : n[1];
  if (n[2] > nmax) nmax = n[2];
  double* lr = (double*)malloc(sizeof(double) * nmax * 4);
  double* li = lr + nmax;
  double* tr = li + nmax;
  double* ti = tr + nmax;
  long s[3] = {(long)n[1] * n[2], n[2], 1};
  for (int ax = 0; ax < 3; ++ax) {
    int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
    for (int i1 = 0; i1 < n[a1]; ++i1)
      for (int i2 = 0; i2 < n[a2]; ++i2) {
        long base = i1 * s[a1] + i2 * s[a2];
        for (int k = 0; k < n[ax]; ++k) { lr[k] = re[base + k * s[ax]]; li[k] = im[base + k * s[ax]]; }
        line_fft(lr, li, n[ax], sign, tr, ti);
        for (int k = 0; k < n[ax]; ++k) { re[base + k * s[ax]] = lr[k]; im[base + k * s[ax]] = li[k]; }
      }
  }
  free(lr);
}

static fftw_plan mk(int kind, int n0, int n1, int n2, void* in, void* out, int sign) {
  fftw_plan p = (fftw_plan)malloc(sizeof(*p));
  p->kind = kind; p->n[0] = n0; p->n[1] = n1; p->n[2] = n2;
  p->sign = sign; p->in = in; p->out = out;
  return p;
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
  (void)flags;
  return mk(0, n0, n1, n2, in, out, sign);
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned flags) {
  (void)flags;
  return mk(1, n0, n1, n2, in, out, -1);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned flags) {
  (void)flags;
  return mk(2, n0, n1, n2, in, out, +1);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }

void fftw_execute(const fftw_plan p) {
  const int* n = p->n;
  long nele = (long)n[0] * n[1] * n[2];
  long nh = (long)n[0] * n[1] * (n[2] / 2 + 1);
  double* re = (double*)malloc(sizeof(double) * nele);
  double* im = (double*)malloc(sizeof(double) * nele);
  if (p->kind == 0) {
    const double* in = (const double*)p->in;
    for (long i = 0; i < nele; ++i) { re[i] = in[2 * i]; im[i] = in[2 * i + 1]; }
    fft3(n, re, im, p->sign);
    double* out = (double*)p->out;
    for (long i = 0; i < nele; ++i) { out[2 * i] = re[i]; out[2 * i + 1] = im[i]; }
  } else if (p->kind == 1) {
    const double* in = (const double*)p->in;
    for (long i = 0; i < nele; ++i) { re[i] = in[i]; im[i] = 0; }
    fft3(n, re, im, -1);
    double* out = (double*)p->out;
    int h = n[2] / 2 + 1;
    for (int a = 0; a < n[0]; ++a)
      for (int b = 0; b < n[1]; ++b)
        for (int c = 0; c < h; ++c) {
          long src = c + (long)n[2] * (b + (long)n[1] * a), dst = c + (long)h * (b + (long)n[1] * a);
          out[2 * dst] = re[src];
          out[2 * dst + 1] = im[src];
        }
  } else {
    const double* in = (const double*)p->in;
    int h = n[2] / 2 + 1;
    for (int a = 0; a < n[0]; ++a)
      for (int b = 0; b < n[1]; ++b)
        for (int c = 0; c < n[2]; ++c) {
          long dst = c + (long)n[2] * (b + (long)n[1] * a);
          if (c < h) {
            long src = c + (long)h * (b + (long)n[1] * a);
            re[dst] = in[2 * src];
            im[dst] = in[2 * src + 1];
          } else {
            int a2 = (n[0] - a) % n[0], b2 = (n[1] - b) % n[1], c2 = n[2] - c;
            long src = c2 + (long)h * (b2 + (long)n[1] * a2);
            re[dst] = in[2 * src];
            im[dst] = -in[2 * src + 1];
          }
        }
    fft3(n, re, im, +1);
    double* out = (double*)p->out;
    for (long i = 0; i < nele; ++i) out[i] = re[i];
  }
  (void)nh;
  free(re);
  free(im);
}
