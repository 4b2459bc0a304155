// Inhomogeneous ik-SPME and real-space error estimates on a grid, FP64 on the GPU.
// Reference: ErrorEstimate_SPME_Ik::reinit / calKernel / calError
// (longRange.hetero/profile.test/template/tools/analyze/src/ErrorEstimate_SPME_Ik.cpp:80-470),
// driven by analyze/app/error.spme.ik.cpp:82-85 with the density profile of
// DensityProfile_PiecewiseConst (analyze/src/DensityProfile.cpp:7-90) on the
// same grid as the mesh.  With N grid points, V the volume, rectangular box:
//   g(m)       = -4 pi f(m) m*,  f = e^{-pi^2 |m*|^2/beta^2} / |m*|^2 / (2 pi V)
//   a_d(m, k)  = (u + 2 pi k)^-n / sum_{l=-3..3} (u + 2 pi l)^-n,  u = 2 pi m_d / K_d
//   k2b        = sum_{k = +-1..+-4} sum_dir V/N |IFFT(i g a_dir(k))|^2
//   k1         = V i g 2 sum_{k, dir} a_dir(k)          (k space)
//   k2a        = FFT(V/N |IFFT(k1 / V)|^2) + 2 FFT(k2b)
//   e1_d = IFFT(k1_d FFT(rho1 V/N)) q/V,  e2 = IFFT(k2a FFT(rho2 V/N)) q^2/V
//   error1 = sum_d e1_d^2 (real and imaginary parts apart), error2 = e2
// (components of g zeroed at the Nyquist index of an even K_d).  The kernel
// takes 25 batched 3D transforms at creation; an evaluation takes 2 + 4.
// rho1 is the density of charge signs, rho2 the number density of charges
// (profile1 / profile2 of the reference).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "device_common.cuh"

int dft3_grid(double2* data, const int n[3], int sign, int batch, cudaStream_t stream);

namespace {

struct EmGrid {
  int K[3];
  long N;
  double L[3];
};

__device__ __forceinline__ int em_c(int i, int K) { return i > (K >> 1) ? i - K : i; }
__device__ __forceinline__ void em_idx(long t, const EmGrid& g, int ii[3]) {
  ii[2] = (int)(t % g.K[2]);
  ii[1] = (int)((t / g.K[2]) % g.K[1]);
  ii[0] = (int)(t / ((long)g.K[2] * g.K[1]));
}

__device__ __forceinline__ double em_pow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

__device__ double em_alias(double u, int n) {
  double s = 1.0 / em_pow(u, n), up = u, un = u;
  for (int l = 0; l < 3; ++l) {
    up += 2.0 * M_PI;
    un -= 2.0 * M_PI;
    s += 1.0 / em_pow(up, n);
    s += 1.0 / em_pow(un, n);
  }
  return s;
}

__global__ void k_em_g(EmGrid g, double beta, double* gm /* [3][N] */, double* fmo /* [N] or null */) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  int ii[3];
  em_idx(t, g, ii);
  const double m[3] = {em_c(ii[0], g.K[0]) / g.L[0], em_c(ii[1], g.K[1]) / g.L[1], em_c(ii[2], g.K[2]) / g.L[2]};
  const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
  const double V = g.L[0] * g.L[1] * g.L[2];
  double fm = 0.0;
  if (m2 != 0.0) {
    const double tt = M_PI / beta;
    fm = exp(-tt * tt * m2) / m2 / (2.0 * M_PI * V);
  }
  for (int d = 0; d < 3; ++d) gm[d * g.N + t] = -4.0 * M_PI * fm * m[d];
  if (fmo) fmo[t] = fm;
}

// w_d = i g_d a(k) for one (k, dir), or with k == 0 the final 2 sum_{k, dir} a
// over 0 < |k| <= kcut; k1 (nullable) receives V w
__global__ void k_em_fill(EmGrid g, int order, int kcut, const double* gm, int k, int dir, double2* w,
                          double2* k1) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  int ii[3];
  em_idx(t, g, ii);
  double a = 0.0;
  if (t != 0) {
    if (k != 0) {
      const double u = 2.0 * M_PI * em_c(ii[dir], g.K[dir]) / g.K[dir];
      a = 1.0 / em_pow(u + 2.0 * M_PI * k, order) * (1.0 / em_alias(u, order));
    } else {
      double u[3], fen[3];
      for (int d = 0; d < 3; ++d) {
        u[d] = 2.0 * M_PI * em_c(ii[d], g.K[d]) / g.K[d];
        fen[d] = 1.0 / em_alias(u[d], order);
      }
      for (int kk = -kcut; kk <= kcut; ++kk) {
        if (kk == 0) continue;
        for (int d = 0; d < 3; ++d) a += 1.0 / em_pow(u[d] + 2.0 * M_PI * kk, order) * fen[d];
      }
      a *= 2.0;
    }
  }
  const double V = g.L[0] * g.L[1] * g.L[2];
  for (int d = 0; d < 3; ++d) {
    double v = gm[d * g.N + t] * a;
    if (t == 0 || ((g.K[d] % 2 == 0) && ii[d] == (g.K[d] >> 1))) v = 0.0;
    w[d * g.N + t] = make_double2(0.0, v);
    if (k1) k1[d * g.N + t] = make_double2(0.0, v * V);
  }
}

// out (+)= sum_d |w_d|^2 V / N as a real complex value
__global__ void k_em_sq(EmGrid g, const double2* w, double2* out, int accumulate) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  double s = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double2 v = w[d * g.N + t];
    s += v.x * v.x + v.y * v.y;
  }
  const double V = g.L[0] * g.L[1] * g.L[2];
  s *= V / (double)g.N;
  if (accumulate) out[t].x += s;
  else out[t] = make_double2(s, 0.0);
}

__global__ void k_em_axpy(long N, double2* a, const double2* b, double c) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= N) return;
  a[t].x += c * b[t].x;
  a[t].y += c * b[t].y;
}

// ---- analytic-differentiation map (ErrorEstimate_SPME_Ana, analyze/src/
// ErrorEstimate_SPME_Ana.cpp:220-667).  F_d(m, k) = -2 f(m) a_d(m, k) is the
// alias-k force kernel of the differentiated B-spline (zero at the Nyquist
// index of an even K_d); A*_dd = L_e L_f / V is the reciprocal box diagonal.
__device__ __forceinline__ double ema_fm(const EmGrid& g, int order, double fm, const int ii[3], int d, int k) {
  if ((g.K[d] % 2 == 0) && ii[d] == (g.K[d] >> 1)) return 0.0;
  const double u = 2.0 * M_PI * em_c(ii[d], g.K[d]) / g.K[d];
  double fen = 1.0 / em_pow(u + 2.0 * M_PI * k, order);
  fen /= em_alias(u, order);
  return -2.0 * fm * fen;
}

__host__ __device__ __forceinline__ double ema_astar(const double L[3], int d) {
  const double V = L[0] * (L[1] * L[2]);
  const int e = (d + 1) % 3, f = (d + 2) % 3;
  return (L[e < f ? e : f] * L[e < f ? f : e]) * (1.0 / V);
}

// component dir of w (k space) set to i (g_dir a_dir(k) + 2 pi k K_dir A*_dd F_dir(k));
// the other components of w are left as they are
__global__ void k_ema_fill_diff(EmGrid g, int order, const double* gm, const double* fm, int k, int dir,
                                double2* w) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  int ii[3];
  em_idx(t, g, ii);
  double v = 0.0;
  if (t != 0) {
    const double u = 2.0 * M_PI * em_c(ii[dir], g.K[dir]) / g.K[dir];
    const double a = 1.0 / em_pow(u + 2.0 * M_PI * k, order) * (1.0 / em_alias(u, order));
    v = gm[dir * g.N + t] * a;
    if ((g.K[dir] % 2 == 0) && ii[dir] == (g.K[dir] >> 1)) v = 0.0;
  }
  v += 2.0 * M_PI * (double)k * g.K[dir] * ema_astar(g.L, dir) * ema_fm(g, order, fm[t], ii, dir, k);
  w[dir * g.N + t] = make_double2(0.0, v);
}

// sum over the grid of F_d(m, k), one block of 256 per (k, d): out[ki * 3 + d],
// ki = 0..2 kcut - 1 for k = -kcut..-1, 1..kcut
__global__ void k_ema_selfsum(EmGrid g, int order, int kcut, const double* fm, double* out) {
  const int b = blockIdx.x, d = b % 3, ki = b / 3;
  const int k = ki < kcut ? ki - kcut : ki - kcut + 1;
  double s = 0.0;
  for (long t = threadIdx.x; t < g.N; t += blockDim.x) {
    int ii[3];
    em_idx(t, g, ii);
    s += ema_fm(g, order, fm[t], ii, d, k);
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = red[0];
}

// f(m) alone (the scalar factor of g)
__global__ void k_ema_fm(EmGrid g, double beta, double* fmo) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  int ii[3];
  em_idx(t, g, ii);
  const double m[3] = {em_c(ii[0], g.K[0]) / g.L[0], em_c(ii[1], g.K[1]) / g.L[1], em_c(ii[2], g.K[2]) / g.L[2]};
  const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
  const double V = g.L[0] * g.L[1] * g.L[2];
  double fm = 0.0;
  if (m2 != 0.0) {
    const double tt = M_PI / beta;
    fm = exp(-tt * tt * m2) / m2 / (2.0 * M_PI * V);
  }
  fmo[t] = fm;
}

// e_d = FFT(rho1 V/N) * V F_d(k) for the three d (FConvRho1 before its backward transform)
__global__ void k_ema_fconv(EmGrid g, int order, const double* fm, int k, const double2* r1, double2* e) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  int ii[3];
  em_idx(t, g, ii);
  const double V = g.L[0] * (g.L[1] * g.L[2]);
  const double2 c = r1[t];
  for (int d = 0; d < 3; ++d) {
    const double b = ema_fm(g, order, fm[t], ii, d, k) * V;
    e[d * g.N + t] = make_double2(c.x * b, c.y * b);
  }
}

__global__ void k_ema_div(long n, double2* a, double s) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  a[t].x /= s;
  a[t].y /= s;
}

__global__ void k_em_load(EmGrid g, const double* rho1, const double* rho2, double2* r) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  const double s = g.L[0] * g.L[1] * g.L[2] / (double)g.N;
  r[t] = make_double2(rho1[t] * s, 0.0);
  r[g.N + t] = make_double2(rho2[t] * s, 0.0);
}

__global__ void k_em_mult(EmGrid g, const double2* k1, const double2* k2a, const double2* r, double2* e) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  const double2 r1 = r[t], r2 = r[g.N + t];
  for (int d = 0; d < 3; ++d) {
    const double2 a = k1[d * g.N + t];
    e[d * g.N + t] = make_double2(r1.x * a.x - r1.y * a.y, r1.x * a.y + r1.y * a.x);
  }
  const double2 b = k2a[t];
  e[3 * g.N + t] = make_double2(r2.x * b.x - r2.y * b.y, r2.x * b.y + r2.y * b.x);
}

__global__ void k_em_finish(EmGrid g, const double2* e, double charge, double* e1, double* e2) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= g.N) return;
  const double V = g.L[0] * g.L[1] * g.L[2];
  double s0 = 0.0, s1 = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double re = e[d * g.N + t].x * charge / V, im = e[d * g.N + t].y;  // calError scales the real parts
    s0 += re * re;
    s1 += im * im;
  }
  e1[2 * t] = s0;
  e1[2 * t + 1] = s1;
  e2[2 * t] = e[3 * g.N + t].x * charge * charge / V;
  e2[2 * t + 1] = e[3 * g.N + t].y;
}

// profile of charge signs and of charges, counts per grid bin
// (DensityProfile_PiecewiseConst::reinit_conf binning)
template <class R>
__global__ void k_em_deposit(int N, const typename V4<R>::T* pos, EmGrid g, double* cnt1, double* cnt2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const typename V4<R>::T p = pos[i];
  if (p.w == R(0)) return;
  const double c[3] = {(double)p.x, (double)p.y, (double)p.z};
  unsigned b[3];
  for (int d = 0; d < 3; ++d) {
    double x = c[d];
    if (x >= g.L[d]) x -= g.L[d];
    else if (x < 0) x += g.L[d];
    const double q = x / (g.L[d] / g.K[d]);
    b[d] = q > 0 ? (unsigned)q : 0u;
    if (b[d] >= (unsigned)g.K[d]) b[d] = g.K[d] - 1;
  }
  const long idx = b[2] + (long)g.K[2] * (b[1] + (long)g.K[1] * b[0]);
  atomicAdd(&cnt1[idx], p.w > R(0) ? 1.0 : -1.0);
  atomicAdd(&cnt2[idx], 1.0);
}

__global__ void k_em_profile(long N, const double* cnt1, const double* cnt2, double inv, double* rho1, double* rho2) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= N) return;
  rho1[t] = cnt1[t] * inv;
  rho2[t] = cnt2[t] * inv;
}

// ---- real-space map (ErrorEstimate_dir, analyze/src/ErrorEstimate_dir.cpp:124-331)
// Integrands: 0: r f(r)^2 sin(2 pi k r), 1: r^2 f(r)^2, 2: -2 erfc(beta r) sin(2 pi k r),
// f(r) = (2 beta/sqrt(pi) e^{-beta^2 r^2} + erfc(beta r)/r) / r.
__device__ double dir_f(int kind, double k, double beta, double r) {
  if (kind == 2) return -2. * erfc(beta * r) * sin(2. * M_PI * k * r);
  const double betar = beta * r, ri = 1. / r;
  const double fr = (2. * beta / sqrt(M_PI) * exp(-betar * betar) + erfc(betar) * ri) * ri;
  if (kind == 0) return r * fr * fr * sin(2. * M_PI * k * r);
  return r * r * fr * fr;
}

// Gauss-4 box of the analyze tools' Integral1D (src/Integral1D.cpp:60-85)
__device__ double dir_coarse(int kind, double k, double beta, double xlo, double xup) {
  const double hx = xup - xlo;
  const double v0 = sqrt((3 - 2 * sqrt(1.2)) / 7.), v1 = sqrt((3 + 2 * sqrt(1.2)) / 7.);
  const double x0 = 0.5 * (xup - xlo) * (-v1) + 0.5 * (xup + xlo);
  const double x1 = 0.5 * (xup - xlo) * (-v0) + 0.5 * (xup + xlo);
  const double x2 = 0.5 * (xup - xlo) * (+v0) + 0.5 * (xup + xlo);
  const double x3 = 0.5 * (xup - xlo) * (+v1) + 0.5 * (xup + xlo);
  const double w0 = (18 + sqrt(30.)) / 36., w1 = (18 - sqrt(30.)) / 36.;
  return 0.5 * hx * (w1 * (dir_f(kind, k, beta, x0) + dir_f(kind, k, beta, x3)) +
                     w0 * (dir_f(kind, k, beta, x1) + dir_f(kind, k, beta, x2)));
}

// Integral1D::cal_int(Gauss4, f, xlo, xup, tol, init_nx): init_nx boxes of
// tol/init_nx; a box is bisected while |coarse - (left + right)| >= 255 tol
// (children tol/2) and while its width is at least 1e-13 of the initial box.
// Depth first with an explicit stack; a stack deeper than DIR_MAXD or more
// than DIR_BUDGET boxes (the reference would not finish either) sets the
// quadrature flag and keeps the best value so far.
constexpr int DIR_MAXD = 56;
constexpr long DIR_BUDGET = 1L << 20;

__device__ double dir_int(int kind, double k, double beta, double xlo, double xup, double tol, int init_nx,
                          unsigned* flag) {
  double sa[DIR_MAXD], sb[DIR_MAXD], st[DIR_MAXD], sc[DIR_MAXD];
  const double hx = (xup - xlo) / (double)init_nx, nxi = 1. / (double)init_nx;
  double total = 0.0;
  long boxes = 0;
  for (int i = 0; i < init_nx; i++) {
    const double x = xlo + i * hx;
    int top = 1;
    sa[0] = x; sb[0] = x + hx; st[0] = tol * nxi; sc[0] = dir_coarse(kind, k, beta, x, x + hx);
    double part = 0.0;
    while (top > 0) {
      --top;
      const double a = sa[top], b = sb[top], t = st[top], coarse = sc[top];
      const double hh = 0.5 * (b - a);
      const double c0 = dir_coarse(kind, k, beta, a, a + hh), c1 = dir_coarse(kind, k, beta, a + hh, b);
      const double v = c0 + c1;
      ++boxes;
      if (fabs(coarse - v) < t * 255 || hh * 2 < 1e-13 * hx) { part += v; continue; }
      if (top + 2 > DIR_MAXD || boxes > DIR_BUDGET) { atomicOr(flag, 1u); part += v; continue; }
      sa[top] = a + hh; sb[top] = b; st[top] = t * 0.5; sc[top] = c1; ++top;  // right, popped later
      sa[top] = a; sb[top] = a + hh; st[top] = t * 0.5; sc[top] = c0; ++top;  // left first
    }
    total += part;
  }
  return total;
}

// one thread per octant point (ax, ay, az) >= 0; every sign image inside
// [-K/2, K - K/2) gets the values (the tables are exactly even in |k| and
// odd in k_d, so the images agree with a per-point evaluation)
__global__ void k_em_dir_tables(EmGrid g, double beta, double rcut, double2* k1, double2* k2a, unsigned* flag) {
  const int hx = g.K[0] / 2 + 1, hy = g.K[1] / 2 + 1, hz = g.K[2] / 2 + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= hx * hy * hz) return;
  const int az = t % hz, ay = (t / hz) % hy, ax = t / (hz * hy);
  const double* L = g.L;
  // makeS1k (|k| from the integer indices)
  const double k1m = sqrt(ax * ax / (L[0] * L[0]) + ay * ay / (L[1] * L[1]) + az * az / (L[2] * L[2]));
  double s1;
  if (k1m != 0) s1 = 2. / k1m * dir_int(0, k1m, beta, rcut, 30, 1e-20, 10, flag);
  else s1 = 4. * M_PI * dir_int(1, k1m, beta, rcut, 30, 1e-20, 10, flag);
  // makeS2k (|k| from the wave vector)
  const double kx0 = ax / L[0], ky0 = ay / L[1], kz0 = az / L[2];
  const double k = sqrt(kx0 * kx0 + ky0 * ky0 + kz0 * kz0);
  double an = 0.0, size = 0.0;
  if (k != 0) {
    an = dir_int(2, k, beta, rcut, 30, 1e-20, 10, flag) / k;
    const double e = 2. * M_PI * k * rcut;
    size = 2. * M_PI * rcut * erfc(beta * rcut) * (2. * cos(e) / e - 2. * sin(e) / (e * e));
    size /= k;
  }
  for (int sx = 0; sx < 2; ++sx) {
    const int ix = sx ? -ax : ax;
    if ((sx && ax == 0) || ix < -(g.K[0] / 2) || ix >= g.K[0] - g.K[0] / 2) continue;
    for (int sy = 0; sy < 2; ++sy) {
      const int iy = sy ? -ay : ay;
      if ((sy && ay == 0) || iy < -(g.K[1] / 2) || iy >= g.K[1] - g.K[1] / 2) continue;
      for (int sz = 0; sz < 2; ++sz) {
        const int iz = sz ? -az : az;
        if ((sz && az == 0) || iz < -(g.K[2] / 2) || iz >= g.K[2] - g.K[2] / 2) continue;
        const int lx = ix < 0 ? ix + g.K[0] : ix, ly = iy < 0 ? iy + g.K[1] : iy, lz = iz < 0 ? iz + g.K[2] : iz;
        const long p = lz + (long)g.K[2] * (ly + (long)g.K[1] * lx);
        k2a[p] = make_double2(s1, 0.0);
        const double kk[3] = {ix / L[0], iy / L[1], iz / L[2]};
        for (int d = 0; d < 3; ++d) {
          double v = 0.0;
          if (k != 0) {
            v = 2 * M_PI * kk[d] * an;
            v += size * kk[d];
          }
          k1[d * g.N + p] = make_double2(0.0, v);
        }
      }
    }
  }
}

}  // namespace

// alias images summed by the reciprocal maps (global_half_N_k_sum of
// ErrorEstimate_SPME_Ik.cpp:5 and ErrorEstimate_SPME_Ana.cpp:5)
constexpr int EM_KCUT_IK = 4;
constexpr int EM_KCUT_ANA = 2;

enum { EM_KIND_IK = 0, EM_KIND_DIR = 1, EM_KIND_ANA = 2 };

struct md_errmap {
  int device = 0;
  int kind = EM_KIND_IK;
  double self_error = 0;    // analytic map: self-force error of a unit charge (times q^4)
  cudaStream_t stream = nullptr;
  EmGrid g;
  double beta = 0;
  int order = 0;
  double2* k1 = nullptr;    // [3][N] k space
  double2* k2a = nullptr;   // [N] k space
  double2* work = nullptr;  // [4][N]
  double2* work2 = nullptr; // [2][N]
  double* rho = nullptr;    // [2][N] current profile (rho1, rho2)
  double* cnt = nullptr;    // [2][N] deposited counts
  int samples = 0;
};

static void em_free(md_errmap* h) {
  void* p[] = {h->k1, h->k2a, h->work, h->work2, h->rho, h->cnt};
  for (void* q : p) if (q) cudaFree(q);
  if (h->stream) cudaStreamDestroy(h->stream);
}

extern "C" int md_errmap_create(md_errmap** out, const int K[3], const double L[3], double beta, int order,
                                int device) {
  if (!out || !K || !L || !(beta > 0) || order < 2 || order > 14) {
    md_set_error("md_errmap_create: bad arguments");
    return MD_ERR_BADARG;
  }
  for (int d = 0; d < 3; ++d)
    if (K[d] < 2 || K[d] > 1024 || !(L[d] > 0)) {
      md_set_error("md_errmap_create: grid %d or box %g out of range on axis %d", K[d], L[d], d);
      return MD_ERR_BADARG;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    md_set_error("md_errmap_create: no CUDA device %d", device);
    return MD_ERR_CUDA;
  }
  MD_CUDA(cudaSetDevice(device));
  md_errmap* h = new md_errmap();
  h->device = device;
  h->beta = beta;
  h->order = order;
  for (int d = 0; d < 3; ++d) { h->g.K[d] = K[d]; h->g.L[d] = L[d]; }
  h->g.N = (long)K[0] * K[1] * K[2];
  const long N = h->g.N;
  double* gm = nullptr;
  double2* k2b = nullptr;
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&h->k1, sizeof(double2) * 3 * N) == cudaSuccess &&
            cudaMalloc(&h->k2a, sizeof(double2) * N) == cudaSuccess &&
            cudaMalloc(&h->work, sizeof(double2) * 4 * N) == cudaSuccess &&
            cudaMalloc(&h->work2, sizeof(double2) * 2 * N) == cudaSuccess &&
            cudaMalloc(&h->rho, sizeof(double) * 2 * N) == cudaSuccess &&
            cudaMalloc(&h->cnt, sizeof(double) * 2 * N) == cudaSuccess &&
            cudaMalloc(&gm, sizeof(double) * 3 * N) == cudaSuccess &&
            cudaMalloc(&k2b, sizeof(double2) * N) == cudaSuccess;
  auto fail = [&](int code) {
    if (gm) cudaFree(gm);
    if (k2b) cudaFree(k2b);
    em_free(h);
    delete h;
    return code;
  };
  if (!ok) return fail(md_cuda_fail(cudaGetLastError(), "md_errmap_create allocation"));
  cudaStream_t s = h->stream;
  const unsigned nb = (unsigned)((N + 255) / 256);
  MD_CUDA(cudaMemsetAsync(k2b, 0, sizeof(double2) * N, s));
  MD_CUDA(cudaMemsetAsync(h->cnt, 0, sizeof(double) * 2 * N, s));
  MD_CUDA(cudaMemsetAsync(h->rho, 0, sizeof(double) * 2 * N, s));
  k_em_g<<<nb, 256, 0, s>>>(h->g, beta, gm, nullptr);
  for (int k = -EM_KCUT_IK; k <= EM_KCUT_IK; ++k) {
    if (k == 0) continue;
    for (int dir = 0; dir < 3; ++dir) {
      k_em_fill<<<nb, 256, 0, s>>>(h->g, order, EM_KCUT_IK, gm, k, dir, h->work, nullptr);
      if (int r = dft3_grid(h->work, h->g.K, +1, 3, s)) return fail(r);
      k_em_sq<<<nb, 256, 0, s>>>(h->g, h->work, k2b, 1);
    }
  }
  k_em_fill<<<nb, 256, 0, s>>>(h->g, order, EM_KCUT_IK, gm, 0, 0, h->work, h->k1);
  if (int r = dft3_grid(h->work, h->g.K, +1, 3, s)) return fail(r);
  k_em_sq<<<nb, 256, 0, s>>>(h->g, h->work, h->k2a, 0);
  if (int r = dft3_grid(h->k2a, h->g.K, -1, 1, s)) return fail(r);
  if (int r = dft3_grid(k2b, h->g.K, -1, 1, s)) return fail(r);
  k_em_axpy<<<nb, 256, 0, s>>>(N, h->k2a, k2b, 2.0);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(gm);
  cudaFree(k2b);
  gm = nullptr;
  k2b = nullptr;
  if (e != cudaSuccess) return fail(md_cuda_fail(e, "md_errmap_create kernel"));
  *out = h;
  return MD_OK;
}

// ErrorEstimate_dir::reinit (analyze/src/ErrorEstimate_dir.cpp:70-122): the
// same object as the ik map with k1 = s2k and k2a = s1k, so set_profile,
// deposit and compute (calError) are shared
extern "C" int md_errmap_create_dir(md_errmap** out, const int K[3], const double L[3], double beta, double rcut,
                                    int device) {
  if (!out || !K || !L || !(beta > 0) || !(rcut > 0) || !(rcut < 30.0)) {
    md_set_error("md_errmap_create_dir: bad arguments (beta > 0, 0 < rcut < 30)");
    return MD_ERR_BADARG;
  }
  for (int d = 0; d < 3; ++d)
    if (K[d] < 2 || K[d] > 1024 || !(L[d] > 0)) {
      md_set_error("md_errmap_create_dir: grid %d or box %g out of range on axis %d", K[d], L[d], d);
      return MD_ERR_BADARG;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    md_set_error("md_errmap_create_dir: no CUDA device %d", device);
    return MD_ERR_CUDA;
  }
  MD_CUDA(cudaSetDevice(device));
  md_errmap* h = new md_errmap();
  h->device = device;
  h->beta = beta;
  h->order = 0;
  h->kind = EM_KIND_DIR;
  for (int d = 0; d < 3; ++d) { h->g.K[d] = K[d]; h->g.L[d] = L[d]; }
  h->g.N = (long)K[0] * K[1] * K[2];
  const long N = h->g.N;
  unsigned* flag = nullptr;
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&h->k1, sizeof(double2) * 3 * N) == cudaSuccess &&
            cudaMalloc(&h->k2a, sizeof(double2) * N) == cudaSuccess &&
            cudaMalloc(&h->work, sizeof(double2) * 4 * N) == cudaSuccess &&
            cudaMalloc(&h->work2, sizeof(double2) * 2 * N) == cudaSuccess &&
            cudaMalloc(&h->rho, sizeof(double) * 2 * N) == cudaSuccess &&
            cudaMalloc(&h->cnt, sizeof(double) * 2 * N) == cudaSuccess &&
            cudaMalloc(&flag, sizeof(unsigned)) == cudaSuccess;
  auto fail = [&](int code) {
    if (flag) cudaFree(flag);
    em_free(h);
    delete h;
    return code;
  };
  if (!ok) return fail(md_cuda_fail(cudaGetLastError(), "md_errmap_create_dir allocation"));
  cudaStream_t s = h->stream;
  MD_CUDA(cudaMemsetAsync(h->cnt, 0, sizeof(double) * 2 * N, s));
  MD_CUDA(cudaMemsetAsync(h->rho, 0, sizeof(double) * 2 * N, s));
  MD_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned), s));
  const int oct = (K[0] / 2 + 1) * (K[1] / 2 + 1) * (K[2] / 2 + 1);
  k_em_dir_tables<<<ceil_div(oct, 64), 64, 0, s>>>(h->g, beta, rcut, h->k1, h->k2a, flag);
  unsigned hf = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hf, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(md_cuda_fail(e, "md_errmap_create_dir kernel"));
  if (hf) {
    md_set_error("md_errmap_create_dir: the adaptive quadrature did not converge (erfc(beta rcut) too large "
                 "for the reference's tolerance)");
    return fail(MD_ERR_BADARG);
  }
  cudaFree(flag);
  flag = nullptr;
  *out = h;
  return MD_OK;
}

// ErrorEstimate_SPME_Ana::reinit / calKernel (analyze/src/ErrorEstimate_SPME_Ana.cpp:140-667):
//   self  = sum_{0<|k|<=2} sum_d (2 pi k K_d A*_dd)^2 (sum_m F_d(m, k))^2
//   k2b   = sum_{0<|k|<=2} sum_dir V/N (|IFFT(i g a_dir(k))|^2
//            + |IFFT(i g a_dir(k) + i 2 pi k K_dir A*_dd F_dir(k) e_dir)|^2)
//   k1    = V i g 2 sum_{k, dir} a_dir(k),  k2a = FFT(V/N |IFFT(k1 / V)|^2) + FFT(k2b)
// The second square of each (k, dir) changes component dir only; the other two
// keep the backward transforms of the first.
extern "C" int md_errmap_create_ana(md_errmap** out, const int K[3], const double L[3], double beta, int order,
                                    int device) {
  if (!out || !K || !L || !(beta > 0) || order < 2 || order > 14) {
    md_set_error("md_errmap_create_ana: bad arguments");
    return MD_ERR_BADARG;
  }
  for (int d = 0; d < 3; ++d)
    if (K[d] < 2 || K[d] > 1024 || !(L[d] > 0)) {
      md_set_error("md_errmap_create_ana: grid %d or box %g out of range on axis %d", K[d], L[d], d);
      return MD_ERR_BADARG;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    md_set_error("md_errmap_create_ana: no CUDA device %d", device);
    return MD_ERR_CUDA;
  }
  MD_CUDA(cudaSetDevice(device));
  md_errmap* h = new md_errmap();
  h->device = device;
  h->beta = beta;
  h->order = order;
  h->kind = EM_KIND_ANA;
  for (int d = 0; d < 3; ++d) { h->g.K[d] = K[d]; h->g.L[d] = L[d]; }
  h->g.N = (long)K[0] * K[1] * K[2];
  const long N = h->g.N;
  constexpr int NSELF = 2 * EM_KCUT_ANA * 3;
  double *gm = nullptr, *fm = nullptr, *selfs = nullptr;
  double2* k2b = nullptr;
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&h->k1, sizeof(double2) * 3 * N) == cudaSuccess &&
            cudaMalloc(&h->k2a, sizeof(double2) * N) == cudaSuccess &&
            cudaMalloc(&h->work, sizeof(double2) * 4 * N) == cudaSuccess &&
            cudaMalloc(&h->work2, sizeof(double2) * 2 * N) == cudaSuccess &&
            cudaMalloc(&h->rho, sizeof(double) * 2 * N) == cudaSuccess &&
            cudaMalloc(&h->cnt, sizeof(double) * 2 * N) == cudaSuccess &&
            cudaMalloc(&gm, sizeof(double) * 3 * N) == cudaSuccess &&
            cudaMalloc(&fm, sizeof(double) * N) == cudaSuccess &&
            cudaMalloc(&selfs, sizeof(double) * NSELF) == cudaSuccess &&
            cudaMalloc(&k2b, sizeof(double2) * N) == cudaSuccess;
  auto fail = [&](int code) {
    void* p[] = {gm, fm, selfs, k2b};
    for (void* q : p) if (q) cudaFree(q);
    em_free(h);
    delete h;
    return code;
  };
  if (!ok) return fail(md_cuda_fail(cudaGetLastError(), "md_errmap_create_ana allocation"));
  cudaStream_t s = h->stream;
  const unsigned nb = (unsigned)((N + 255) / 256);
  MD_CUDA(cudaMemsetAsync(k2b, 0, sizeof(double2) * N, s));
  MD_CUDA(cudaMemsetAsync(h->cnt, 0, sizeof(double) * 2 * N, s));
  MD_CUDA(cudaMemsetAsync(h->rho, 0, sizeof(double) * 2 * N, s));
  k_em_g<<<nb, 256, 0, s>>>(h->g, beta, gm, fm);
  k_ema_selfsum<<<NSELF, 256, 0, s>>>(h->g, order, EM_KCUT_ANA, fm, selfs);
  for (int k = -EM_KCUT_ANA; k <= EM_KCUT_ANA; ++k) {
    if (k == 0) continue;
    for (int dir = 0; dir < 3; ++dir) {
      k_em_fill<<<nb, 256, 0, s>>>(h->g, order, EM_KCUT_ANA, gm, k, dir, h->work, nullptr);
      if (int r = dft3_grid(h->work, h->g.K, +1, 3, s)) return fail(r);
      k_em_sq<<<nb, 256, 0, s>>>(h->g, h->work, k2b, 1);
      k_ema_fill_diff<<<nb, 256, 0, s>>>(h->g, order, gm, fm, k, dir, h->work);
      if (int r = dft3_grid(h->work + dir * N, h->g.K, +1, 1, s)) return fail(r);
      k_em_sq<<<nb, 256, 0, s>>>(h->g, h->work, k2b, 1);
    }
  }
  k_em_fill<<<nb, 256, 0, s>>>(h->g, order, EM_KCUT_ANA, gm, 0, 0, h->work, h->k1);
  if (int r = dft3_grid(h->work, h->g.K, +1, 3, s)) return fail(r);
  k_em_sq<<<nb, 256, 0, s>>>(h->g, h->work, h->k2a, 0);
  if (int r = dft3_grid(h->k2a, h->g.K, -1, 1, s)) return fail(r);
  if (int r = dft3_grid(k2b, h->g.K, -1, 1, s)) return fail(r);
  k_em_axpy<<<nb, 256, 0, s>>>(N, h->k2a, k2b, 1.0);
  double hs[NSELF];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hs, selfs, sizeof(hs), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(md_cuda_fail(e, "md_errmap_create_ana kernel"));
  double self = 0.0;
  for (int ki = 0; ki < 2 * EM_KCUT_ANA; ++ki) {
    const int k = ki < EM_KCUT_ANA ? ki - EM_KCUT_ANA : ki - EM_KCUT_ANA + 1;
    for (int d = 0; d < 3; ++d) {
      const double astar = ema_astar(L, d), sd = hs[ki * 3 + d];
      self += 4. * M_PI * M_PI * k * k * K[d] * K[d] * astar * astar * sd * sd;
    }
  }
  h->self_error = self;
  cudaFree(gm); cudaFree(fm); cudaFree(selfs); cudaFree(k2b);
  gm = fm = selfs = nullptr;
  k2b = nullptr;
  *out = h;
  return MD_OK;
}

extern "C" int md_errmap_self_error(md_errmap* h, double* out) {
  if (!h || !out) return MD_ERR_BADARG;
  *out = h->self_error;
  return MD_OK;
}

// FConvRho1_d(k) of ErrorEstimate_SPME_Ana::calError: IFFT(FFT(rho1 V/N) V F_d(k)) / V
// for the three d, out [3][N][2]
extern "C" int md_errmap_ana_fconv(md_errmap* h, int k, double* out) {
  if (!h || !out) return MD_ERR_BADARG;
  if (h->kind != EM_KIND_ANA) {
    md_set_error("md_errmap_ana_fconv: the map is not the analytic-differentiation map");
    return MD_ERR_BADARG;
  }
  if (k == 0 || k < -EM_KCUT_ANA || k > EM_KCUT_ANA) {
    md_set_error("md_errmap_ana_fconv: alias index %d outside 0 < |k| <= %d", k, EM_KCUT_ANA);
    return MD_ERR_BADARG;
  }
  MD_CUDA(cudaSetDevice(h->device));
  cudaStream_t s = h->stream;
  const long N = h->g.N;
  const unsigned nb = (unsigned)((N + 255) / 256);
  double* fm = reinterpret_cast<double*>(h->work + 3 * N);  // last N complex of work: f(m)
  k_em_load<<<nb, 256, 0, s>>>(h->g, h->rho, h->rho + N, h->work2);
  if (int r = dft3_grid(h->work2, h->g.K, -1, 1, s)) return r;
  k_ema_fm<<<nb, 256, 0, s>>>(h->g, h->beta, fm);
  k_ema_fconv<<<nb, 256, 0, s>>>(h->g, h->order, fm, k, h->work2, h->work);
  if (int r = dft3_grid(h->work, h->g.K, +1, 3, s)) return r;
  const double V = h->g.L[0] * (h->g.L[1] * h->g.L[2]);
  k_ema_div<<<(unsigned)((3 * N + 255) / 256), 256, 0, s>>>(3 * N, h->work, V);
  MD_CHECK_LAUNCH("errmap fconv");
  MD_CUDA(cudaMemcpyAsync(out, h->work, sizeof(double2) * 3 * N, cudaMemcpyDeviceToHost, s));
  MD_CUDA(cudaStreamSynchronize(s));
  return MD_OK;
}

extern "C" int md_errmap_destroy(md_errmap* h) {
  if (!h) return MD_OK;
  cudaSetDevice(h->device);
  em_free(h);
  delete h;
  return MD_OK;
}

extern "C" int md_errmap_set_profile(md_errmap* h, const double* rho1, const double* rho2) {
  if (!h || !rho1 || !rho2) return MD_ERR_BADARG;
  MD_CUDA(cudaSetDevice(h->device));
  const size_t b = sizeof(double) * h->g.N;
  MD_CUDA(cudaMemcpyAsync(h->rho, rho1, b, cudaMemcpyHostToDevice, h->stream));
  MD_CUDA(cudaMemcpyAsync(h->rho + h->g.N, rho2, b, cudaMemcpyHostToDevice, h->stream));
  MD_CUDA(cudaStreamSynchronize(h->stream));
  return MD_OK;
}

// one sample of the system's charges (sign and number per bin); the profile
// becomes the average over the samples deposited so far
extern "C" int md_errmap_deposit(md_errmap* h, md_system* sys) {
  if (!h || !sys) return MD_ERR_BADARG;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  for (int d = 0; d < 3; ++d)
    if (std::fabs(hs.L[d] - h->g.L[d]) > 1e-12 * h->g.L[d]) {
      md_set_error("md_errmap_deposit: the system box differs from the error map's");
      return MD_ERR_BADARG;
    }
  const int nb = ceil_div(sys->N, 256);
  if (sys->prec == MD_PREC_FP64)
    k_em_deposit<double><<<nb, 256, 0, sys->stream>>>(sys->N, (const double4a*)sys->pos, h->g, h->cnt,
                                                      h->cnt + h->g.N);
  else
    k_em_deposit<float><<<nb, 256, 0, sys->stream>>>(sys->N, (const float4*)sys->pos, h->g, h->cnt, h->cnt + h->g.N);
  MD_CHECK_LAUNCH("errmap deposit");
  h->samples += 1;
  const double dv = h->g.L[0] * h->g.L[1] * h->g.L[2] / (double)h->g.N;
  k_em_profile<<<(unsigned)((h->g.N + 255) / 256), 256, 0, sys->stream>>>(h->g.N, h->cnt, h->cnt + h->g.N,
                                                                         1.0 / (dv * h->samples), h->rho,
                                                                         h->rho + h->g.N);
  MD_CHECK_LAUNCH("errmap profile");
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}

// ErrorEstimate_SPME_Ik::calError: error1 [N][2], error2 [N][2] (real, imaginary);
// the RMS force error of a grid point is sqrt(error1[i][0] + error2[i][0])
// the convolutions of calError: work[0..3) = IFFT(k1_d FFT(rho1 V/N)),
// work[3] = IFFT(k2a FFT(rho2 V/N)), unscaled
static int em_convolve(md_errmap* h) {
  MD_CUDA(cudaSetDevice(h->device));
  cudaStream_t s = h->stream;
  const long N = h->g.N;
  const unsigned nb = (unsigned)((N + 255) / 256);
  k_em_load<<<nb, 256, 0, s>>>(h->g, h->rho, h->rho + N, h->work2);
  if (int r = dft3_grid(h->work2, h->g.K, -1, 2, s)) return r;
  k_em_mult<<<nb, 256, 0, s>>>(h->g, h->k1, h->k2a, h->work2, h->work);
  return dft3_grid(h->work, h->g.K, +1, 4, s);
}

__global__ void k_em_meanf(long N, const double2* e, double scale, double* out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 3 * N) return;
  out[t] = e[t].x * scale;
}

// print_meanf of the maps (ErrorEstimate_SPME_Ana.cpp:806-842): the mean force error
// field e1_d = Re IFFT(k1_d FFT(rho1 V/N)) q / V, out [3][K0][K1][K2]
extern "C" int md_errmap_mean_force(md_errmap* h, double charge, double* out) {
  if (!h || !out) return MD_ERR_BADARG;
  if (int r = em_convolve(h)) return r;
  const long N = h->g.N;
  const double V = h->g.L[0] * h->g.L[1] * h->g.L[2];
  double* d = reinterpret_cast<double*>(h->work2);  // 2N complex = 4N doubles >= 3N
  k_em_meanf<<<(unsigned)((3 * N + 255) / 256), 256, 0, h->stream>>>(N, h->work, charge / V, d);
  MD_CHECK_LAUNCH("errmap mean force");
  MD_CUDA(cudaMemcpyAsync(out, d, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, h->stream));
  MD_CUDA(cudaStreamSynchronize(h->stream));
  return MD_OK;
}

extern "C" int md_errmap_compute(md_errmap* h, double charge, double* error1, double* error2) {
  if (!h || !error1 || !error2) return MD_ERR_BADARG;
  if (int r = em_convolve(h)) return r;
  cudaStream_t s = h->stream;
  const long N = h->g.N;
  const unsigned nb = (unsigned)((N + 255) / 256);
  double* d = reinterpret_cast<double*>(h->work2);  // 4N doubles: error1, error2
  k_em_finish<<<nb, 256, 0, s>>>(h->g, h->work, charge, d, d + 2 * N);
  MD_CHECK_LAUNCH("errmap compute");
  MD_CUDA(cudaMemcpyAsync(error1, d, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, s));
  MD_CUDA(cudaMemcpyAsync(error2, d + 2 * N, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, s));
  MD_CUDA(cudaStreamSynchronize(s));
  return MD_OK;
}

extern "C" int md_errmap_get_profile(md_errmap* h, double* rho1, double* rho2) {
  if (!h) return MD_ERR_BADARG;
  MD_CUDA(cudaSetDevice(h->device));
  MD_CUDA(cudaStreamSynchronize(h->stream));
  if (rho1) MD_CUDA(cudaMemcpy(rho1, h->rho, sizeof(double) * h->g.N, cudaMemcpyDeviceToHost));
  if (rho2) MD_CUDA(cudaMemcpy(rho2, h->rho + h->g.N, sizeof(double) * h->g.N, cudaMemcpyDeviceToHost));
  return MD_OK;
}

// ---------------------------------------------------------------------------
// Choice of the splitting parameter and the mesh for an inhomogeneous system
// (no counterpart function in the reference; it applies the reference's error
// estimates the way their users pick beta and K).  The budget is split evenly:
// target / sqrt(2) for the real space and for the reciprocal space.
//  - beta: the real-space estimate of errorEstimatePME
//    (RE/src/ElectrostaticInteraction.cpp:349-401), 2 q_rms sqrt(c2 / (N rcut V))
//    exp(-beta^2 rcut^2), taken with c2 / V replaced by the largest local sum
//    of q^2 per volume, averaged over cubes of edge about 2 rcut around each
//    bin of a rcut/2 grid: the short-range limit of the inhomogeneous real-space
//    map.  (The map itself, ErrorEstimate_dir, is built by a quadrature that
//    does not converge at the beta rcut of about 3 that such targets need.)
//  - K: powers of two per axis.  Starting from the homogeneous ik estimate
//    (EleRecBSpline.cpp:154-206), the axis with the coarsest spacing is
//    doubled until the largest per-bin RMS error of the inhomogeneous ik-SPME
//    map (ErrorEstimate_SPME_Ik) of the system's charge profile on that mesh
//    is within budget, then the axis with the finest spacing is halved while
//    it stays within budget.
__global__ void k_em_rms_max(long n, const double* e1, const double* e2, unsigned long long* out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double v = 0.0;
  if (t < n) {
    const double s = e1[2 * t] + e2[2 * t];
    v = s > 0.0 ? sqrt(s) : 0.0;  // a negative sum is rounding in an empty bin
  }
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
}

// largest per-bin RMS force error of the ik map on mesh K for the system's profile
static int em_ik_max(md_system* sys, const int K[3], const double L[3], double beta, int order, double charge,
                     double* out) {
  md_errmap* h = nullptr;
  if (int r = md_errmap_create(&h, K, L, beta, order, sys->device)) return r;
  int r = md_errmap_deposit(h, sys);
  unsigned long long* dmax = nullptr;
  if (!r && cudaMallocAsync((void**)&dmax, sizeof(unsigned long long), h->stream) != cudaSuccess)
    r = md_cuda_fail(cudaGetLastError(), "error map maximum");
  if (!r) r = em_convolve(h);
  if (!r) {
    const long N = h->g.N;
    const unsigned nb = (unsigned)((N + 255) / 256);
    double* d = reinterpret_cast<double*>(h->work2);
    cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), h->stream);
    k_em_finish<<<nb, 256, 0, h->stream>>>(h->g, h->work, charge, d, d + 2 * N);
    k_em_rms_max<<<nb, 256, 0, h->stream>>>(N, d, d + 2 * N, dmax);
    unsigned long long bits = 0;
    if (cudaMemcpyAsync(&bits, dmax, sizeof(bits), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      r = md_cuda_fail(cudaGetLastError(), "error map maximum");
    double v;
    memcpy(&v, &bits, sizeof(v));
    *out = v;
  }
  if (dmax) cudaFreeAsync(dmax, h->stream);
  md_errmap_destroy(h);
  return r;
}

extern "C" int md_choose_spme_params(md_system* sys, double rcut, int order, double target, int kmax,
                                     double* beta, int K[3], double* err_dir, double* err_rec) {
  if (!sys || !(rcut > 0) || order < 2 || order > 14 || !(target > 0) || !beta || !K || kmax < 2 * order) {
    md_set_error("md_choose_spme_params: bad arguments");
    return MD_ERR_BADARG;
  }
  if (kmax > 1024) kmax = 1024;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  const int N = sys->N;
  std::vector<double> pos(3 * (size_t)N), q(N);
  if (int r = md_system_get_positions(sys, pos.data())) return r;
  if (int r = md_system_get_charges(sys, q.data())) return r;
  double c2 = 0.0;
  for (double v : q) c2 += v * v;
  if (!(c2 > 0)) { md_set_error("md_choose_spme_params: the system has no charges"); return MD_ERR_BADARG; }
  const double qrms = sqrt(c2 / N);
  // local q^2 density: bins of at most rcut/2, box average over +-m bins (periodic)
  int nb[3], m[3];
  double hb[3];
  for (int d = 0; d < 3; ++d) {
    nb[d] = std::max(1, (int)floor(hs.L[d] / (0.5 * rcut)));
    hb[d] = hs.L[d] / nb[d];
    m[d] = std::min((int)ceil(rcut / hb[d]), (nb[d] - 1) / 2);
  }
  const size_t nbt = (size_t)nb[0] * nb[1] * nb[2];
  std::vector<double> w(nbt, 0.0), t1(nbt), t2(nbt);
  for (int i = 0; i < N; ++i) {
    int b[3];
    for (int d = 0; d < 3; ++d) {
      double x = pos[3 * (size_t)i + d] - floor(pos[3 * (size_t)i + d] / hs.L[d]) * hs.L[d];
      b[d] = std::min(nb[d] - 1, std::max(0, (int)(x / hb[d])));
    }
    w[b[2] + (size_t)nb[2] * (b[1] + (size_t)nb[1] * b[0])] += q[i] * q[i];
  }
  // separable periodic box filter along z, y, x
  auto filt = [&](const std::vector<double>& in, std::vector<double>& out, int axis) {
    for (int i0 = 0; i0 < nb[0]; ++i0)
      for (int i1 = 0; i1 < nb[1]; ++i1)
        for (int i2 = 0; i2 < nb[2]; ++i2) {
          double s = 0.0;
          for (int k = -m[axis]; k <= m[axis]; ++k) {
            int c[3] = {i0, i1, i2};
            c[axis] = ((c[axis] + k) % nb[axis] + nb[axis]) % nb[axis];
            s += in[c[2] + (size_t)nb[2] * (c[1] + (size_t)nb[1] * c[0])];
          }
          out[i2 + (size_t)nb[2] * (i1 + (size_t)nb[1] * i0)] = s;
        }
  };
  filt(w, t1, 2);
  filt(t1, t2, 1);
  filt(t2, t1, 0);
  double vol = 1.0;
  for (int d = 0; d < 3; ++d) vol *= (2 * m[d] + 1) * hb[d];
  double rho_max = 0.0;
  for (double v : t1) rho_max = std::max(rho_max, v / vol);
  const double tb = target / sqrt(2.0);
  const double pre = 2.0 * qrms * sqrt(rho_max / rcut);
  const double b = sqrt(std::max(log(pre / tb), 1.0)) / rcut;
  *beta = b;
  if (err_dir) *err_dir = pre * exp(-b * b * rcut * rcut);
  // mesh: homogeneous estimate first, then the inhomogeneous map
  int k[3];
  for (int d = 0; d < 3; ++d) {
    k[d] = 1;
    while (k[d] <= order) k[d] <<= 1;
  }
  // meshes are kept to at most 2^27 points (an ik map of that size holds
  // about 30 GB of FP64 kernels and profiles)
  const long long max_points = 1ll << 27;
  auto coarsest = [&](int lim) {
    int a = -1;
    const long long pts = (long long)k[0] * k[1] * k[2];
    for (int d = 0; d < 3; ++d)
      if (2 * k[d] <= lim && 2 * pts <= max_points && (a < 0 || hs.L[d] / k[d] > hs.L[a] / k[a])) a = d;
    return a;
  };
  for (int it = 0; it < 40; ++it) {
    double e = 0.0;
    if (int r = md_error_estimate_spme_ik(sys, k, order, b, &e)) return r;
    if (e <= tb) break;
    const int a = coarsest(kmax);
    if (a < 0) break;
    k[a] *= 2;
  }
  double e = 0.0;
  for (int it = 0; it < 40; ++it) {
    if (int r = em_ik_max(sys, k, hs.L, b, order, qrms, &e)) return r;
    if (e <= tb) break;
    const int a = coarsest(kmax);
    if (a < 0) {
      md_set_error("md_choose_spme_params: meshes up to %d per axis and 2^27 points give %g > %g in reciprocal "
                   "space", kmax, e, tb);
      return MD_ERR_BADARG;
    }
    k[a] *= 2;
  }
  for (int it = 0; it < 40; ++it) {
    int a = -1;
    for (int d = 0; d < 3; ++d)
      if (k[d] / 2 > order && (a < 0 || hs.L[d] / k[d] < hs.L[a] / k[a])) a = d;
    if (a < 0) break;
    k[a] /= 2;
    double e2 = 0.0;
    if (int r = em_ik_max(sys, k, hs.L, b, order, qrms, &e2)) return r;
    if (e2 > tb) {
      k[a] *= 2;
      break;
    }
    e = e2;
  }
  for (int d = 0; d < 3; ++d) K[d] = k[d];
  if (err_rec) *err_rec = e;
  return MD_OK;
}
