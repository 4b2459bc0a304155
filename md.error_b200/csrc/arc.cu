// Adaptive cutoff estimate (AdaptRCut), its density profile and the tail
// pressure correction, all in FP64 on the GPU.
// Reference (ENG = shortRange.inhomo/template/tools/simulation.hetero.cutoff):
//   DensityProfile_PiecewiseConst  ENG/src/DensityProfile.cu:27-99
//   AdaptRCut::makeS1k/makeS2k     ENG/src/AdaptRCut.cu:265-416
//   AdaptRCut::calError/calRCut/refineRCut  ENG/src/AdaptRCut.cu:182-508
//   Integral1D Gauss4              ENG/src/Integral1D.cu:164-232
//   PressureCorrection             ENG/src/PressureCorrection.cu:175-340
//   AssignRCut::getRCut + assign   ENG/src/AssignRCut.cu:46-117
//
// k-space kernels: the radial integrals depend on |k| only, so one thread per
// point of the k-grid octant runs the adaptive Gauss-4 quadrature (explicit
// stack, same subdivision rule as the reference) for every rc interval and
// writes the kernel values of all sign images.  The 3D transforms of the
// (odd-sized) bin grid are batched direct DFTs along each axis with the line
// and its twiddles in shared memory.  Error map, bisection and refinement are
// element-wise kernels; nothing returns to the host until asked.
#include <cmath>
#include <cstring>
#include <algorithm>
#include <vector>
#include "device_common.cuh"

struct md_adapt_rcut {
  int n[3] = {0, 0, 0};
  long nele = 0;
  int nrc = 0;
  std::vector<double> rc;
  // the box at construction: DensityProfile_PiecewiseConst::reinit,
  // AdaptRCut::reinit and PressureCorrection::reinit take it once
  // (ENG/src/DensityProfile.cu:22-43, ENG/src/AdaptRCut.cu:96-162,
  // ENG/src/PressureCorrection.cu:41-54) and bin, build the kernel tables and
  // normalise with it for the whole run, also when NPT moves the box
  double box_tab[3] = {0, 0, 0};
  double* d_rc = nullptr;
  double* counts = nullptr;   // deposited atom counts per bin
  double* rho = nullptr;      // profile (calculate)
  double2* rhok = nullptr;
  double* s1k = nullptr;      // [nrc][nele] real
  double* s2k = nullptr;      // [3][nrc][nele] imaginary
  double* pck = nullptr;      // [3][nrc][nele] real (pressure-correction kernels)
  double* ints = nullptr;     // [4][nrc][octant points] radial integrals of the tables
  double2* work = nullptr;    // [4*nrc][nele]
  double* error = nullptr;    // [nrc][nele]
  double* rcut = nullptr;     // [nele]
  int* rcidx = nullptr;       // [nele]
  int* rcidx2 = nullptr;
  double* rerr = nullptr;
  double* pcorr = nullptr;    // [3]
  int ndata = 0;
  cudaStream_t stream = nullptr;
  md_system* sys = nullptr;
};

// ------------------------------------------------------------ quadrature
__device__ __forceinline__ double pow_int_d(double x, int nn) {
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

// integrands: 13 -> x^-13 sin(2 pi k x); 5 -> x^-5 sin(2 pi k x);
// 1 / 25 -> -24 x^-4.5 J_{1/2}(2 pi k x) / J_{5/2}(2 pi k x) (closed forms)
__device__ __forceinline__ double fn_eval(int kind, double k, double x) {
  double s, c;
  sincospi(2.0 * k * x, &s, &c);
  if (kind == 13) return pow_int_d(x, -13) * s;
  if (kind == 5) return pow_int_d(x, -5) * s;
  const double z = 2.0 * M_PI * k * x;
  const double pre = -24.0 / (pow_int_d(x, 4) * sqrt(x));
  if (z == 0.0) return 0.0;
  const double r = sqrt(2.0 / (M_PI * z));
  if (kind == 1) return pre * r * s;
  return pre * r * ((3.0 / (z * z) - 1.0) * s - 3.0 * c / z);
}

__device__ double g4_coarse(int kind, double k, double xlo, double xup) {
  const double v0 = 0.33998104358485626, v1 = 0.86113631159405258;   // Gauss-Legendre 4 nodes
  const double w0 = 0.65214515486254614, w1 = 0.34785484513745386;   // and weights
  const double hm = 0.5 * (xup - xlo), c = 0.5 * (xup + xlo);
  return hm * (w1 * (fn_eval(kind, k, c - hm * v1) + fn_eval(kind, k, c + hm * v1)) +
               w0 * (fn_eval(kind, k, c - hm * v0) + fn_eval(kind, k, c + hm * v0)));
}

// Integral1D::cal_int(Gauss4, f, xlo, xup, tol): bisect a box while
// |coarse - (left + right)| >= 255 tol, children get tol/2; stop below
// 1e-13 of the interval.  Depth-first with an explicit stack.
__device__ double g4_adaptive(int kind, double k, double xlo, double xup, double tol, unsigned* flags) {
  const int MAXD = 64;
  double sa[MAXD], sb[MAXD], st[MAXD], sc[MAXD];
  int top = 0;
  const double ghx = xup - xlo;
  sa[0] = xlo; sb[0] = xup; st[0] = tol; sc[0] = g4_coarse(kind, k, xlo, xup);
  top = 1;
  double total = 0.0;
  while (top > 0) {
    --top;
    const double a = sa[top], b = sb[top], t = st[top], coarse = sc[top];
    const double hh = 0.5 * (b - a);
    const double c0 = g4_coarse(kind, k, a, a + hh), c1 = g4_coarse(kind, k, a + hh, b);
    const double v = c0 + c1;
    if (fabs(coarse - v) < t * 255 || hh * 2 < 1e-13 * ghx) { total += v; continue; }
    if (top + 2 > MAXD) { atomicOr(flags, FLAG_QUADRATURE); total += v; continue; }
    sa[top] = a + hh; sb[top] = b; st[top] = t * 0.5; sc[top] = c1; ++top;   // right, popped later
    sa[top] = a; sb[top] = a + hh; st[top] = t * 0.5; sc[top] = c0; ++top;   // left first
  }
  return total;
}

__device__ __forceinline__ long lin(const int n[3], int x, int y, int z) { return z + (long)n[2] * (y + (long)n[1] * x); }

struct ArcDims { int n[3]; int nrc; double box[3]; };

__device__ __forceinline__ double oct_k(const ArcDims& g, int t) {
  const int hy = g.n[1] / 2 + 1, hz = g.n[2] / 2 + 1;
  const int az = t % hz, ay = (t / hz) % hy, ax = t / (hz * hy);
  const double kx0 = ax / g.box[0], ky0 = ay / g.box[1], kz0 = az / g.box[2];
  return sqrt(kx0 * kx0 + ky0 * ky0 + kz0 * kz0);
}

// The radial integrals of the tables, one thread per (integrand, cutoff
// interval, octant point): the integrand kinds 13, 5, 1 and 25 over
// [rc_c, rc_{c+1}] (the last up to 30) with the reference's tolerances.
// A warp covers 32 octant points of one (kind, interval).
__global__ void k_arc_integrals(ArcDims g, const double* rc, double* ints, unsigned* flags) {
  const int noct = (g.n[0] / 2 + 1) * (g.n[1] / 2 + 1) * (g.n[2] / 2 + 1);
  const int nrc = g.nrc;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * nrc * noct) return;
  const int pt = (int)(t % noct), c = (int)((t / noct) % nrc), kind = (int)(t / ((long)noct * nrc));
  const double k = oct_k(g, pt);
  double v = 0.0;
  if (k != 0) {
    const double hi = (c == nrc - 1) ? 30.0 : rc[c + 1];
    const int kinds[4] = {13, 5, 1, 25};
    const double tols[4] = {1e-12, 1e-16, 1e-7, 1e-7};
    v = g4_adaptive(kinds[kind], k, rc[c], hi, tols[kind], flags);
  }
  ints[t] = v;
}

// one thread per octant point (ax, ay, az) >= 0: the cumulative sums of the
// radial integrals and the angular factors, written to every sign image
__global__ void k_arc_tables(ArcDims g, const double* rc, const double* ints, double* s1k, double* s2k,
                             double* pck) {
  const int hx = g.n[0] / 2 + 1, hy = g.n[1] / 2 + 1, hz = g.n[2] / 2 + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int noct = hx * hy * hz;
  if (t >= noct) return;
  const int az = t % hz, ay = (t / hz) % hy, ax = t / (hz * hy);
  const int nrc = g.nrc;
  const long nele = (long)g.n[0] * g.n[1] * g.n[2];
  const double eps = 1.0, sigma = 1.0;
  const double pref = 16. * 36. * pow_int_d(sigma, 12) * eps;
  const double pre = 8. * eps * pow_int_d(sigma, 6);
  const double k = oct_k(g, t);
  const int MAXRC = 32;
  double S1[MAXRC], T[MAXRC], I1[MAXRC], I5[MAXRC];
  auto integral = [&](int kind, int c) { return ints[((long)kind * nrc + c) * noct + t]; };
  // cumulative integrals from the top interval [rc_last, 30] down
  double cum13 = 0, cum5 = 0;
  for (int c = nrc - 1; c >= 0; --c) {
    if (k != 0) {
      cum13 += 2. / k * pref * integral(0, c);
      S1[c] = cum13;
      cum5 += integral(1, c) * pre / k * 2 * M_PI;
      const double r = rc[c], r6 = pow_int_d(r, 6);
      const double e = 2. * M_PI * k * r;
      double size = -2. * M_PI * r * r * (4. * eps * pow_int_d(sigma, 6) / r6) * (2. * cos(e) / e - 2. * sin(e) / (e * e));
      size /= k;
      T[c] = cum5 + size;
      I1[c] = integral(2, c);
      I5[c] = integral(3, c);
    } else {
      S1[c] = 4. * M_PI * pref / 11. * pow_int_d(rc[c], -11);
      T[c] = 0;
      I1[c] = I5[c] = 0;
    }
  }
  // write every sign image of this octant point
  for (int sx = 0; sx < 2; ++sx) {
    if (sx && ax == 0) continue;
    for (int sy = 0; sy < 2; ++sy) {
      if (sy && ay == 0) continue;
      for (int sz = 0; sz < 2; ++sz) {
        if (sz && az == 0) continue;
        const int ix = sx ? -ax : ax, iy = sy ? -ay : ay, iz = sz ? -az : az;
        const int lx = ix < 0 ? ix + g.n[0] : ix, ly = iy < 0 ? iy + g.n[1] : iy, lz = iz < 0 ? iz + g.n[2] : iz;
        const long p = lin(g.n, lx, ly, lz);
        const double kx = ix / g.box[0], ky = iy / g.box[1], kz = iz / g.box[2];
        // angular factors of PressureCorrection::makeKernel
        double cp = 0, sp = 0, c2t = 1;
        if (k != 0) {
          const double phi = acos(kz / k);
          double theta = 0.;
          if (phi != 0.) {
            double tt = kx / (k * sin(phi));
            tt = fmin(1.0, fmax(-1.0, tt));
            theta = acos(tt);
            if (ky < 0) theta = 2. * M_PI - theta;
          }
          cp = cos(phi); sp = sin(phi); c2t = cos(theta * 2);
        }
        const double sc = (k != 0) ? M_PI / sqrt(k) : 0.0;
        double cx = 0, cy = 0, cz = 0;
        for (int c = nrc - 1; c >= 0; --c) {
          s1k[(long)c * nele + p] = S1[c];
          s2k[(0L * nrc + c) * nele + p] = kx * T[c];
          s2k[(1L * nrc + c) * nele + p] = ky * T[c];
          s2k[(2L * nrc + c) * nele + p] = kz * T[c];
          if (k != 0) {
            cx += sc * (2. / 3. * I1[c] + (-1. / 3. + cp * cp - sp * sp * c2t) * I5[c]);
            cy += sc * (2. / 3. * I1[c] + (-1. / 3. + cp * cp + sp * sp * c2t) * I5[c]);
            cz += sc * 4. / 3. * (0.5 * I1[c] + (0.5 - 1.5 * cp * cp) * I5[c]);
          }
          pck[(0L * nrc + c) * nele + p] = cx;
          pck[(1L * nrc + c) * nele + p] = cy;
          pck[(2L * nrc + c) * nele + p] = cz;
        }
      }
    }
  }
}

// ------------------------------------------------------------ batched DFT
// One block per line; lines of all `batch` arrays of the grid along `axis`.
// out[k] = sum_j in[j] exp(sign 2 pi i jk/n), in place.  n <= 1024.
// A block takes `per` lines of one axis (several short lines per block, so
// that lanes are not idle on 41-point lines).  A line of composite length
// n = n1 n2 (n1 its smallest prime factor) is transformed in two stages
// (Cooley-Tukey: n2 inner DFTs of length n1, the twiddles W_n^{j2 k1}, n1
// DFTs of length n2), n (n1 + n2) products instead of n^2; a prime length
// is summed directly.  All factors come from one table of W_n^m.
__global__ void k_dft_axis(double2* data, ArcDims g, int axis, int sign, int batch, int n1, int per) {
  extern __shared__ double2 sm[];
  const int n = g.n[axis], n2 = n / n1;
  double2* tw = sm;                  // [n]
  double2* lines_sm = sm + n;        // [per][n] input, then stage-1 output
  double2* tmp = lines_sm + per * n; // [per][n] stage-1 results (two-stage only)
  const long nele = (long)g.n[0] * g.n[1] * g.n[2];
  const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
  const long lines = (long)g.n[a1] * g.n[a2];
  const long stride[3] = {(long)g.n[1] * g.n[2], (long)g.n[2], 1};
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double s, c;
    sincospi(2.0 * j / n, &s, &c);
    tw[j] = make_double2(c, sign * s);
  }
  // load the block's lines
  double2* base[8];
  for (int q = 0; q < per; ++q) {
    const long lid = (long)blockIdx.x * per + q;
    base[q] = nullptr;
    if (lid < lines * batch) {
      const int b = (int)(lid / lines);
      const long r = lid % lines;
      const int i1 = (int)(r / g.n[a2]), i2 = (int)(r % g.n[a2]);
      base[q] = data + (long)b * nele + i1 * stride[a1] + i2 * stride[a2];
    }
  }
  for (int t = threadIdx.x; t < per * n; t += blockDim.x) {
    const int q = t / n, j = t - q * n;
    lines_sm[t] = base[q] ? base[q][j * stride[axis]] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  auto cmul_acc = [](double2& acc, const double2 x, const double2 w) {
    acc.x += x.x * w.x - x.y * w.y;
    acc.y += x.x * w.y + x.y * w.x;
  };
  if (n1 == n) {
    for (int t = threadIdx.x; t < per * n; t += blockDim.x) {
      const int q = t / n, kk = t - q * n;
      if (!base[q]) continue;
      const double2* line = lines_sm + q * n;
      double2 acc = make_double2(0.0, 0.0);
      int m = 0;
      for (int j = 0; j < n; ++j) {
        cmul_acc(acc, line[j], tw[m]);
        m += kk;
        if (m >= n) m -= n;
      }
      base[q][kk * stride[axis]] = acc;
    }
    return;
  }
  // stage 1: y[k1][j2] = W_n^{j2 k1} sum_j1 x[n2 j1 + j2] W_n1^{j1 k1}
  for (int t = threadIdx.x; t < per * n; t += blockDim.x) {
    const int q = t / n, r = t - q * n, k1 = r / n2, j2 = r - k1 * n2;
    const double2* line = lines_sm + q * n;
    double2 acc = make_double2(0.0, 0.0);
    const int step = (k1 * n2) % n;  // W_n1^{k1} = W_n^{k1 n2}
    int m = 0;
    for (int j1 = 0; j1 < n1; ++j1) {
      cmul_acc(acc, line[n2 * j1 + j2], tw[m]);
      m += step;
      if (m >= n) m -= n;
    }
    const double2 w = tw[(j2 * k1) % n];
    tmp[q * n + r] = make_double2(acc.x * w.x - acc.y * w.y, acc.x * w.y + acc.y * w.x);
  }
  __syncthreads();
  // stage 2: X[k1 + n1 k2] = sum_j2 y[k1][j2] W_n2^{j2 k2}
  for (int t = threadIdx.x; t < per * n; t += blockDim.x) {
    const int q = t / n, r = t - q * n, k1 = r % n1, k2 = r / n1;
    if (!base[q]) continue;
    const double2* y = tmp + q * n + k1 * n2;
    double2 acc = make_double2(0.0, 0.0);
    const int step = (k2 * n1) % n;  // W_n2^{k2} = W_n^{k2 n1}
    int m = 0;
    for (int j2 = 0; j2 < n2; ++j2) {
      cmul_acc(acc, y[j2], tw[m]);
      m += step;
      if (m >= n) m -= n;
    }
    base[q][(k1 + n1 * k2) * stride[axis]] = acc;
  }
}

// Power-of-two lines: radix-2 Stockham FFT of one line per block in shared
// memory (autosorting, natural order in and out; Govindaraju et al., SC'08),
// same convention and result as k_dft_axis.  Stage Ns (1, 2, 4, ...): for
// butterfly j < n/2, k = j mod Ns, v1 = x[j + n/2] exp(sign i pi k / Ns);
// y[2 Ns floor(j/Ns) + k] = x[j] + v1, y[... + Ns] = x[j] - v1.  Twiddles
// exp(sign 2 pi i t / n), t < n/2, from FP64 sincospi once per block.
__global__ void k_fft2_axis(double2* data, ArcDims g, int axis, int sign, int batch, int logn) {
  extern __shared__ double2 sm[];
  const int n = 1 << logn, h = n >> 1;
  double2* x = sm;
  double2* y = sm + n;
  double2* tw = sm + 2 * n;
  const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
  const long lines = (long)g.n[a1] * g.n[a2];
  const long lid = blockIdx.x;
  if (lid >= lines * batch) return;
  const long nele = (long)g.n[0] * g.n[1] * g.n[2];
  const int b = (int)(lid / lines);
  const long r = lid % lines;
  const int i1 = (int)(r / g.n[a2]), i2 = (int)(r % g.n[a2]);
  const long stride[3] = {(long)g.n[1] * g.n[2], (long)g.n[2], 1};
  double2* base = data + (long)b * nele + i1 * stride[a1] + i2 * stride[a2];
  const long st = stride[axis];
  for (int j = threadIdx.x; j < n; j += blockDim.x) x[j] = base[j * st];
  for (int t = threadIdx.x; t < h; t += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * t / n, &sn, &cs);
    tw[t] = make_double2(cs, sign * sn);
  }
  __syncthreads();
  for (int ls = 0; ls < logn; ++ls) {
    const int Ns = 1 << ls;
    for (int j = threadIdx.x; j < h; j += blockDim.x) {
      const int k = j & (Ns - 1);
      const double2 w = tw[k << (logn - 1 - ls)];  // exp(sign i pi k / Ns)
      const double2 v0 = x[j], u = x[j + h];
      const double2 v1 = make_double2(u.x * w.x - u.y * w.y, u.x * w.y + u.y * w.x);
      const int d = ((j >> ls) << (ls + 1)) + k;
      y[d] = make_double2(v0.x + v1.x, v0.y + v1.y);
      y[d + Ns] = make_double2(v0.x - v1.x, v0.y - v1.y);
    }
    __syncthreads();
    double2* t = x;
    x = y;
    y = t;
  }
  for (int j = threadIdx.x; j < n; j += blockDim.x) base[j * st] = x[j];
}

// unnormalised 3D DFT (sign -1 forward, +1 backward) of `batch` consecutive
// complex grids [n0][n1][n2], in place, any sizes up to 1024 per axis;
// power-of-two axes by the FFT above, others by the direct sum
int dft3_grid(double2* data, const int n[3], int sign, int batch, cudaStream_t stream) {
  ArcDims g;
  for (int d = 0; d < 3; ++d) g.n[d] = n[d];
  for (int axis = 2; axis >= 0; --axis) {
    const int na = g.n[axis];
    long lines = (long)g.n[(axis + 1) % 3] * g.n[(axis + 2) % 3] * batch;
    if (na >= 2 && (na & (na - 1)) == 0) {
      int logn = 0;
      while ((1 << logn) < na) ++logn;
      const size_t smem = sizeof(double2) * (2 * na + na / 2);
      k_fft2_axis<<<(unsigned)lines, 128, smem, stream>>>(data, g, axis, sign, batch, logn);
      MD_CHECK_LAUNCH("fft axis");
    } else {
      int n1 = na;  // smallest prime factor
      for (int f = 2; f * f <= na; ++f)
        if (na % f == 0) { n1 = f; break; }
      const int per = std::max(1, std::min(8, 128 / na));  // lines per block
      size_t smem = sizeof(double2) * (na + 2 * (size_t)per * na);
      k_dft_axis<<<(unsigned)((lines + per - 1) / per), 128, smem, stream>>>(data, g, axis, sign, batch, n1, per);
      MD_CHECK_LAUNCH("dft axis");
    }
  }
  return MD_OK;
}

static int dft3(md_adapt_rcut* a, double2* data, int sign, int batch) {
  return dft3_grid(data, a->n, sign, batch, a->sys->stream);
}

// ------------------------------------------------------------ element-wise kernels
template <class R>
__global__ void k_arc_deposit(int N, const typename V4<R>::T* pos, ArcDims g, double* counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const typename V4<R>::T p = pos[i];
  const double c[3] = {(double)(float)p.x, (double)(float)p.y, (double)(float)p.z};
  unsigned b[3];
  for (int d = 0; d < 3; ++d) {
    const double L = g.box[d];  // the profile's box (fixed at construction)
    double tmp = c[d];
    if (c[d] >= L) tmp -= L; else if (c[d] < 0) tmp += L;
    const double h = L / g.n[d];
    double q = tmp / h;
    b[d] = q > 0 ? (unsigned)q : 0u;
    if (b[d] >= (unsigned)g.n[d]) b[d] = g.n[d] - 1;
  }
  atomicAdd(&counts[b[2] + (long)g.n[2] * (b[1] + (long)g.n[1] * b[0])], 1.0);
}

__global__ void k_arc_profile(long nele, const double* counts, double inv, double* rho, double2* out) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  const double r = counts ? counts[i] * inv : rho[i];
  rho[i] = r;
  out[i] = make_double2(r, 0.0);
}

// The four products of each cutoff, s1k rho_k and i s2k_d rho_k (d = x, y, z),
// are Hermitian (rho real, s1k real and even, s2k real and odd), so their
// inverse transforms are real; they go two to a complex transform, A + i B,
// whose real part is IFFT(A) and imaginary part IFFT(B):
//   work[2c]     = s1k r + i (i s2k_x r) = (s1k - s2k_x) r
//   work[2c + 1] = i s2k_y r + i (i s2k_z r) = (-s2k_z + i s2k_y) r
__global__ void k_arc_multiply(long nele, int nrc, const double2* rhok, double scale, const double* s1k,
                               const double* s2k, double2* work) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  const double2 r = make_double2(rhok[i].x * scale, rhok[i].y * scale);
  for (int c = 0; c < nrc; ++c) {
    const double s = s1k[(long)c * nele + i];
    const double bx = s2k[((long)0 * nrc + c) * nele + i];
    const double by = s2k[((long)1 * nrc + c) * nele + i];
    const double bz = s2k[((long)2 * nrc + c) * nele + i];
    work[(long)(2 * c) * nele + i] = make_double2(r.x * (s - bx), r.y * (s - bx));
    work[(long)(2 * c + 1) * nele + i] = make_double2(-by * r.y - bz * r.x, by * r.x - bz * r.y);
  }
}

__global__ void k_arc_error(long nele, int nrc, const double2* work, double Vi, double* error) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  for (int c = 0; c < nrc; ++c) {
    const double2 a = work[(long)(2 * c) * nele + i], b = work[(long)(2 * c + 1) * nele + i];
    const double e1 = a.x * Vi, ex = a.y * Vi, ey = b.x * Vi, ez = b.y * Vi;
    error[(long)c * nele + i] = sqrt(e1 + ex * ex + ey * ey + ez * ez);
  }
}

// calRCutOnePoint (AdaptRCut.cu:418-460)
__global__ void k_arc_rcut(long nele, int nrc, const double* rc, const double* error, double prec,
                           double* rcut, int* idx, double* rerr) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  unsigned a = 0, b = nrc - 1;
  const double ea = error[i], eb0 = error[(long)b * nele + i];
  if (ea - prec <= 0) { rcut[i] = rc[a]; idx[i] = a; rerr[i] = ea; return; }
  if (eb0 - prec >= 0) { rcut[i] = rc[b]; idx[i] = b; rerr[i] = eb0; return; }
  double eb = eb0;
  while (b - a > 1) {
    const unsigned c = (a + b) / 2;
    const double ec = error[(long)c * nele + i];
    if (ec > prec) a = c; else { b = c; eb = ec; }
  }
  rcut[i] = rc[b]; idx[i] = b; rerr[i] = eb;
}

// refineRCut (AdaptRCut.cu:470-508)
__global__ void k_arc_refine(ArcDims g, const int* in, int* out, const double* rc, const double* error,
                             double* rcut, double* rerr) {
  const long nele = (long)g.n[0] * g.n[1] * g.n[2];
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  const int z = (int)(i % g.n[2]), y = (int)((i / g.n[2]) % g.n[1]), x = (int)(i / ((long)g.n[2] * g.n[1]));
  int m = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz) {
        const int jx = (x + dx + g.n[0]) % g.n[0], jy = (y + dy + g.n[1]) % g.n[1], jz = (z + dz + g.n[2]) % g.n[2];
        m = max(m, in[lin(g.n, jx, jy, jz)]);
      }
  out[i] = m;
  rcut[i] = rc[m];
  rerr[i] = error[(long)m * nele + i];
}

// pck_aa rho_k is Hermitian (pck real and even): xx and yy of a cutoff share
// one complex transform, (pck_xx + i pck_yy) r in work[c], zz is work[nrc + c]
__global__ void k_pc_multiply(long nele, int nrc, const double2* rhok, double scale, const double* pck, double2* work) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  const double2 r = make_double2(rhok[i].x * scale, rhok[i].y * scale);
  for (int c = 0; c < nrc; ++c) {
    const double kx = pck[((long)0 * nrc + c) * nele + i], ky = pck[((long)1 * nrc + c) * nele + i];
    const double kz = pck[((long)2 * nrc + c) * nele + i];
    work[(long)c * nele + i] = make_double2(kx * r.x - ky * r.y, kx * r.y + ky * r.x);
    work[(long)(nrc + c) * nele + i] = make_double2(r.x * kz, r.y * kz);
  }
}

// PressureCorrection::correction (ENG/src/PressureCorrection.cu:175-211) adds the
// new sum to the members pxx, pyy, pzz, which it never resets, and then divides
// them by V: p_new = (p_old + S / V) / V with S = sum_i 0.5 conv_aa[idx_i](i)
// rho_i dv.  The old value's share is scaled here; k_pc_reduce then adds S / V^2.
__global__ void k_pc_carry(double* p, double inv_volume) {
  if (threadIdx.x < 3) p[threadIdx.x] *= inv_volume;
}

// p_aa += sum_i 0.5 conv_aa[idx_i](i) rho_i dv / V^2
__global__ void k_pc_reduce(long nele, int nrc, const double2* work, const int* idx, const double* rho,
                            double fac, double* partials, unsigned* counter, double* out) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double v[3] = {0, 0, 0};
  if (i < nele) {
    const int c = idx[i];
    const double2 xy = work[(long)c * nele + i];
    const double conv[3] = {xy.x, xy.y, work[(long)(nrc + c) * nele + i].x};
    for (int d = 0; d < 3; ++d) v[d] = 0.5 * conv[d] * rho[i] * fac;
  }
  block_reduce_finish<3>(v, partials, counter, out, false);
}

__global__ void k_store_pcorr(const double* p, DevState* st) {
  for (int d = 0; d < 3; ++d) st->stats[MD_STAT_PRESSURE_CORR_XX + d] = p[d];
}

__global__ void k_lattice_from_rcut(long nele, const double* rcut, float* lat, DevState* st) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < nele) lat[i] = (float)rcut[i];
  if (i == 0) atomicOr(&st->flags, FLAG_FORCE_REBUILD);
}

// ------------------------------------------------------------ host side
static int build_tables(md_adapt_rcut* a) {
  DevState hs;
  if (int r = a->sys->read_state(hs)) return r;
  ArcDims g;
  for (int d = 0; d < 3; ++d) { g.n[d] = a->n[d]; g.box[d] = hs.L[d]; a->box_tab[d] = hs.L[d]; }
  g.nrc = a->nrc;
  int oct = (g.n[0] / 2 + 1) * (g.n[1] / 2 + 1) * (g.n[2] / 2 + 1);
  k_arc_integrals<<<ceil_div(4L * g.nrc * oct, 128), 128, 0, a->sys->stream>>>(g, a->d_rc, a->ints,
                                                                              &a->sys->st->flags);
  MD_CHECK_LAUNCH("arc integrals");
  k_arc_tables<<<ceil_div(oct, 64), 64, 0, a->sys->stream>>>(g, a->d_rc, a->ints, a->s1k, a->s2k, a->pck);
  MD_CHECK_LAUNCH("arc tables");
  return MD_OK;
}

extern "C" int md_arc_create(md_adapt_rcut** out, md_system* sys, double refh, double rcmin, double rcmax,
                             double rcstep) {
  if (!out || !sys || !(refh > 0) || !(rcmin > 0) || !(rcmax >= rcmin) || !(rcstep > 0)) {
    md_set_error("md_arc_create: bad arguments");
    return MD_ERR_BADARG;
  }
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  md_adapt_rcut* a = new md_adapt_rcut();
  a->sys = sys;
  a->sys->stream = sys->stream;
  for (int d = 0; d < 3; ++d) {  // DensityProfile_PiecewiseConst::reinit: odd bin counts
    unsigned v = (unsigned)(hs.L[d] / refh);
    if ((v - (v / 2) * 2) == 0) v++;
    a->n[d] = (int)v;
  }
  if (a->n[0] > 1024 || a->n[1] > 1024 || a->n[2] > 1024) {
    delete a;
    md_set_error("md_arc_create: more than 1024 bins along one direction");
    return MD_ERR_BADARG;
  }
  for (double r = rcmin; r <= rcmax; r += rcstep) a->rc.push_back(r);  // AdaptRCut::reinit rcList
  a->nrc = (int)a->rc.size();
  if (a->nrc > 32) { delete a; md_set_error("md_arc_create: at most 32 cutoffs"); return MD_ERR_BADARG; }
  a->nele = (long)a->n[0] * a->n[1] * a->n[2];
  const long ne = a->nele;
  const int nrc = a->nrc;
  bool ok = cudaMalloc(&a->d_rc, sizeof(double) * nrc) == cudaSuccess &&
            cudaMalloc(&a->counts, sizeof(double) * ne) == cudaSuccess &&
            cudaMalloc(&a->rho, sizeof(double) * ne) == cudaSuccess &&
            cudaMalloc(&a->rhok, sizeof(double2) * ne) == cudaSuccess &&
            cudaMalloc(&a->s1k, sizeof(double) * nrc * ne) == cudaSuccess &&
            cudaMalloc(&a->s2k, sizeof(double) * 3 * nrc * ne) == cudaSuccess &&
            cudaMalloc(&a->pck, sizeof(double) * 3 * nrc * ne) == cudaSuccess &&
            cudaMalloc(&a->ints, sizeof(double) * 4 * nrc * (size_t)((a->n[0] / 2 + 1) * (a->n[1] / 2 + 1) *
                                                                    (a->n[2] / 2 + 1))) == cudaSuccess &&
            cudaMalloc(&a->work, sizeof(double2) * 4 * nrc * ne) == cudaSuccess &&
            cudaMalloc(&a->error, sizeof(double) * nrc * ne) == cudaSuccess &&
            cudaMalloc(&a->rcut, sizeof(double) * ne) == cudaSuccess &&
            cudaMalloc(&a->rcidx, sizeof(int) * ne) == cudaSuccess &&
            cudaMalloc(&a->rcidx2, sizeof(int) * ne) == cudaSuccess &&
            cudaMalloc(&a->rerr, sizeof(double) * ne) == cudaSuccess &&
            cudaMalloc(&a->pcorr, sizeof(double) * 3) == cudaSuccess;
  if (!ok) {
    md_cuda_fail(cudaGetLastError(), "md_arc_create");
    md_arc_destroy(a);
    return MD_ERR_CUDA;
  }
  cudaMemcpyAsync(a->d_rc, a->rc.data(), sizeof(double) * nrc, cudaMemcpyHostToDevice, a->sys->stream);
  cudaMemsetAsync(a->counts, 0, sizeof(double) * ne, a->sys->stream);
  cudaMemsetAsync(a->rho, 0, sizeof(double) * ne, a->sys->stream);
  cudaMemsetAsync(a->pcorr, 0, sizeof(double) * 3, a->sys->stream);  // pxx = pyy = pzz = 0 (:82)
  if (int r = build_tables(a)) { md_arc_destroy(a); return r; }
  *out = a;
  return MD_OK;
}

extern "C" int md_arc_destroy(md_adapt_rcut* a) {
  if (!a) return MD_OK;
  void* p[] = {a->d_rc, a->counts, a->rho, a->rhok, a->s1k, a->s2k, a->pck, a->ints, a->work,
               a->error, a->rcut, a->rcidx, a->rcidx2, a->rerr, a->pcorr};
  for (void* q : p) if (q) cudaFree(q);
  delete a;
  return MD_OK;
}

extern "C" int md_arc_get_dims(md_adapt_rcut* a, int n[3], int* nrc) {
  if (!a) return MD_ERR_BADARG;
  if (n) for (int d = 0; d < 3; ++d) n[d] = a->n[d];
  if (nrc) *nrc = a->nrc;
  return MD_OK;
}

extern "C" int md_arc_deposit(md_adapt_rcut* a, md_system* sys) {
  if (!a || !sys) return MD_ERR_BADARG;
  ArcDims g;
  for (int d = 0; d < 3; ++d) { g.n[d] = a->n[d]; g.box[d] = a->box_tab[d]; }
  g.nrc = a->nrc;
  int nb = ceil_div(sys->N, 256);
  if (sys->prec == MD_PREC_FP64)
    k_arc_deposit<double><<<nb, 256, 0, a->sys->stream>>>(sys->N, (double4a*)sys->pos, g, a->counts);
  else
    k_arc_deposit<float><<<nb, 256, 0, a->sys->stream>>>(sys->N, (float4*)sys->pos, g, a->counts);
  MD_CHECK_LAUNCH("arc deposit");
  a->ndata++;
  return MD_OK;
}

extern "C" int md_arc_clear_profile(md_adapt_rcut* a) {
  if (!a) return MD_ERR_BADARG;
  MD_CUDA(cudaMemsetAsync(a->counts, 0, sizeof(double) * a->nele, a->sys->stream));
  a->ndata = 0;
  return MD_OK;
}

extern "C" int md_arc_set_profile(md_adapt_rcut* a, const double* rho) {
  if (!a || !rho) return MD_ERR_BADARG;
  MD_CUDA(cudaMemcpyAsync(a->rho, rho, sizeof(double) * a->nele, cudaMemcpyHostToDevice, a->sys->stream));
  MD_CUDA(cudaStreamSynchronize(a->sys->stream));
  a->ndata = -1;  // explicit profile: do not renormalise counts
  return MD_OK;
}

extern "C" int md_arc_get_profile(md_adapt_rcut* a, double* rho) {
  if (!a || !rho) return MD_ERR_BADARG;
  MD_CUDA(cudaMemcpyAsync(rho, a->rho, sizeof(double) * a->nele, cudaMemcpyDeviceToHost, a->sys->stream));
  MD_CUDA(cudaStreamSynchronize(a->sys->stream));
  return MD_OK;
}

// DensityProfile::calculate (counts / (dv * ndata), or the explicit profile)
// and the forward transform of the profile into rhok; bin volume and the
// kernel tables are those of the construction box.
static int arc_profile_transform(md_adapt_rcut* a, const char* who) {
  const long ne = a->nele;
  const int nb = (int)((ne + 255) / 256);
  const double* B = a->box_tab;
  if (a->ndata > 0) {
    double dv = (B[0] / a->n[0]) * (B[1] / a->n[1]) * (B[2] / a->n[2]);
    k_arc_profile<<<nb, 256, 0, a->sys->stream>>>(ne, a->counts, 1.0 / (dv * a->ndata), a->rho, a->rhok);
  } else if (a->ndata < 0) {
    k_arc_profile<<<nb, 256, 0, a->sys->stream>>>(ne, nullptr, 0.0, a->rho, a->rhok);
  } else {
    md_set_error("%s: no density samples deposited", who);
    return MD_ERR_BADARG;
  }
  MD_CHECK_LAUNCH("arc profile");
  return dft3(a, a->rhok, -1, 1);
}

extern "C" int md_arc_update(md_adapt_rcut* a, double prec, int nrefine) {
  if (!a || !(prec > 0) || nrefine < 0) { md_set_error("md_arc_update: bad arguments"); return MD_ERR_BADARG; }
  md_system* sys = a->sys;
  if (int r = arc_profile_transform(a, "md_arc_update")) return r;
  const long ne = a->nele;
  const int nb = (int)((ne + 255) / 256);
  const double* B = a->box_tab;
  const double V = B[0] * B[1] * B[2];
  k_arc_multiply<<<nb, 256, 0, a->sys->stream>>>(ne, a->nrc, a->rhok, V / ne, a->s1k, a->s2k, a->work);
  MD_CHECK_LAUNCH("arc multiply");
  if (int r = dft3(a, a->work, +1, 2 * a->nrc)) return r;
  k_arc_error<<<nb, 256, 0, a->sys->stream>>>(ne, a->nrc, a->work, 1.0 / V, a->error);
  k_arc_rcut<<<nb, 256, 0, a->sys->stream>>>(ne, a->nrc, a->d_rc, a->error, prec, a->rcut, a->rcidx, a->rerr);
  MD_CHECK_LAUNCH("arc rcut");
  ArcDims g;
  for (int d = 0; d < 3; ++d) g.n[d] = a->n[d];
  for (int it = 0; it < nrefine; ++it) {
    k_arc_refine<<<nb, 256, 0, a->sys->stream>>>(g, a->rcidx, a->rcidx2, a->d_rc, a->error, a->rcut, a->rerr);
    MD_CHECK_LAUNCH("arc refine");
    std::swap(a->rcidx, a->rcidx2);
  }
  // PressureCorrection::correction on the same profile and rc map
  k_pc_multiply<<<nb, 256, 0, a->sys->stream>>>(ne, a->nrc, a->rhok, V / ne, a->pck, a->work);
  MD_CHECK_LAUNCH("pc multiply");
  if (int r = dft3(a, a->work, +1, 2 * a->nrc)) return r;
  const double dv = (B[0] / a->n[0]) * (B[1] / a->n[1]) * (B[2] / a->n[2]);
  if (nb > sys->max_partial_blocks) { md_set_error("partials buffer too small"); return MD_ERR_BADARG; }
  k_pc_carry<<<1, 32, 0, a->sys->stream>>>(a->pcorr, 1.0 / V);
  MD_CHECK_LAUNCH("pc carry");
  k_pc_reduce<<<nb, 256, 0, a->sys->stream>>>(ne, a->nrc, a->work, a->rcidx, a->rho, dv / (V * V), sys->partials,
                                         &sys->st->red_counter[RED_MISC], a->pcorr);
  MD_CHECK_LAUNCH("pc reduce");
  return MD_OK;
}

extern "C" int md_arc_get_error(md_adapt_rcut* a, double* err) {
  if (!a || !err) return MD_ERR_BADARG;
  MD_CUDA(cudaMemcpyAsync(err, a->error, sizeof(double) * a->nrc * a->nele, cudaMemcpyDeviceToHost, a->sys->stream));
  MD_CUDA(cudaStreamSynchronize(a->sys->stream));
  return MD_OK;
}

extern "C" int md_arc_get_rcut(md_adapt_rcut* a, double* rcut, int* idx, double* result_error) {
  if (!a) return MD_ERR_BADARG;
  if (rcut) MD_CUDA(cudaMemcpyAsync(rcut, a->rcut, sizeof(double) * a->nele, cudaMemcpyDeviceToHost, a->sys->stream));
  if (idx) MD_CUDA(cudaMemcpyAsync(idx, a->rcidx, sizeof(int) * a->nele, cudaMemcpyDeviceToHost, a->sys->stream));
  if (result_error) MD_CUDA(cudaMemcpyAsync(result_error, a->rerr, sizeof(double) * a->nele, cudaMemcpyDeviceToHost, a->sys->stream));
  MD_CUDA(cudaStreamSynchronize(a->sys->stream));
  DevState hs;
  if (int r = a->sys->read_state(hs)) return r;
  if (hs.flags & FLAG_QUADRATURE) { md_set_error("adaptive quadrature reached its depth bound"); return MD_ERR_BADARG; }
  return MD_OK;
}

extern "C" int md_arc_get_tables(md_adapt_rcut* a, double* s1k, double* s2k, double* pck) {
  if (!a) return MD_ERR_BADARG;
  const size_t m = (size_t)a->nrc * a->nele;
  if (s1k) MD_CUDA(cudaMemcpyAsync(s1k, a->s1k, sizeof(double) * m, cudaMemcpyDeviceToHost, a->sys->stream));
  if (s2k) MD_CUDA(cudaMemcpyAsync(s2k, a->s2k, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, a->sys->stream));
  if (pck) MD_CUDA(cudaMemcpyAsync(pck, a->pck, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, a->sys->stream));
  MD_CUDA(cudaStreamSynchronize(a->sys->stream));
  return MD_OK;
}

// AssignRCut::getRCut + assign: the device lattice the cell sort reads, and a
// forced list rebuild at the next step.  Lattice storage is reused when the
// size matches so a captured step keeps a valid pointer.
extern "C" int md_arc_assign(md_adapt_rcut* a, md_system* sys) {
  if (!a || !sys) return MD_ERR_BADARG;
  const long ne = a->nele;
  if (!sys->d_lattice || (long)sys->lat_n[0] * sys->lat_n[1] * sys->lat_n[2] != ne) {
    if (sys->d_lattice) cudaFree(sys->d_lattice);
    sys->d_lattice = nullptr;
    MD_CUDA(cudaMalloc(&sys->d_lattice, sizeof(float) * ne));
  }
  for (int d = 0; d < 3; ++d) sys->lat_n[d] = a->n[d];
  k_lattice_from_rcut<<<(int)((ne + 255) / 256), 256, 0, a->sys->stream>>>(ne, a->rcut, sys->d_lattice, sys->st);
  MD_CHECK_LAUNCH("lattice");
  return MD_OK;
}

extern "C" int md_arc_pressure_correction(md_adapt_rcut* a, md_system* sys, double out[3]) {
  if (!a || !sys) return MD_ERR_BADARG;
  k_store_pcorr<<<1, 1, 0, a->sys->stream>>>(a->pcorr, sys->st);
  MD_CHECK_LAUNCH("store pcorr");
  if (out) {
    MD_CUDA(cudaMemcpyAsync(out, a->pcorr, sizeof(double) * 3, cudaMemcpyDeviceToHost, a->sys->stream));
    MD_CUDA(cudaStreamSynchronize(a->sys->stream));
  }
  return MD_OK;
}

// ------------------------------------------------------------ LFC
// Long-range force correction (FCR = shortRange.inhomo/template/tools/
// simulation.fcorr):
//   ForceCorr::makeS2k        FCR/src/ForceCorr.cu:193-262: the AdaptRCut
//                             kernel i k_d T(k) of the single cutoff rc (the
//                             x^-5 quadrature over [rc, 30] and the boundary
//                             term), so the tables of an md_adapt_rcut with
//                             rcmin = rcmax = rc are reused
//   ForceCorr::calError       FCR/src/ForceCorr.cu:150-179:
//                             field_d = IFFT(s2k_d FFT(rho) V / nele) / V
//   AssignForceCorr::getForceCorr / zero / assign
//                             FCR/src/AssignForceCorr.cu:55-178: the per-bin
//                             field (working precision) and, at assign, each
//                             atom's value at its bin (binary32 binning)
//   InteractionEngine (LFC)   FCR/src/InteractionEngine_interface.cu:1118:
//                             the force kernel adds the atom's value
// The per-atom values are stored by original atom id, so the cell sort
// never has to carry them.
struct md_fcorr {
  md_adapt_rcut* arc = nullptr;  // bins, density samples and the kernel table
  double* field = nullptr;       // [3][nele] real parts, [3][nele] imaginary parts
  double4a* corr = nullptr;      // per-atom value by atom id
  int N = 0;
};

__global__ void k_fc_multiply(long nele, const double2* rhok, double scale, const double* s2k, double2* work) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  const double2 r = make_double2(rhok[i].x * scale, rhok[i].y * scale);
  for (int d = 0; d < 3; ++d) {
    const double b = s2k[(long)d * nele + i];  // one cutoff: s2k[d][0][i]
    work[(long)d * nele + i] = make_double2(-r.y * b, r.x * b);
  }
}

__global__ void k_fc_extract(long nele, const double2* work, double Vi, double* field) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= nele) return;
  for (int d = 0; d < 3; ++d) {
    const double2 w = work[(long)d * nele + i];
    field[(long)d * nele + i] = w.x * Vi;
    field[(long)(3 + d) * nele + i] = w.y * Vi;
  }
}

// AssignForceCorr::assign: bin of the (wrapped) binary32 coordinate,
// ix = int((x nx) / Lx); the value in the working precision R
template <class R>
__global__ void k_fc_assign(int N, const typename V4<R>::T* __restrict__ pos, const int* __restrict__ id,
                            const DevState* st, int nx, int ny, int nz, const double* __restrict__ field,
                            long nele, double4a* __restrict__ corr) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const typename V4<R>::T p = pos[k];
  float x = (float)p.x, y = (float)p.y, z = (float)p.z;
  const float Lx = st->Lf[0], Ly = st->Lf[1], Lz = st->Lf[2];
  if (x < 0) x = __fadd_rn(x, Lx); else if (x >= Lx) x = __fsub_rn(x, Lx);
  if (y < 0) y = __fadd_rn(y, Ly); else if (y >= Ly) y = __fsub_rn(y, Ly);
  if (z < 0) z = __fadd_rn(z, Lz); else if (z >= Lz) z = __fsub_rn(z, Lz);
  int ix = __float2int_rz(__fdiv_rn(__fmul_rn(x, (float)nx), Lx));
  int iy = __float2int_rz(__fdiv_rn(__fmul_rn(y, (float)ny), Ly));
  int iz = __float2int_rz(__fdiv_rn(__fmul_rn(z, (float)nz), Lz));
  ix = min(max(ix, 0), nx - 1); iy = min(max(iy, 0), ny - 1); iz = min(max(iz, 0), nz - 1);
  const long b = iz + (long)nz * (iy + (long)ny * ix);
  corr[id[k]] = double4a{(double)(R)field[b], (double)(R)field[nele + b], (double)(R)field[2 * nele + b], 0.0};
}

const double4a* fcorr_values(const md_fcorr* f) { return f ? f->corr : nullptr; }

extern "C" int md_fcorr_create(md_fcorr** out, md_system* sys, double rc, double refh) {
  if (!out || !sys || !(rc > 0) || !(rc < 30.0) || !(refh > 0)) {
    md_set_error("md_fcorr_create: bad arguments (0 < rc < 30, refh > 0)");
    return MD_ERR_BADARG;
  }
  md_fcorr* f = new md_fcorr();
  f->N = sys->N;
  if (int r = md_arc_create(&f->arc, sys, refh, rc, rc, 1.0)) { delete f; return r; }
  const long ne = f->arc->nele;
  bool ok = cudaMalloc(&f->field, sizeof(double) * 6 * ne) == cudaSuccess &&
            cudaMalloc(&f->corr, sizeof(double4a) * sys->N) == cudaSuccess &&
            cudaMemsetAsync(f->field, 0, sizeof(double) * 6 * ne, sys->stream) == cudaSuccess &&
            cudaMemsetAsync(f->corr, 0, sizeof(double4a) * sys->N, sys->stream) == cudaSuccess;
  if (!ok) {
    md_cuda_fail(cudaGetLastError(), "md_fcorr_create");
    md_fcorr_destroy(f);
    return MD_ERR_CUDA;
  }
  *out = f;
  return MD_OK;
}

extern "C" int md_fcorr_destroy(md_fcorr* f) {
  if (!f) return MD_OK;
  md_arc_destroy(f->arc);
  if (f->field) cudaFree(f->field);
  if (f->corr) cudaFree(f->corr);
  delete f;
  return MD_OK;
}

extern "C" int md_fcorr_get_dims(md_fcorr* f, int n[3]) {
  if (!f || !n) return MD_ERR_BADARG;
  return md_arc_get_dims(f->arc, n, nullptr);
}

extern "C" int md_fcorr_deposit(md_fcorr* f, md_system* sys) {
  if (!f || !sys || sys->N != f->N) return MD_ERR_BADARG;
  return md_arc_deposit(f->arc, sys);
}

extern "C" int md_fcorr_clear_profile(md_fcorr* f) {
  if (!f) return MD_ERR_BADARG;
  return md_arc_clear_profile(f->arc);
}

extern "C" int md_fcorr_set_profile(md_fcorr* f, const double* rho) {
  if (!f || !rho) return MD_ERR_BADARG;
  return md_arc_set_profile(f->arc, rho);
}

extern "C" int md_fcorr_get_profile(md_fcorr* f, double* rho) {
  if (!f || !rho) return MD_ERR_BADARG;
  return md_arc_get_profile(f->arc, rho);
}

extern "C" int md_fcorr_update(md_fcorr* f) {
  if (!f) return MD_ERR_BADARG;
  md_adapt_rcut* a = f->arc;
  if (int r = arc_profile_transform(a, "md_fcorr_update")) return r;
  const long ne = a->nele;
  const int nb = (int)((ne + 255) / 256);
  const double V = a->box_tab[0] * a->box_tab[1] * a->box_tab[2];
  k_fc_multiply<<<nb, 256, 0, a->sys->stream>>>(ne, a->rhok, V / ne, a->s2k, a->work);
  MD_CHECK_LAUNCH("fcorr multiply");
  if (int r = dft3(a, a->work, +1, 3)) return r;
  k_fc_extract<<<nb, 256, 0, a->sys->stream>>>(ne, a->work, 1.0 / V, f->field);
  MD_CHECK_LAUNCH("fcorr extract");
  return MD_OK;
}

extern "C" int md_fcorr_zero(md_fcorr* f) {
  if (!f) return MD_ERR_BADARG;
  MD_CUDA(cudaMemsetAsync(f->field, 0, sizeof(double) * 6 * f->arc->nele, f->arc->sys->stream));
  return MD_OK;
}

extern "C" int md_fcorr_get_field(md_fcorr* f, double* re, double* im) {
  if (!f) return MD_ERR_BADARG;
  const long ne = f->arc->nele;
  cudaStream_t s = f->arc->sys->stream;
  if (re) MD_CUDA(cudaMemcpyAsync(re, f->field, sizeof(double) * 3 * ne, cudaMemcpyDeviceToHost, s));
  if (im) MD_CUDA(cudaMemcpyAsync(im, f->field + 3 * ne, sizeof(double) * 3 * ne, cudaMemcpyDeviceToHost, s));
  MD_CUDA(cudaStreamSynchronize(s));
  DevState hs;
  if (int r = f->arc->sys->read_state(hs)) return r;
  if (hs.flags & FLAG_QUADRATURE) { md_set_error("adaptive quadrature reached its depth bound"); return MD_ERR_BADARG; }
  return MD_OK;
}

extern "C" int md_fcorr_assign(md_fcorr* f, md_system* sys) {
  if (!f || !sys || sys->N != f->N) { md_set_error("md_fcorr_assign: bad arguments"); return MD_ERR_BADARG; }
  md_adapt_rcut* a = f->arc;
  const int nb = ceil_div(sys->N, 256);
  if (sys->prec == MD_PREC_FP64)
    k_fc_assign<double><<<nb, 256, 0, sys->stream>>>(sys->N, (const double4a*)sys->pos, sys->id, sys->st, a->n[0],
                                                       a->n[1], a->n[2], f->field, a->nele, f->corr);
  else
    k_fc_assign<float><<<nb, 256, 0, sys->stream>>>(sys->N, (const float4*)sys->pos, sys->id, sys->st, a->n[0],
                                                      a->n[1], a->n[2], f->field, a->nele, f->corr);
  MD_CHECK_LAUNCH("fcorr assign");
  return MD_OK;
}

extern "C" int md_fcorr_get_values(md_fcorr* f, double* v) {
  if (!f || !v) return MD_ERR_BADARG;
  std::vector<double4a> h(f->N);
  cudaStream_t s = f->arc->sys->stream;
  MD_CUDA(cudaMemcpyAsync(h.data(), f->corr, sizeof(double4a) * f->N, cudaMemcpyDeviceToHost, s));
  MD_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < f->N; ++i) { v[3 * i] = h[i].x; v[3 * i + 1] = h[i].y; v[3 * i + 2] = h[i].z; }
  return MD_OK;
}
