// Smooth particle-mesh Ewald (reciprocal part) and the exact Ewald sum.
// Reference (RE = longRange.hetero/profile.test/template/tools/real.error):
//   calQ spread                      RE/src/EleRecBSpline.cpp:541-619
//   calB / calPsiFPhiF (ik)          RE/src/EleRecBSpline.cpp:729-877
//   applyInteractionCalPotential ik  RE/src/EleRecBSpline.cpp:393-536
//   analytic differentiation         RE/src/EleRecFBSpline.cpp:771-907, 1146-1195
//   exact reciprocal sum (ES)        RE/src/EleRecES.cpp:49-144
//
// Chain per call: spread (one thread per atom x (k0,k1) column, atomic adds
// along k2) -> R2C along z -> C2C along y, x (forward) -> k-space pass (energy
// and virial in FP64, influence multiply; ik writes the three products
// i(-2 pi m_d) psi Q^, analytic writes psi Q^) -> C2C x, y (inverse) -> C2R
// along z with the Hermitian completion of an r2c half spectrum (the FFTW c2r
// convention the reference relies on) -> gather (one warp per atom).
// The FFT is a radix-2 Stockham transform of whole lines in shared memory;
// a block holds several lines that are adjacent in memory so that strided
// axes load coalesced.  Mixed precision: mesh, FFT and gather in FP32,
// energy/virial and force accumulation in FP64.  Power-of-two mesh sizes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "device_common.cuh"

template <class R> struct C2;
template <> struct C2<float> { typedef float2 T; };
template <> struct C2<double> { typedef double2 T; };

struct md_spme {
  md_system* sys = nullptr;
  int K[3] = {0, 0, 0};
  int K2h = 0;
  int order = 6;
  int method = 0;  // 0 ik, 1 analytic
  double beta = 1.0;
  size_t nreal = 0, nhalf = 0;
  void* Q = nullptr;      // real mesh
  void* C = nullptr;      // complex half meshes: [0] Q^, [1..3] products
  void* G = nullptr;      // real convolution meshes (3 for ik, 1 analytic)
  void* psi = nullptr;    // influence function on the half spectrum (ik normalisation)
  double* d_box_tab = nullptr;  // box psi was computed for (device; 0 = never)
};

// ---------------------------------------------------------------- B-spline weights
// M_n(f + j), j = 0..n-1 (and derivatives) by the recursion
// M_k(u) = (u M_{k-1}(u) + (k - u) M_{k-1}(u - 1)) / (k - 1)  (Essmann et al. 1995)
template <class R>
__device__ __forceinline__ void bspline_w(int n, R f, R* w, R* dw) {
  w[0] = f;
  w[1] = R(1) - f;
  for (int j = 2; j < n; ++j) w[j] = R(0);
  for (int k = 3; k <= n; ++k) {
    if (k == n && dw) {
      for (int j = 0; j < n; ++j) dw[j] = (j < n - 1 ? w[j] : R(0)) - (j > 0 ? w[j - 1] : R(0));
    }
    const R inv = R(1) / R(k - 1);
    for (int j = k - 1; j >= 0; --j) {
      const R u = f + R(j);
      const R a = (j < k - 1) ? w[j] : R(0);
      const R b = (j > 0) ? w[j - 1] : R(0);
      w[j] = (u * a + (R(k) - u) * b) * inv;
    }
  }
  if (n == 2 && dw) { dw[0] = R(1); dw[1] = R(-1); }
}

template <class R>
__device__ __forceinline__ void grid_coord(R x, R Linv, int K, int& base, R& frac) {
  R u = R(K) * x * Linv;
  u -= floor_r(u / R(K)) * R(K);
  R b = floor_r(u);
  frac = u - b;
  base = (int)b;
  if (base >= K) { base -= K; }
}

__device__ __forceinline__ int wrapk(int k, int K) { return k < 0 ? k + K : k; }

// ---------------------------------------------------------------- spread
template <class R>
__global__ void k_spme_spread(int N, const typename V4<R>::T* __restrict__ pos, int n, int K0, int K1, int K2,
                              const DevState* __restrict__ st, R* __restrict__ Q) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int nn = n * n;
  const long i = t / nn;
  if (i >= N) return;
  const int ab = (int)(t - i * nn), a = ab / n, b = ab % n;
  const typename V4<R>::T p = pos[i];
  if (p.w == R(0)) return;
  int b0, b1, b2;
  R f0, f1, f2;
  grid_coord<R>(p.x, (R)st->Li[0], K0, b0, f0);
  grid_coord<R>(p.y, (R)st->Li[1], K1, b1, f1);
  grid_coord<R>(p.z, (R)st->Li[2], K2, b2, f2);
  R w0[16], w1[16], w2[16];
  bspline_w<R>(n, f0, w0, nullptr);
  bspline_w<R>(n, f1, w1, nullptr);
  bspline_w<R>(n, f2, w2, nullptr);
  const R qab = p.w * w0[a] * w1[b];
  const long row = ((long)wrapk(b0 - a, K0) * K1 + wrapk(b1 - b, K1)) * K2;
  for (int c = 0; c < n; ++c) atomicAdd(&Q[row + wrapk(b2 - c, K2)], qab * w2[c]);
}

// ---------------------------------------------------------------- FFT
// Stockham radix-2 of one length-n line held in shared memory (two buffers);
// the `lpb` lines of the block are processed together, n/2 threads per line.
template <class T2>
__device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

template <class R>
__device__ void line_fft(typename C2<R>::T* x, typename C2<R>::T* y, const typename C2<R>::T* tw, int n,
                         int lpb, typename C2<R>::T** out) {
  typedef typename C2<R>::T T2;
  const int half = n >> 1;
  const int l = threadIdx.x / half, p = threadIdx.x % half;
  for (int m = 1; m < n; m <<= 1) {
    if (l < lpb) {
      const int k = p % m, j = p / m;
      const T2 w = tw[k * (half / m)];
      const T2 c0 = x[l * n + p], c1 = cmul(w, x[l * n + p + half]);
      T2 s, d;
      s.x = c0.x + c1.x; s.y = c0.y + c1.y;
      d.x = c0.x - c1.x; d.y = c0.y - c1.y;
      y[l * n + j * 2 * m + k] = s;
      y[l * n + j * 2 * m + k + m] = d;
    }
    __syncthreads();
    T2* t = x; x = y; y = t;
  }
  *out = x;
}

template <class R>
__device__ void load_twiddles(typename C2<R>::T* tw, int n, int sign) {
  for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
    double s, c;
    sincospi(2.0 * t / n, &s, &c);
    tw[t].x = (R)c;
    tw[t].y = (R)(sign * s);
  }
}

// mode 0: real input lines (z, contiguous) -> half-complex output
// mode 1: complex lines along axis x or y of the half-complex array
// mode 2: half-complex z lines -> real output (Hermitian completion)
template <class R>
__global__ void k_fft(const void* in, void* out, int mode, int n, int lpb, long nlines, long stride,
                      long lines_inner, long outer_stride, long in_astride, long out_astride, int sign) {
  typedef typename C2<R>::T T2;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  T2* tw = reinterpret_cast<T2*>(fft_smem);
  T2* x = tw + n / 2;
  T2* y = x + lpb * n;
  load_twiddles<R>(tw, n, sign);
  const long line0 = (long)blockIdx.x * lpb;
  const int batch = blockIdx.y;
  const int nh = n / 2 + 1;
  // load
  for (int e = threadIdx.x; e < lpb * n; e += blockDim.x) {
    int l, k;
    if (mode == 1) { l = e % lpb; k = e / lpb; }  // lines adjacent in memory: coalesce across l
    else { l = e / n; k = e % n; }
    const long L = line0 + l;
    T2 v;
    v.x = R(0); v.y = R(0);
    if (L < nlines) {
      if (mode == 0) {
        const R* src = reinterpret_cast<const R*>(in) + batch * in_astride + L * n;
        v.x = src[k];
      } else if (mode == 1) {
        const T2* src = reinterpret_cast<const T2*>(in) + batch * in_astride;
        const long o = (L / lines_inner) * outer_stride + (L % lines_inner);
        v = src[o + k * stride];
      } else {
        const T2* src = reinterpret_cast<const T2*>(in) + batch * in_astride + L * nh;
        if (k < nh) v = src[k];
        else { const T2 u = src[n - k]; v.x = u.x; v.y = -u.y; }
      }
    }
    x[l * n + k] = v;
  }
  __syncthreads();
  T2* res;
  line_fft<R>(x, y, tw, n, lpb, &res);
  // store
  for (int e = threadIdx.x; e < lpb * n; e += blockDim.x) {
    int l, k;
    if (mode == 1) { l = e % lpb; k = e / lpb; }
    else { l = e / n; k = e % n; }
    const long L = line0 + l;
    if (L >= nlines) continue;
    const T2 v = res[l * n + k];
    if (mode == 0) {
      if (k < nh) reinterpret_cast<T2*>(out)[batch * out_astride + L * nh + k] = v;
    } else if (mode == 1) {
      const long o = (L / lines_inner) * outer_stride + (L % lines_inner);
      reinterpret_cast<T2*>(out)[batch * out_astride + o + k * stride] = v;
    } else {
      reinterpret_cast<R*>(out)[batch * out_astride + L * n + k] = v.x;
    }
  }
}

// ---------------------------------------------------------------- influence
__device__ __forceinline__ double bmod_d(int n, int K, int m) {
  // |b(m)|^2 = 1 / |sum_{k=0}^{n-2} M_n(k+1) exp(2 pi i m k / K)|^2 (calB)
  double w[16];
  bspline_w<double>(n, 0.0, w, nullptr);  // w[j] = M_n(j)
  double re = 0, im = 0;
  for (int k = 0; k < n - 1; ++k) {
    double s, c;
    sincospi(2.0 * (double)((long)m * k % K) / K, &s, &c);
    re += w[k + 1] * c;
    im += w[k + 1] * s;
  }
  return 1.0 / (re * re + im * im);
}

// psi is recomputed only when the box differs from `tab`, the box it was last
// computed for (NPT); the comparison is made on the device so that no host
// round trip is needed, and `tab` is updated by k_spme_box_tab afterwards
template <class R>
__global__ void k_spme_influence(int K0, int K1, int K2, int n, double beta, const DevState* st, R* psi,
                                 const double* tab) {
  const int K2h = K2 / 2 + 1;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)K0 * K1 * K2h) return;
  if (st->L[0] == tab[0] && st->L[1] == tab[1] && st->L[2] == tab[2]) return;
  const int k = (int)(t % K2h), j = (int)((t / K2h) % K1), i = (int)(t / ((long)K2h * K1));
  const int ip = i <= K0 / 2 ? i : i - K0, jp = j <= K1 / 2 ? j : j - K1, kp = k;
  if (!ip && !jp && !kp) { psi[t] = R(0); return; }
  const double V = st->L[0] * st->L[1] * st->L[2];
  const double m0 = ip * st->Li[0], m1 = jp * st->Li[1], m2 = kp * st->Li[2];
  const double mm = m0 * m0 + m1 * m1 + m2 * m2;
  const double B = bmod_d(n, K0, i) * bmod_d(n, K1, j) * bmod_d(n, K2, k);
  const double sc = M_PI * M_PI / beta / beta;
  psi[t] = (R)(exp(-sc * mm) / mm * B / (M_PI * V));
}

__global__ void k_spme_box_tab(const DevState* st, double* tab) {
  for (int d = 0; d < 3; ++d) tab[d] = st->L[d];
}

// energy + diagonal virial and the products written into C[1..]
template <class R>
__global__ void __launch_bounds__(256)
k_spme_kspace(int K0, int K1, int K2, int method, double beta, const R* __restrict__ psi,
              typename C2<R>::T* __restrict__ C, size_t nhalf, DevState* st, double* partials, int with_stats) {
  typedef typename C2<R>::T T2;
  const int K2h = K2 / 2 + 1;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (t < (long)nhalf) {
    const int k = (int)(t % K2h), j = (int)((t / K2h) % K1), i = (int)(t / ((long)K2h * K1));
    const int ip = i <= K0 / 2 ? i : i - K0, jp = j <= K1 / 2 ? j : j - K1, kp = k;
    const T2 q = C[t];
    const R ps = psi[t];
    const double m[3] = {ip * st->Li[0], jp * st->Li[1], kp * st->Li[2]};
    if (method == 0) {
      for (int d = 0; d < 3; ++d) {
        const R c = (R)(-2.0 * M_PI * m[d]) * ps;  // phi_d = i (-2 pi m_d) psi
        T2 g;
        g.x = -q.y * c;
        g.y = q.x * c;
        C[(1 + d) * nhalf + t] = g;
      }
    } else {
      T2 g;
      g.x = q.x * (R(0.5) * ps);  // analytic: psi / 2 (FBSpline normalisation)
      g.y = q.y * (R(0.5) * ps);
      C[nhalf + t] = g;
    }
    if (with_stats && (ip || jp || kp)) {
      // E = 1/2 sum_m |Q^|^2 psi over the full spectrum: interior z planes count twice
      const double wgt = (k == 0 || (2 * k == K2)) ? 1.0 : 2.0;
      const double e = 0.5 * wgt * ((double)q.x * q.x + (double)q.y * q.y) * (double)ps;
      const double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
      const double f = 2.0 * (1.0 + M_PI * M_PI * mm / (beta * beta)) / mm;
      v[0] = e;
      // pressure tensor V P_aa = sum_m E_m (1 - f m_a^2); the virial slots hold W_aa = -V P_aa
      for (int d = 0; d < 3; ++d) v[1 + d] = -e * (1.0 - f * m[d] * m[d]);
    }
  }
  if (with_stats) block_reduce_finish<4>(v, partials, &st->red_counter[RED_SPME], st->scratch, true);
}

__global__ void k_spme_stats_merge(DevState* st) {
  // reciprocal energy into its slot, its diagonal virial added to the virial slots
  st->stats[MD_STAT_ELEC_REC] = st->scratch[0];
  for (int d = 0; d < 3; ++d) st->stats[MD_STAT_VIRIAL_XX + d] += st->scratch[1 + d];
}

// ---------------------------------------------------------------- gather
template <class R>
__global__ void __launch_bounds__(256)
k_spme_gather(int N, const typename V4<R>::T* __restrict__ pos, int n, int K0, int K1, int K2, int method,
              const DevState* __restrict__ st, const R* __restrict__ G, size_t nreal, double4a* __restrict__ force) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= N) return;
  const typename V4<R>::T p = pos[warp];
  int b0, b1, b2;
  R f0, f1, f2;
  grid_coord<R>(p.x, (R)st->Li[0], K0, b0, f0);
  grid_coord<R>(p.y, (R)st->Li[1], K1, b1, f1);
  grid_coord<R>(p.z, (R)st->Li[2], K2, b2, f2);
  R w0[16], w1[16], w2[16], d0[16], d1[16], d2[16];
  bspline_w<R>(n, f0, w0, d0);
  bspline_w<R>(n, f1, w1, d1);
  bspline_w<R>(n, f2, w2, d2);
  R fx = 0, fy = 0, fz = 0;
  for (int ab = lane; ab < n * n; ab += 32) {
    const int a = ab / n, b = ab % n;
    const long row = ((long)wrapk(b0 - a, K0) * K1 + wrapk(b1 - b, K1)) * K2;
    for (int c = 0; c < n; ++c) {
      const long idx = row + wrapk(b2 - c, K2);
      if (method == 0) {
        const R w = w0[a] * w1[b] * w2[c];
        fx += G[idx] * w;
        fy += G[nreal + idx] * w;
        fz += G[2 * nreal + idx] * w;
      } else {
        const R g = G[idx];
        fx -= g * d0[a] * w1[b] * w2[c];
        fy -= g * w0[a] * d1[b] * w2[c];
        fz -= g * w0[a] * w1[b] * d2[c];
      }
    }
  }
  double Fx = fx, Fy = fy, Fz = fz;
  for (int o = 16; o > 0; o >>= 1) {
    Fx += __shfl_xor_sync(0xffffffffu, Fx, o);
    Fy += __shfl_xor_sync(0xffffffffu, Fy, o);
    Fz += __shfl_xor_sync(0xffffffffu, Fz, o);
  }
  if (lane == 0) {
    const double q = (double)p.w;
    double4a f = force[warp];
    if (method == 0) {
      f.x += q * Fx; f.y += q * Fy; f.z += q * Fz;
    } else {
      f.x += 2.0 * q * Fx * K0 * st->Li[0];
      f.y += 2.0 * q * Fy * K1 * st->Li[1];
      f.z += 2.0 * q * Fz * K2 * st->Li[2];
    }
    force[warp] = f;
  }
}

// ---------------------------------------------------------------- adjoint
// The reciprocal energy is the quadratic form E = 1/2 sum_m psi(m) |Q^(m)|^2
// = 1/2 sum_k Q(k) Phi(k) with Phi = IFFT(psi Q^) (unnormalised transforms),
// Q(k) = sum_i q_i theta_i(k), theta_i(k) = prod_d M_n(u_id - k_d), u = K x / L.
// Hence
//   dE/dq_i      = sum_k theta_i(k) Phi(k)                      (potential)
//   dE/dx_id     = q_i sum_k d theta_i(k)/du_d Phi(k) K_d / L_d  (exact gradient,
//                  the analytic-differentiation force with its sign flipped)
//   dE/dpsi(m)   = 1/2 |Q^(m)|^2
//   dE/dbeta     = sum_m 1/2 |Q^(m)|^2 psi(m) 2 pi^2 |m|^2 / beta^3
// The adjoint recomputes the spread mesh and its transform instead of
// keeping them from an earlier forward call.
template <class R>
__global__ void __launch_bounds__(256)
k_spme_adj_kspace(int K0, int K1, int K2, double beta, const R* __restrict__ psi, typename C2<R>::T* __restrict__ C,
                  size_t nhalf, DevState* st, double* partials, double* __restrict__ dpsi) {
  typedef typename C2<R>::T T2;
  const int K2h = K2 / 2 + 1;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double v[2] = {0, 0};
  if (t < (long)nhalf) {
    const int k = (int)(t % K2h), j = (int)((t / K2h) % K1), i = (int)(t / ((long)K2h * K1));
    const int ip = i <= K0 / 2 ? i : i - K0, jp = j <= K1 / 2 ? j : j - K1, kp = k;
    const T2 q = C[t];
    const R ps = psi[t];
    T2 g;
    g.x = q.x * ps;
    g.y = q.y * ps;
    C[nhalf + t] = g;
    // interior z planes of the half spectrum stand for two full-spectrum modes
    const double wgt = (k == 0 || (2 * k == K2)) ? 1.0 : 2.0;
    const double q2 = 0.5 * wgt * ((double)q.x * q.x + (double)q.y * q.y);
    if (dpsi) dpsi[t] = (ip || jp || kp) ? q2 : 0.0;
    if (ip || jp || kp) {
      const double m0 = ip * st->Li[0], m1 = jp * st->Li[1], m2 = kp * st->Li[2];
      const double mm = m0 * m0 + m1 * m1 + m2 * m2;
      v[0] = q2 * (double)ps;
      v[1] = v[0] * 2.0 * M_PI * M_PI * mm / (beta * beta * beta);
    }
  }
  block_reduce_finish<2>(v, partials, &st->red_counter[RED_SPME], st->scratch, true);
}

template <class R>
__global__ void __launch_bounds__(256)
k_spme_adj_gather(int N, const typename V4<R>::T* __restrict__ pos, const int* __restrict__ id, int n, int K0,
                  int K1, int K2, const DevState* __restrict__ st, const R* __restrict__ Phi,
                  double* __restrict__ dq, double* __restrict__ dr) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= N) return;
  const typename V4<R>::T p = pos[warp];
  int b0, b1, b2;
  R f0, f1, f2;
  grid_coord<R>(p.x, (R)st->Li[0], K0, b0, f0);
  grid_coord<R>(p.y, (R)st->Li[1], K1, b1, f1);
  grid_coord<R>(p.z, (R)st->Li[2], K2, b2, f2);
  R w0[16], w1[16], w2[16], d0[16], d1[16], d2[16];
  bspline_w<R>(n, f0, w0, d0);
  bspline_w<R>(n, f1, w1, d1);
  bspline_w<R>(n, f2, w2, d2);
  double pot = 0, gx = 0, gy = 0, gz = 0;
  for (int ab = lane; ab < n * n; ab += 32) {
    const int a = ab / n, b = ab % n;
    const long row = ((long)wrapk(b0 - a, K0) * K1 + wrapk(b1 - b, K1)) * K2;
    for (int c = 0; c < n; ++c) {
      const R g = Phi[row + wrapk(b2 - c, K2)];
      pot += (double)(g * w0[a] * w1[b] * w2[c]);
      gx += (double)(g * d0[a] * w1[b] * w2[c]);
      gy += (double)(g * w0[a] * d1[b] * w2[c]);
      gz += (double)(g * w0[a] * w1[b] * d2[c]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    pot += __shfl_xor_sync(0xffffffffu, pot, o);
    gx += __shfl_xor_sync(0xffffffffu, gx, o);
    gy += __shfl_xor_sync(0xffffffffu, gy, o);
    gz += __shfl_xor_sync(0xffffffffu, gz, o);
  }
  if (lane == 0) {
    const double q = (double)p.w;
    const int o = id[warp];  // results in the caller's atom order
    if (dq) dq[o] = pot;
    if (dr) {
      dr[3 * o] = q * gx * K0 * st->Li[0];
      dr[3 * o + 1] = q * gy * K1 * st->Li[1];
      dr[3 * o + 2] = q * gz * K2 * st->Li[2];
    }
  }
}

// ---------------------------------------------------------------- self-force correction
// SelfCorr (RE/src/SelfCorr.cpp:99-220), analytic differentiation, |k| <= 3:
//   c_d(k) = sum_{m != 0} f(m) (-2) g_d(m_d, k) (-4 pi k K_d / L_d),
//   f(m) = e^{-pi^2 |m|^2 / beta^2} / |m|^2 / (2 pi V)
//   g_d(m, k) = (u + 2 pi k)^-n / sum_{l=-3..3} (u + 2 pi l)^-n, u = 2 pi m / K_d
//   (0 at the Nyquist index of an even K_d);
//   F_id -= sum_{k=1..3} c_d(k) q_i^2 sin(2 pi k K_d x_id / L_d).
// g_d depends on m_d alone, so the K^3 sum is regrouped per axis: W_d(i) is
// the sum of f over the other two indices (one block per (i, d)), then the
// nine c_d(k) are 1-D sums.
__global__ void __launch_bounds__(256)
k_selfcorr_weights(int K0, int K1, int K2, double beta, const DevState* st, double* W /* [3][Kmax] */, int Kmax) {
  const int d = blockIdx.y, i = blockIdx.x;
  const int K[3] = {K0, K1, K2};
  if (i >= K[d]) return;
  const int a = (d + 1) % 3, b = (d + 2) % 3;
  int p[3];
  p[d] = i > (K[d] >> 1) ? i - K[d] : i;
  const double V = st->L[0] * st->L[1] * st->L[2];
  const double t = M_PI / beta, scal = 1.0 / (2.0 * M_PI * V);
  double acc = 0.0;
  for (int e = threadIdx.x; e < K[a] * K[b]; e += blockDim.x) {
    const int ia = e / K[b], ib = e % K[b];
    p[a] = ia > (K[a] >> 1) ? ia - K[a] : ia;
    p[b] = ib > (K[b] >> 1) ? ib - K[b] : ib;
    const double m0 = p[0] * st->Li[0], m1 = p[1] * st->Li[1], m2 = p[2] * st->Li[2];
    const double mm = m0 * m0 + m1 * m1 + m2 * m2;
    if (mm == 0.0) continue;
    acc += exp(-t * t * mm) / mm * scal;
  }
  __shared__ double sh[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
    W[d * Kmax + i] = s;
  }
}

__device__ __forceinline__ double ipow_dev(double x, int n) {
  double r = 1.0;
  for (int k = 0; k < n; ++k) r *= x;
  return r;
}

// one warp per (d, k), k = 1..3: c[d][k]
__global__ void k_selfcorr_coef(int K0, int K1, int K2, int order, const DevState* st, const double* W, int Kmax,
                                double* coef /* [3][4] */) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w >= 9) return;
  const int d = w / 3, kk = 1 + w % 3;
  const int K[3] = {K0, K1, K2};
  double acc = 0.0;
  for (int i = lane; i < K[d]; i += 32) {
    if (i == (K[d] >> 1) && (K[d] % 2 == 0)) continue;
    const int p = i > (K[d] >> 1) ? i - K[d] : i;
    const double u = 2.0 * M_PI * p / K[d];
    double s = 1.0 / ipow_dev(u, order), up = u, un = u;
    for (int l = 0; l < 3; ++l) {
      up += 2.0 * M_PI;
      un -= 2.0 * M_PI;
      s += 1.0 / ipow_dev(up, order);
      s += 1.0 / ipow_dev(un, order);
    }
    const double g = 1.0 / ipow_dev(u + 2.0 * M_PI * kk, order) / s;
    acc += W[d * Kmax + i] * (-2.0 * g) * (-4.0) * M_PI * kk * (double)K[d] * st->Li[d];
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) coef[d * 4 + kk] = acc;
}

template <class R>
__global__ void __launch_bounds__(256)
k_selfcorr_apply(int N, const typename V4<R>::T* __restrict__ pos, int K0, int K1, int K2, const DevState* st,
                 const double* __restrict__ coef, double4a* __restrict__ force) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const typename V4<R>::T p = pos[i];
  const double q2 = (double)p.w * (double)p.w;
  const double x[3] = {(double)p.x, (double)p.y, (double)p.z};
  const int K[3] = {K0, K1, K2};
  double f[3] = {0, 0, 0};
  for (int d = 0; d < 3; ++d)
    for (int kk = 1; kk <= 3; ++kk)
      f[d] -= coef[d * 4 + kk] * q2 * sinpi(2.0 * kk * K[d] * st->Li[d] * x[d]);
  double4a F = force[i];
  F.x += f[0]; F.y += f[1]; F.z += f[2];
  force[i] = F;
}

// ---------------------------------------------------------------- exact Ewald (FP64)
// S(m) = sum_i q_i exp(2 pi i m.r_i) for every m of the |m_d| <= K_d/2 box
// (EleRecES::calPotential), then E = sum_m e^{-pi^2 m^2/beta^2}/m^2 |S|^2 / (2 pi V)
// and F_i = sum_m (2/V) e^{..}/m^2 (S_r q_i sin - S_i q_i cos) m (applyInteraction).
__global__ void k_ewald_sk(int N, const double4a* __restrict__ pos, const float4* __restrict__ posf, int prec,
                           int M0, int M1, int M2, const DevState* st, double2* __restrict__ S) {
  const long nm = (long)(2 * M0 + 1) * (2 * M1 + 1) * (2 * M2 + 1);
  const long mi = blockIdx.x;
  if (mi >= nm) return;
  const int m2 = (int)(mi % (2 * M2 + 1)) - M2, m1 = (int)((mi / (2 * M2 + 1)) % (2 * M1 + 1)) - M1,
            m0 = (int)(mi / ((long)(2 * M2 + 1) * (2 * M1 + 1))) - M0;
  const double m[3] = {m0 * st->Li[0], m1 * st->Li[1], m2 * st->Li[2]};
  double sr = 0, si = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    double x, y, z, q;
    if (prec == MD_PREC_FP64) { const double4a p = pos[i]; x = p.x; y = p.y; z = p.z; q = p.w; }
    else { const float4 p = posf[i]; x = p.x; y = p.y; z = p.z; q = p.w; }
    double s, c;
    sincospi(2.0 * (m[0] * x + m[1] * y + m[2] * z), &s, &c);
    sr += q * c;
    si += q * s;
  }
  double v[2] = {sr, si};
  __shared__ double red[32][2];
  for (int o = 16; o > 0; o >>= 1) {
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    v[1] += __shfl_xor_sync(0xffffffffu, v[1], o);
  }
  if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5][0] = v[0]; red[threadIdx.x >> 5][1] = v[1]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += red[w][0]; b += red[w][1]; }
    S[mi] = make_double2(a, b);
  }
}

__global__ void k_ewald_force(int N, const double4a* __restrict__ pos, const float4* __restrict__ posf, int prec,
                              int M0, int M1, int M2, double beta, const DevState* st, const double2* __restrict__ S,
                              double4a* __restrict__ force, int add_forces, double* partials, unsigned* counter,
                              double* energy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const long nm = (long)(2 * M0 + 1) * (2 * M1 + 1) * (2 * M2 + 1);
  const double V = st->L[0] * st->L[1] * st->L[2];
  const double sc = M_PI * M_PI / (beta * beta);
  double x = 0, y = 0, z = 0, q = 0;
  if (i < N) {
    if (prec == MD_PREC_FP64) { const double4a p = pos[i]; x = p.x; y = p.y; z = p.z; q = p.w; }
    else { const float4 p = posf[i]; x = p.x; y = p.y; z = p.z; q = p.w; }
  }
  double fx = 0, fy = 0, fz = 0, e = 0;
  for (long mi = 0; mi < nm; ++mi) {
    const int m2 = (int)(mi % (2 * M2 + 1)) - M2, m1 = (int)((mi / (2 * M2 + 1)) % (2 * M1 + 1)) - M1,
              m0 = (int)(mi / ((long)(2 * M2 + 1) * (2 * M1 + 1))) - M0;
    if (!m0 && !m1 && !m2) continue;
    const double m[3] = {m0 * st->Li[0], m1 * st->Li[1], m2 * st->Li[2]};
    const double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
    const double ex = exp(-sc * mm) / mm;
    const double2 s = S[mi];
    if (i == 0) e += ex * (s.x * s.x + s.y * s.y);
    if (i < N) {
      double sn, cs;
      sincospi(2.0 * (m[0] * x + m[1] * y + m[2] * z), &sn, &cs);
      const double coeff = (s.x * q * sn - s.y * q * cs) * 2.0 / V * ex;
      fx += coeff * m[0]; fy += coeff * m[1]; fz += coeff * m[2];
    }
  }
  if (i < N && add_forces) {
    double4a f = force[i];
    f.x += fx; f.y += fy; f.z += fz;
    force[i] = f;
  }
  if (i == 0) *energy = e / (2.0 * M_PI * V);
  (void)partials; (void)counter;
}

// ---------------------------------------------------------------- host
template <class R>
static int fft_launch(md_spme* s, Recorder* rec, const void* in, void* out, int mode, int axis, int sign,
                      int batch) {
  const int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2], K2h = s->K2h;
  int n;
  long nlines, stride = 1, inner = 1, outer = 0, in_as = 0, out_as = 0;
  if (mode == 0) {
    n = K2; nlines = (long)K0 * K1;
  } else if (mode == 2) {
    n = K2; nlines = (long)K0 * K1;
    in_as = (long)s->nhalf; out_as = (long)s->nreal;
  } else if (axis == 1) {
    n = K1; nlines = (long)K0 * K2h; stride = K2h; inner = K2h; outer = (long)K1 * K2h;
    in_as = out_as = (long)s->nhalf;
  } else {
    n = K0; nlines = (long)K1 * K2h; stride = (long)K1 * K2h; inner = (long)K1 * K2h; outer = 0;
    in_as = out_as = (long)s->nhalf;
  }
  int lpb = 512 / n;
  if (lpb < 1) lpb = 1;
  const int threads = lpb * n / 2 < 32 ? 32 : lpb * n / 2;
  const size_t smem = sizeof(typename C2<R>::T) * (n / 2 + 2 * (size_t)lpb * n);
  dim3 grid((unsigned)((nlines + lpb - 1) / lpb), batch);
  void* a[] = {&in, &out, &mode, &n, &lpb, &nlines, &stride, &inner, &outer, &in_as, &out_as, &sign};
  return rec_launch(rec, (const void*)k_fft<R>, grid, dim3(threads), smem, a);
}

template <class R>
__global__ void k_zero_mesh(size_t n, R* Q) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t < n) Q[t] = R(0);
}

// influence refresh (only when the box changed), spread and the forward
// transform: C[0] = Q^ on the half spectrum.  Every launch goes through the
// recorder, so the chain is either run on the stream or recorded into the
// step graph of the simulation driver.
template <class R>
static int spme_forward_mesh(md_spme* s, Recorder* rec) {
  typedef typename C2<R>::T T2;
  md_system* sys = s->sys;
  int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2], n = s->order, N = sys->N;
  R* Q = (R*)s->Q;
  T2* C = (T2*)s->C;
  R* psi = (R*)s->psi;
  DevState* st = sys->st;
  double beta = s->beta;
  size_t nreal = s->nreal;
  {
    void* a[] = {&K0, &K1, &K2, &n, &beta, &st, &psi, &s->d_box_tab};
    if (int r = rec_launch(rec, (const void*)k_spme_influence<R>, dim3((unsigned)((s->nhalf + 255) / 256)),
                           dim3(256), 0, a)) return r;
  }
  {
    void* a[] = {&st, &s->d_box_tab};
    if (int r = rec_launch(rec, (const void*)k_spme_box_tab, dim3(1), dim3(1), 0, a)) return r;
  }
  {
    void* a[] = {&nreal, &Q};
    if (int r = rec_launch(rec, (const void*)k_zero_mesh<R>, dim3((unsigned)((nreal + 255) / 256)), dim3(256), 0, a))
      return r;
  }
  {
    const long nt = (long)N * n * n;
    const void* pos = sys->pos;
    void* a[] = {&N, &pos, &n, &K0, &K1, &K2, &st, &Q};
    if (int r = rec_launch(rec, (const void*)k_spme_spread<R>, dim3((unsigned)((nt + 255) / 256)), dim3(256), 0, a))
      return r;
  }
  if (int r = fft_launch<R>(s, rec, Q, C, 0, 2, -1, 1)) return r;
  if (int r = fft_launch<R>(s, rec, C, C, 1, 1, -1, 1)) return r;
  if (int r = fft_launch<R>(s, rec, C, C, 1, 0, -1, 1)) return r;
  return MD_OK;
}

template <class R>
static int spme_run(md_spme* s, bool with_stats, Recorder* rec) {
  typedef typename C2<R>::T T2;
  md_system* sys = s->sys;
  int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2], n = s->order, N = sys->N, method = s->method;
  T2* C = (T2*)s->C;
  R* G = (R*)s->G;
  DevState* st = sys->st;
  if (int r = spme_forward_mesh<R>(s, rec)) return r;
  const int nb = (int)((s->nhalf + 255) / 256);
  if (with_stats && nb > sys->max_partial_blocks) { md_set_error("partials buffer too small for the mesh"); return MD_ERR_BADARG; }
  {
    double beta = s->beta;
    const R* psi = (const R*)s->psi;
    size_t nhalf = s->nhalf;
    int ws = with_stats ? 1 : 0;
    void* a[] = {&K0, &K1, &K2, &method, &beta, &psi, &C, &nhalf, &st, &sys->partials, &ws};
    if (int r = rec_launch(rec, (const void*)k_spme_kspace<R>, dim3(nb), dim3(256), 0, a)) return r;
  }
  if (with_stats) {
    void* a[] = {&st};
    if (int r = rec_launch(rec, (const void*)k_spme_stats_merge, dim3(1), dim3(1), 0, a)) return r;
  }
  const int nconv = method == 0 ? 3 : 1;
  T2* Cp = C + s->nhalf;
  if (int r = fft_launch<R>(s, rec, Cp, Cp, 1, 0, +1, nconv)) return r;
  if (int r = fft_launch<R>(s, rec, Cp, Cp, 1, 1, +1, nconv)) return r;
  if (int r = fft_launch<R>(s, rec, Cp, G, 2, 2, +1, nconv)) return r;
  {
    const void* pos = sys->pos;
    size_t nreal = s->nreal;
    void* a[] = {&N, &pos, &n, &K0, &K1, &K2, &method, &st, &G, &nreal, &sys->force};
    if (int r = rec_launch(rec, (const void*)k_spme_gather<R>, dim3((unsigned)(((long)N * 32 + 255) / 256)),
                           dim3(256), 0, a)) return r;
  }
  return MD_OK;
}

bool spme_belongs_to(const md_spme* s, const md_system* sys) { return s && s->sys == sys; }

// the chain of one SPME force evaluation, recorded (driver) or launched
int spme_apply_impl(md_spme* s, bool with_stats, Recorder* rec) {
  return s->sys->prec == MD_PREC_FP64 ? spme_run<double>(s, with_stats, rec) : spme_run<float>(s, with_stats, rec);
}

// energy and gradient: recompute the mesh and its transform, influence
// multiply (energy, dE/dbeta, dE/dpsi), one inverse transform to Phi, gather
template <class R>
static int spme_energy_grad(md_spme* s, double* energy, double* dq, double* dr, double* dbeta, double* dpsi) {
  typedef typename C2<R>::T T2;
  md_system* sys = s->sys;
  cudaStream_t st_ = sys->stream;
  const int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2], n = s->order;
  T2* C = (T2*)s->C;
  R* G = (R*)s->G;
  const int nb = (int)((s->nhalf + 255) / 256);
  if (nb > sys->max_partial_blocks) { md_set_error("partials buffer too small for the mesh"); return MD_ERR_BADARG; }
  // device outputs: dq [N], dr [N][3], dpsi [nhalf] (FP64, caller's atom order)
  const size_t nq = dq ? (size_t)sys->N : 0, nr = dr ? 3 * (size_t)sys->N : 0, np = dpsi ? s->nhalf : 0;
  double* d = nullptr;
  if (nq + nr + np) MD_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * (nq + nr + np), st_));
  double* d_q = dq ? d : nullptr;
  double* d_r = dr ? d + nq : nullptr;
  double* d_p = dpsi ? d + nq + nr : nullptr;
  Recorder rec;
  rec.stream = st_;
  if (int r = spme_forward_mesh<R>(s, &rec)) return r;
  k_spme_adj_kspace<R><<<nb, 256, 0, st_>>>(K0, K1, K2, s->beta, (const R*)s->psi, C, s->nhalf, sys->st,
                                             sys->partials, d_p);
  MD_CHECK_LAUNCH("spme adjoint kspace");
  if (dq || dr) {
    T2* Cp = C + s->nhalf;
    if (int r = fft_launch<R>(s, &rec, Cp, Cp, 1, 0, +1, 1)) return r;
    if (int r = fft_launch<R>(s, &rec, Cp, Cp, 1, 1, +1, 1)) return r;
    if (int r = fft_launch<R>(s, &rec, Cp, G, 2, 2, +1, 1)) return r;
    k_spme_adj_gather<R><<<(unsigned)(((long)sys->N * 32 + 255) / 256), 256, 0, st_>>>(
        sys->N, (const typename V4<R>::T*)sys->pos, sys->id, n, K0, K1, K2, sys->st, G, d_q, d_r);
    MD_CHECK_LAUNCH("spme adjoint gather");
  }
  double red[2];
  MD_CUDA(cudaMemcpyAsync(red, sys->st->scratch, sizeof(red), cudaMemcpyDeviceToHost, st_));
  if (dq) MD_CUDA(cudaMemcpyAsync(dq, d_q, sizeof(double) * nq, cudaMemcpyDeviceToHost, st_));
  if (dr) MD_CUDA(cudaMemcpyAsync(dr, d_r, sizeof(double) * nr, cudaMemcpyDeviceToHost, st_));
  if (dpsi) MD_CUDA(cudaMemcpyAsync(dpsi, d_p, sizeof(double) * np, cudaMemcpyDeviceToHost, st_));
  if (d) MD_CUDA(cudaFreeAsync(d, st_));
  MD_CUDA(cudaStreamSynchronize(st_));
  if (energy) *energy = red[0];
  if (dbeta) *dbeta = red[1];
  return MD_OK;
}

static bool pow2(int k) { return k >= 2 && (k & (k - 1)) == 0; }

extern "C" int md_spme_create(md_spme** out, md_system* sys, const int K[3], int order, double beta, int method) {
  if (!out || !sys || !K || order < 2 || order > 14 || !(beta > 0) || (method != 0 && method != 1)) {
    md_set_error("md_spme_create: bad arguments");
    return MD_ERR_BADARG;
  }
  for (int d = 0; d < 3; ++d)
    if (!pow2(K[d]) || K[d] > 1024 || K[d] <= order) {
      md_set_error("md_spme_create: mesh sizes must be powers of two in (order, 1024]");
      return MD_ERR_BADARG;
    }
  md_spme* s = new md_spme();
  s->sys = sys;
  for (int d = 0; d < 3; ++d) s->K[d] = K[d];
  s->K2h = K[2] / 2 + 1;
  s->order = order;
  s->beta = beta;
  s->method = method;
  s->nreal = (size_t)K[0] * K[1] * K[2];
  s->nhalf = (size_t)K[0] * K[1] * s->K2h;
  const size_t rs = sys->real_size();
  bool ok = cudaMalloc(&s->Q, rs * s->nreal) == cudaSuccess &&
            cudaMalloc(&s->C, 2 * rs * s->nhalf * 4) == cudaSuccess &&
            cudaMalloc(&s->G, rs * s->nreal * 3) == cudaSuccess &&
            cudaMalloc(&s->psi, rs * s->nhalf) == cudaSuccess &&
            cudaMalloc(&s->d_box_tab, sizeof(double) * 3) == cudaSuccess &&
            cudaMemset(s->d_box_tab, 0, sizeof(double) * 3) == cudaSuccess;
  if (!ok) {
    md_cuda_fail(cudaGetLastError(), "md_spme_create");
    md_spme_destroy(s);
    return MD_ERR_CUDA;
  }
  *out = s;
  return MD_OK;
}

extern "C" int md_spme_destroy(md_spme* s) {
  if (!s) return MD_OK;
  void* p[] = {s->Q, s->C, s->G, s->psi, s->d_box_tab};
  for (void* q : p) if (q) cudaFree(q);
  delete s;
  return MD_OK;
}

extern "C" int md_spme_apply(md_spme* s, md_system* sys, int with_stats) {
  if (!s || !sys || sys != s->sys) { md_set_error("md_spme_apply: bad arguments"); return MD_ERR_BADARG; }
  Recorder rec;
  rec.stream = sys->stream;
  return spme_apply_impl(s, with_stats != 0, &rec);
}

extern "C" int md_spme_energy_grad(md_spme* s, md_system* sys, double* energy, double* dE_dq, double* dE_dr,
                                   double* dE_dbeta, double* dE_dpsi) {
  if (!s || !sys || sys != s->sys) { md_set_error("md_spme_energy_grad: bad arguments"); return MD_ERR_BADARG; }
  return sys->prec == MD_PREC_FP64 ? spme_energy_grad<double>(s, energy, dE_dq, dE_dr, dE_dbeta, dE_dpsi)
                                   : spme_energy_grad<float>(s, energy, dE_dq, dE_dr, dE_dbeta, dE_dpsi);
}

__global__ void k_mesh_out(size_t n, const float* a, const double* b, double* out);

extern "C" int md_spme_self_correction(md_spme* s, md_system* sys) {
  if (!s || !sys || sys != s->sys) { md_set_error("md_spme_self_correction: bad arguments"); return MD_ERR_BADARG; }
  const int Kmax = std::max(s->K[0], std::max(s->K[1], s->K[2]));
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * (3 * Kmax + 12), sys->stream));
  k_selfcorr_weights<<<dim3(Kmax, 3), 256, 0, sys->stream>>>(s->K[0], s->K[1], s->K[2], s->beta, sys->st, d, Kmax);
  MD_CHECK_LAUNCH("selfcorr weights");
  k_selfcorr_coef<<<1, 9 * 32, 0, sys->stream>>>(s->K[0], s->K[1], s->K[2], s->order, sys->st, d, Kmax,
                                                 d + 3 * Kmax);
  MD_CHECK_LAUNCH("selfcorr coef");
  const int nb = ceil_div(sys->N, 256);
  if (sys->prec == MD_PREC_FP64)
    k_selfcorr_apply<double><<<nb, 256, 0, sys->stream>>>(sys->N, (const double4a*)sys->pos, s->K[0], s->K[1],
                                                           s->K[2], sys->st, d + 3 * Kmax, sys->force);
  else
    k_selfcorr_apply<float><<<nb, 256, 0, sys->stream>>>(sys->N, (const float4*)sys->pos, s->K[0], s->K[1],
                                                         s->K[2], sys->st, d + 3 * Kmax, sys->force);
  MD_CHECK_LAUNCH("selfcorr apply");
  MD_CUDA(cudaFreeAsync(d, sys->stream));
  return MD_OK;
}

extern "C" int md_spme_get_influence(md_spme* s, double* psi) {
  if (!s || !psi) return MD_ERR_BADARG;
  md_system* sys = s->sys;
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * s->nhalf, sys->stream));
  const bool f = sys->prec != MD_PREC_FP64;
  k_mesh_out<<<(unsigned)((s->nhalf + 255) / 256), 256, 0, sys->stream>>>(
      s->nhalf, f ? (const float*)s->psi : nullptr, f ? nullptr : (const double*)s->psi, d);
  MD_CHECK_LAUNCH("influence out");
  MD_CUDA(cudaMemcpyAsync(psi, d, sizeof(double) * s->nhalf, cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaFreeAsync(d, sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}

__global__ void k_mesh_out(size_t n, const float* a, const double* b, double* out) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t < n) out[t] = a ? (double)a[t] : b[t];
}

extern "C" int md_spme_get_mesh(md_spme* s, double* Q) {
  if (!s || !Q) return MD_ERR_BADARG;
  md_system* sys = s->sys;
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * s->nreal, sys->stream));
  const bool f = sys->prec != MD_PREC_FP64;
  k_mesh_out<<<(unsigned)((s->nreal + 255) / 256), 256, 0, sys->stream>>>(
      s->nreal, f ? (const float*)s->Q : nullptr, f ? nullptr : (const double*)s->Q, d);
  MD_CHECK_LAUNCH("mesh out");
  MD_CUDA(cudaMemcpyAsync(Q, d, sizeof(double) * s->nreal, cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaFreeAsync(d, sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}

__global__ void k_self_energy(int N, const float4* pf, const double4a* pd, int prec, double beta, DevState* st,
                              double* partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0};
  if (i < N) {
    const double q = prec == MD_PREC_FP64 ? pd[i].w : (double)pf[i].w;
    v[0] = -beta / sqrt(M_PI) * q * q;
  }
  block_reduce_finish<1>(v, partials, &st->red_counter[RED_MISC], &st->stats[MD_STAT_ELEC_SELF], true);
}

extern "C" int md_ewald_self_energy(md_system* sys, double beta, double* out) {
  if (!sys || !(beta > 0)) return MD_ERR_BADARG;
  k_self_energy<<<ceil_div(sys->N, 256), 256, 0, sys->stream>>>(sys->N, (float4*)sys->pos, (double4a*)sys->pos,
                                                                 sys->prec, beta, sys->st, sys->partials);
  MD_CHECK_LAUNCH("self energy");
  if (out) {
    DevState hs;
    if (int r = sys->read_state(hs)) return r;
    *out = hs.stats[MD_STAT_ELEC_SELF];
  }
  return MD_OK;
}

extern "C" int md_ewald_exact(md_system* sys, const int K[3], double beta, double* energy, int add_forces) {
  if (!sys || !K || !(beta > 0)) return MD_ERR_BADARG;
  const int M0 = K[0] / 2, M1 = K[1] / 2, M2 = K[2] / 2;
  const long nm = (long)(2 * M0 + 1) * (2 * M1 + 1) * (2 * M2 + 1);
  double2* S = nullptr;
  double* e = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&S, sizeof(double2) * nm, sys->stream));
  MD_CUDA(cudaMallocAsync((void**)&e, sizeof(double), sys->stream));
  k_ewald_sk<<<(unsigned)nm, 256, 0, sys->stream>>>(sys->N, (double4a*)sys->pos, (float4*)sys->pos, sys->prec, M0, M1,
                                                     M2, sys->st, S);
  MD_CHECK_LAUNCH("ewald sk");
  k_ewald_force<<<ceil_div(sys->N, 128), 128, 0, sys->stream>>>(sys->N, (double4a*)sys->pos, (float4*)sys->pos,
                                                                 sys->prec, M0, M1, M2, beta, sys->st, S, sys->force,
                                                                 add_forces, nullptr, nullptr, e);
  MD_CHECK_LAUNCH("ewald force");
  double h = 0;
  MD_CUDA(cudaMemcpyAsync(&h, e, sizeof(double), cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaFreeAsync(S, sys->stream));
  MD_CUDA(cudaFreeAsync(e, sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  if (energy) *energy = h;
  return MD_OK;
}

