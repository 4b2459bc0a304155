// SPME (ik differentiation) with a piecewise cubic Hermite interpolation basis,
// and the hand-written adjoints that give the gradients of its energy and of a
// force-error functional with respect to the charges, the positions and the
// basis coefficients, for a batch of candidate bases, in FP64 on the GPU.
//
// The basis is optiBasis's symmetric Hermite basis (optiBasis/Hermite.py:6-130,
// optiBasis/HatComput.py:155-300): phi(x) = p(|x|) on |x| < CC grid units, p
// the cubic Hermite interpolant on nbin bins of width h = CC/nbin with value 1
// and slope 0 at 0 and the candidate's values v_j and slopes d_j at the other
// knots (coefficients [v_1..v_n, d_1..d_n], n = nbin, or nbin - 1 when bound0:
// value and slope 0 at CC).  The SPME it defines (RE/src/EleRecBSpline.cpp:
// 393-536 with the B-spline replaced by phi):
//   u_i,d   = K_d frac(r_i,d / L_d),  W_i(k) = prod_d phi(u_i,d - k_d)
//   Q(k)    = sum_i q_i W_i(k)                         (periodic in k)
//   Qh(m)   = sum_k Q(k) exp(-2 pi i m.k / K)
//   G(m)    = exp(-pi^2 |m|^2 / beta^2) / (pi V |m|^2) prod_d 1 / b_d(m_d)^2,
//             |m|^2 = sum_d (m_d / L_d)^2, G(0) = 0,
//             b_d(m)  = sum_{k integer} phi(k) exp(-2 pi i m k / K_d)   (real)
//   E       = 1/2 sum_m G(m) |Qh(m)|^2
//   phi_pot = IFFT(G Qh) (unnormalised: E = 1/2 sum_k Q phi_pot by Parseval)
//   F_i     = -q_i sum_k W_i(k) grad phi_pot(k),  grad phi_pot by ik:
//             IFFT(i 2 pi m_a/L_a G Qh) (the Nyquist term of axis a zeroed)
// b_d is the interpolation factor of SPME (1/|b(m)|^2 of calB,
// EleRecBSpline.cpp:729-796, is prod over the integer samples of the spline);
// with phi a (scaled) even-order cardinal B-spline this is the reference SPME.
//
// Adjoints (R = 2 (F - F_ref) / N the residual of the force-error functional
// L = 1/N sum_i |F_i - F_ref,i|^2, B_a = -sum_i q_i R_i,a W_i the residuals
// spread on the mesh, E_a = IFFT(i 2 pi m_a/L_a G Qh) the ik field):
//   dE/dq_i = sum_k W_i phi_pot,  dE/dr_i = q_i sum_k grad W_i phi_pot,
//   dE/dc   = sum_i q_i sum_k dW_i/dc phi_pot - sum_d sum_m P_d(m) db_d(m)/dc / b_d(m),
//             P_d(m_d) = sum over the other two indices of G |Qh|^2;
//   dL/dq_i = R_i . g_i + sum_k W_i Lam,   g_i = -sum_k W_i grad phi_pot,
//   dL/dr_i = -q_i sum_a R_i,a sum_k grad W_i E_a + q_i sum_k grad W_i Lam,
//   dL/dc   = -sum_i q_i sum_k dW_i/dc (R_i . E(k)) + sum_i q_i sum_k dW_i/dc Lam
//             - 2 sum_d sum_m H_d(m) db_d(m)/dc / b_d(m),
//   Lam     = -Re IFFT(sum_a i 2 pi m_a/L_a G Bh_a),
//   H_d     = marginals of Re(sum_a conj(Bh_a) i 2 pi m_a/L_a Qh) G
// (all inverse transforms unnormalised).
// Weights, their position and coefficient derivatives are evaluated in the
// spread and gather kernels; the 3D transforms are the FP64 grid transforms
// (radix-2 FFT for power-of-two meshes).
#include <cmath>
#include <cstring>
#include <vector>
#include "device_common.cuh"

int dft3_grid(double2* data, const int n[3], int sign, int batch, cudaStream_t stream);

namespace {

constexpr int HS_MAX_S = 16;      // stencil points per axis (2 ceil(CC))
constexpr int HS_MAX_NBIN = 64;
constexpr int HS_MAX_COEF = 2 * HS_MAX_NBIN;
constexpr int HS_THREADS = 128;
constexpr int HS_G = 8;                        // lanes per atom in the spread and gather
constexpr int HS_ATOMS = HS_THREADS / HS_G;    // atoms per spread / gather block

struct HsGeom {
  int K[3];
  double L[3];
  double beta, CC, h;
  int nbin, nk, ncoef, S, half;  // half = ceil(CC)
  long Kt;
};

// cubic Hermite polynomials and their derivatives in t
__device__ __forceinline__ void herm(double t, double v[4], double dv[4]) {
  v[0] = (1 + 2 * t) * (1 - t) * (1 - t);  // h00
  v[1] = t * (1 - t) * (1 - t);            // h10
  v[2] = t * t * (3 - 2 * t);              // h01
  v[3] = t * t * (t - 1);                  // h11
  dv[0] = 6 * t * (t - 1);
  dv[1] = (3 * t - 1) * (t - 1);
  dv[2] = 6 * t * (1 - t);
  dv[3] = t * (3 * t - 2);
}

// knot value / slope of the candidate c (knot 0: 1, 0; knots past nk: 0, 0)
__device__ __forceinline__ double knot_v(const HsGeom& g, const double* c, int j) {
  return j == 0 ? 1.0 : (j <= g.nk ? c[j - 1] : 0.0);
}
__device__ __forceinline__ double knot_d(const HsGeom& g, const double* c, int j) {
  return (j == 0 || j > g.nk) ? 0.0 : c[g.nk + j - 1];
}

// phi(x), phi'(x) and the (at most four) coefficients with a nonzero
// derivative dphi(x)/dc_b: index idx[t] (-1: none) and value dc[t]
struct PhiEval {
  double v, dv;
  int idx[4];
  double dc[4];
};

__device__ __forceinline__ PhiEval phi_eval(const HsGeom& g, const double* c, double x) {
  PhiEval e;
  e.v = 0.0;
  e.dv = 0.0;
  for (int t = 0; t < 4; ++t) { e.idx[t] = -1; e.dc[t] = 0.0; }
  const double ax = fabs(x);
  if (!(ax < g.CC)) return e;
  int j = (int)(ax / g.h);
  if (j >= g.nbin) j = g.nbin - 1;
  const double t = ax / g.h - j;
  double hv[4], hd[4];
  herm(t, hv, hd);
  const double V0 = knot_v(g, c, j), D0 = knot_d(g, c, j), V1 = knot_v(g, c, j + 1), D1 = knot_d(g, c, j + 1);
  const double p = hv[0] * V0 + hv[1] * g.h * D0 + hv[2] * V1 + hv[3] * g.h * D1;
  const double dp = (hd[0] * V0 + hd[1] * g.h * D0 + hd[2] * V1 + hd[3] * g.h * D1) / g.h;
  const double sg = x < 0 ? -1.0 : 1.0;
  e.v = p;
  e.dv = sg * dp;
  // dp/dv_j = h00, dp/dd_j = h10 h, dp/dv_{j+1} = h01, dp/dd_{j+1} = h11 h
  if (j >= 1 && j <= g.nk) { e.idx[0] = j - 1; e.dc[0] = hv[0]; e.idx[1] = g.nk + j - 1; e.dc[1] = hv[1] * g.h; }
  if (j + 1 <= g.nk) { e.idx[2] = j; e.dc[2] = hv[2]; e.idx[3] = g.nk + j; e.dc[3] = hv[3] * g.h; }
  return e;
}

__device__ __forceinline__ long mesh_index(const HsGeom& g, const int k[3]) {
  return (long)k[2] + (long)g.K[2] * ((long)k[1] + (long)g.K[1] * k[0]);
}

// stencil of one atom, shared by its HS_G lanes: first point k0_d and the
// weights phi and phi' per axis; the lanes evaluate the 3 S entries between
// them.  u_d is returned to every lane (the coefficient derivatives are
// re-evaluated from it at the end).
struct GroupStencil {
  int k0[3];
  double v[3][HS_MAX_S], dv[3][HS_MAX_S];
};

__device__ void group_stencil(const HsGeom& g, const double* c, const double* r, int sub, GroupStencil& s,
                              double u[3], int k0[3]) {
  for (int d = 0; d < 3; ++d) {
    double f = r[d] / g.L[d];
    f -= floor(f);
    u[d] = g.K[d] * f;
    k0[d] = (int)floor(u[d]) - g.half + 1;
  }
  if (sub == 0)
    for (int d = 0; d < 3; ++d) s.k0[d] = k0[d];
  for (int t = sub; t < 3 * g.S; t += HS_G) {
    const int d = t / g.S, j = t - d * g.S;
    const PhiEval e = phi_eval(g, c, u[d] - (double)(k0[d] + j));
    s.v[d][j] = e.v;
    s.dv[d][j] = e.dv;
  }
}

template <int W>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, W);
  return v;
}

__device__ __forceinline__ int wrap(int k, int K) {
  k %= K;
  return k < 0 ? k + K : k;
}

// b_d(m) and db_d(m)/dc_b for one candidate: one thread per (axis, m)
__global__ void k_hs_factor(HsGeom g, const double* __restrict__ c, double* __restrict__ bfac,
                            double* __restrict__ dbfac, int Kmax) {
  const int d = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= g.K[d]) return;
  double b = 0.0;
  double db[HS_MAX_COEF];
  for (int t = 0; t < g.ncoef; ++t) db[t] = 0.0;
  for (int k = -g.half; k <= g.half; ++k) {
    const PhiEval e = phi_eval(g, c, (double)k);
    double s, cs;
    sincospi(2.0 * (double)((long)m * (long)(k < 0 ? k + g.K[d] : k) % g.K[d]) / g.K[d], &s, &cs);
    b += e.v * cs;  // phi even: the imaginary parts cancel
    for (int t = 0; t < 4; ++t)
      if (e.idx[t] >= 0) db[e.idx[t]] += e.dc[t] * cs;
  }
  bfac[d * Kmax + m] = b;
  for (int t = 0; t < g.ncoef; ++t) dbfac[((long)d * g.ncoef + t) * Kmax + m] = db[t];
}

// spread: mode 0: Q += q_i W_i; mode 1: B_a -= q_i R_i,a W_i (three meshes).
// HS_G lanes per atom share its S^3 stencil points (lane l: points l, l + HS_G, ...).
__global__ void __launch_bounds__(HS_THREADS)
k_hs_spread(HsGeom g, int N, const double* __restrict__ q, const double* __restrict__ r,
            const double* __restrict__ c, int mode, const double* __restrict__ R, double2* __restrict__ mesh) {
  __shared__ GroupStencil gs[HS_ATOMS];
  const int grp = threadIdx.x / HS_G, sub = threadIdx.x % HS_G;
  const int i = blockIdx.x * HS_ATOMS + grp;
  if (i >= N) return;  // whole groups leave together; no block barrier below
  GroupStencil& s = gs[grp];
  double u[3];
  int k0[3];
  group_stencil(g, c, r + 3 * (long)i, sub, s, u, k0);
  __syncwarp(((1u << HS_G) - 1u) << (threadIdx.x & 31 & ~(HS_G - 1)));  // the group's lanes
  double a[3] = {q[i], 0.0, 0.0};
  if (mode == 1) for (int d = 0; d < 3; ++d) a[d] = -q[i] * R[3 * (long)i + d];
  const int S = g.S, S2 = S * S, S3 = S2 * S;
  for (int t = sub; t < S3; t += HS_G) {
    const int j0 = t / S2, j1 = (t / S) % S, j2 = t % S;
    const double w = s.v[0][j0] * s.v[1][j1] * s.v[2][j2];
    if (w == 0.0) continue;
    const int k[3] = {wrap(k0[0] + j0, g.K[0]), wrap(k0[1] + j1, g.K[1]), wrap(k0[2] + j2, g.K[2])};
    const long p = mesh_index(g, k);
    if (mode == 0) {
      atomicAdd(&mesh[p].x, a[0] * w);
    } else {
      for (int d = 0; d < 3; ++d) atomicAdd(&mesh[d * g.Kt + p].x, a[d] * w);
    }
  }
}

__device__ __forceinline__ void mvec(const HsGeom& g, long p, int m[3], double mv[3], bool nyq[3]) {
  const int i2 = (int)(p % g.K[2]);
  const int i1 = (int)((p / g.K[2]) % g.K[1]);
  const int i0 = (int)(p / ((long)g.K[2] * g.K[1]));
  const int id[3] = {i0, i1, i2};
  for (int d = 0; d < 3; ++d) {
    m[d] = id[d];
    const int md = id[d] <= g.K[d] / 2 ? id[d] : id[d] - g.K[d];
    mv[d] = md / g.L[d];
    nyq[d] = (g.K[d] % 2 == 0) && id[d] == g.K[d] / 2;
  }
}

__device__ __forceinline__ double influence(const HsGeom& g, const int m[3], const double mv[3],
                                            const double* __restrict__ bfac, int Kmax) {
  const double m2 = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
  if (m2 == 0.0) return 0.0;
  const double V = g.L[0] * g.L[1] * g.L[2];
  double b2 = 1.0;
  for (int d = 0; d < 3; ++d) {
    const double b = bfac[d * Kmax + m[d]];
    b2 *= b * b;
  }
  return exp(-M_PI * M_PI * m2 / (g.beta * g.beta)) / (M_PI * V * m2) / b2;
}

// k space of the forward pass: energy partials, the field transforms
// (i 2 pi m_a G Qh, a = 0..2), the potential transform G Qh, and the marginals
// P_d(m_d) of G |Qh|^2 (atomics)
__global__ void k_hs_kspace_fwd(HsGeom g, const double2* __restrict__ Qh, const double* __restrict__ bfac, int Kmax,
                                double2* __restrict__ field /* [4][Kt] */, double* __restrict__ marg,
                                double* __restrict__ epart) {
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double e = 0.0;
  if (p < g.Kt) {
    int m[3];
    double mv[3];
    bool nyq[3];
    mvec(g, p, m, mv, nyq);
    const double G = influence(g, m, mv, bfac, Kmax);
    const double2 z = Qh[p];
    const double a2 = z.x * z.x + z.y * z.y;
    e = 0.5 * G * a2;
    for (int d = 0; d < 3; ++d) {
      const double k = nyq[d] ? 0.0 : 2.0 * M_PI * mv[d] * G;  // i k z = (-k z.y, k z.x)
      field[d * g.Kt + p] = make_double2(-k * z.y, k * z.x);
    }
    field[3 * g.Kt + p] = make_double2(G * z.x, G * z.y);
    if (marg && G != 0.0)
      for (int d = 0; d < 3; ++d) atomicAdd(&marg[d * Kmax + m[d]], G * a2);
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    epart[blockIdx.x] = t;
  }
}

// k space of the loss adjoint: Lam transform -sum_a i k_a G Bh_a, and the
// marginals of Re(sum_a conj(Bh_a) i k_a Qh) G
__global__ void k_hs_kspace_adj(HsGeom g, const double2* __restrict__ Qh, const double2* __restrict__ Bh,
                                const double* __restrict__ bfac, int Kmax, double2* __restrict__ lam,
                                double* __restrict__ marg) {
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= g.Kt) return;
  int m[3];
  double mv[3];
  bool nyq[3];
  mvec(g, p, m, mv, nyq);
  const double G = influence(g, m, mv, bfac, Kmax);
  const double2 z = Qh[p];
  double lx = 0.0, ly = 0.0, h = 0.0;
  for (int d = 0; d < 3; ++d) {
    if (nyq[d]) continue;
    const double k = 2.0 * M_PI * mv[d];
    const double2 b = Bh[d * g.Kt + p];
    lx += k * G * b.y;   // -i k G b = (k G b.y, -k G b.x)
    ly -= k * G * b.x;
    // Re(conj(b) i k z) = k (b.x (-z.y) + b.y z.x)... conj(b) = (b.x, -b.y); i k z = (-k z.y, k z.x)
    h += k * (-b.x * z.y + b.y * z.x);
  }
  lam[p] = make_double2(lx, ly);
  if (marg && G != 0.0) {
    const double v = h * G;
    for (int d = 0; d < 3; ++d) atomicAdd(&marg[d * Kmax + m[d]], v);
  }
}

// The real parts of three field meshes and one scalar mesh interleaved per
// point (one 32-byte read per stencil point in the gather)
__global__ void k_hs_pack4(long Kt, const double2* __restrict__ a, const double2* __restrict__ s,
                           double4a* __restrict__ out) {
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p < Kt) out[p] = double4a{a[p].x, a[Kt + p].x, a[2 * Kt + p].x, s[p].x};
}

// Gather.  mode 0 (energy): F_i, dE/dq_i, dE/dr_i, dE/dc partials from the
// field meshes E_a and the potential (f4 = (E_0, E_1, E_2, phi)).  mode 1
// (loss, first pass): F_i only (into F).  mode 2 (loss, adjoint): dL/dq_i,
// dL/dr_i, dL/dc partials from f4 = (E_0, E_1, E_2, Lam).  HS_G lanes per atom
// split its S^3 stencil points; their sums are combined by shuffles in a
// fixed order.
__global__ void __launch_bounds__(HS_THREADS)
k_hs_gather(HsGeom g, int N, const double* __restrict__ q, const double* __restrict__ r,
            const double* __restrict__ c, int mode, const double4a* __restrict__ f4,
            const double* __restrict__ R, double* __restrict__ F, double* __restrict__ dq, double* __restrict__ dr,
            double* __restrict__ cpart) {
  __shared__ double csum[HS_MAX_COEF];
  __shared__ GroupStencil gs[HS_ATOMS];
  for (int t = threadIdx.x; t < g.ncoef; t += blockDim.x) csum[t] = 0.0;
  const int grp = threadIdx.x / HS_G, sub = threadIdx.x % HS_G;
  const int i = blockIdx.x * HS_ATOMS + grp;
  const bool live = i < N;
  GroupStencil& s = gs[grp];
  double u[3] = {0, 0, 0};
  int k0[3] = {0, 0, 0};
  if (live) group_stencil(g, c, r + 3 * (long)i, sub, s, u, k0);
  __syncthreads();
  const int S = g.S, S2 = S * S, S3 = S2 * S;
  const double qi = live ? q[i] : 0.0;
  double Ri[3] = {0, 0, 0};
  if (live && mode == 2)
    for (int d = 0; d < 3; ++d) Ri[d] = R[3 * (long)i + d];
  double Ef[3] = {0, 0, 0};    // sum W E_a
  double pot = 0.0;            // sum W phi (mode 0) or sum W Lam (mode 2)
  double gpot[3] = {0, 0, 0};  // sum grad W phi / Lam
  double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // sum d_b W E_a
  // partial contractions per axis for the coefficient gradient: T[d][j] =
  // sum over the other two axes of (scalar field) prod_{d' != d} w
  double T[3][HS_MAX_S];
  for (int d = 0; d < 3; ++d)
    for (int j = 0; j < S; ++j) T[d][j] = 0.0;
  const double kl[3] = {g.K[0] / g.L[0], g.K[1] / g.L[1], g.K[2] / g.L[2]};
  if (live)
    for (int t = sub; t < S3; t += HS_G) {
      const int j0 = t / S2, j1 = (t / S) % S, j2 = t % S;
      const double av = s.v[0][j0], adv = s.dv[0][j0], bv = s.v[1][j1], bdv = s.dv[1][j1];
      const double ev = s.v[2][j2], edv = s.dv[2][j2];
      const bool any = (av != 0.0 || adv != 0.0) && (bv != 0.0 || bdv != 0.0) && (ev != 0.0 || edv != 0.0);
      if (!any) continue;
      const double w12 = bv * ev, w02 = av * ev, w01 = av * bv;
      const double w = av * w12;
      const int k[3] = {wrap(k0[0] + j0, g.K[0]), wrap(k0[1] + j1, g.K[1]), wrap(k0[2] + j2, g.K[2])};
      const long p = mesh_index(g, k);
      const double gw[3] = {adv * kl[0] * w12, bdv * kl[1] * w02, edv * kl[2] * w01};
      const double4a fv = f4[p];  // E_0, E_1, E_2 and the scalar field (phi or Lam)
      const double E3[3] = {fv.x, fv.y, fv.z};
      for (int d = 0; d < 3; ++d) Ef[d] += w * E3[d];
      double sc = 0.0;  // the scalar field whose coefficient contraction is needed
      if (mode == 0) {
        const double ph = fv.w;
        pot += w * ph;
        for (int d = 0; d < 3; ++d) gpot[d] += gw[d] * ph;
        sc = ph;
      } else if (mode == 2) {
        const double lm = fv.w;
        pot += w * lm;
        for (int d = 0; d < 3; ++d) gpot[d] += gw[d] * lm;
        for (int a2 = 0; a2 < 3; ++a2)
          for (int b2 = 0; b2 < 3; ++b2) M[a2][b2] += gw[b2] * E3[a2];
        sc = lm - (Ri[0] * E3[0] + Ri[1] * E3[1] + Ri[2] * E3[2]);
      }
      if (mode != 1) {
        T[0][j0] += sc * w12;
        T[1][j1] += sc * w02;
        T[2][j2] += sc * w01;
      }
    }
  // group sums (every lane of the group ends with the totals)
  for (int d = 0; d < 3; ++d) Ef[d] = group_sum<HS_G>(Ef[d]);
  if (mode != 1) {
    pot = group_sum<HS_G>(pot);
    for (int d = 0; d < 3; ++d) gpot[d] = group_sum<HS_G>(gpot[d]);
    for (int d = 0; d < 3; ++d)
      for (int j = 0; j < S; ++j) T[d][j] = group_sum<HS_G>(T[d][j]);
  }
  if (mode == 2)
    for (int a2 = 0; a2 < 3; ++a2)
      for (int b2 = 0; b2 < 3; ++b2) M[a2][b2] = group_sum<HS_G>(M[a2][b2]);
  if (live && sub == 0) {
    if (mode == 0 || mode == 1)
      for (int d = 0; d < 3; ++d) F[3 * (long)i + d] = -qi * Ef[d];
    if (mode == 0) {
      if (dq) dq[i] = pot;
      if (dr) for (int d = 0; d < 3; ++d) dr[3 * (long)i + d] = qi * gpot[d];
    } else if (mode == 2) {
      // dL/dq_i = R_i . g_i + sum W Lam, g_i = -sum W E
      if (dq) dq[i] = -(Ri[0] * Ef[0] + Ri[1] * Ef[1] + Ri[2] * Ef[2]) + pot;
      if (dr)
        for (int b2 = 0; b2 < 3; ++b2) {
          double v = 0.0;
          for (int a2 = 0; a2 < 3; ++a2) v += Ri[a2] * M[a2][b2];
          dr[3 * (long)i + b2] = -qi * v + qi * gpot[b2];
        }
    }
  }
  if (live && mode != 1 && cpart) {
    // the group's lanes split the 3 S stencil entries, re-evaluating which
    // coefficients each weight depends on
    for (int t = sub; t < 3 * S; t += HS_G) {
      const int d = t / S, j = t - d * S;
      const double tv = qi * T[d][j];
      if (tv == 0.0) continue;
      const PhiEval e = phi_eval(g, c, u[d] - (double)(k0[d] + j));
      for (int b2 = 0; b2 < 4; ++b2)
        if (e.idx[b2] >= 0) atomicAdd(&csum[e.idx[b2]], tv * e.dc[b2]);
    }
  }
  __syncthreads();
  if (cpart)
    for (int t = threadIdx.x; t < g.ncoef; t += blockDim.x) cpart[(long)blockIdx.x * g.ncoef + t] = csum[t];
}

// coefficient gradient: block partials in a fixed order, plus the
// interpolation factor term -w sum_d sum_m marg_d(m) db_d(m)/dc / b_d(m)
__global__ void k_hs_coef_finish(HsGeom g, const double* __restrict__ cpart, int nblk, const double* __restrict__ marg,
                                 const double* __restrict__ bfac, const double* __restrict__ dbfac, int Kmax,
                                 double wfac, double* __restrict__ out, const double* __restrict__ epart, int neblk,
                                 double* __restrict__ energy) {
  const int t = threadIdx.x;
  if (out && t < g.ncoef) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += cpart[(long)b * g.ncoef + t];
    double f = 0.0;
    for (int d = 0; d < 3; ++d)
      for (int m = 0; m < g.K[d]; ++m) {
        const double b = bfac[d * Kmax + m];
        f += marg[d * Kmax + m] * dbfac[((long)d * g.ncoef + t) * Kmax + m] / b;
      }
    out[t] = s - wfac * f;
  }
  if (t == 0 && energy) {
    double e = 0.0;
    for (int b = 0; b < neblk; ++b) e += epart[b];
    *energy = e;
  }
}

__global__ void k_hs_residual(int N, const double* __restrict__ F, const double* __restrict__ Fref,
                              double* __restrict__ R, double* __restrict__ part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < N)
    for (int d = 0; d < 3; ++d) {
      const double e = F[3 * (long)i + d] - Fref[3 * (long)i + d];
      R[3 * (long)i + d] = 2.0 * e / N;
      l += e * e / N;
    }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_hs_sum(const double* __restrict__ part, int n, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += part[b];
    *out = s;
  }
}

}  // namespace

struct md_hspme {
  int device = 0;
  int N = 0;
  HsGeom g;
  int Kmax = 0;
  double2* mesh = nullptr;   // [4][Kt]: Q / Qh, then field and potential [4][Kt] below
  double2* fld = nullptr;    // [4][Kt]
  double2* bmesh = nullptr;  // [3][Kt] residual spread / transforms
  double2* lam = nullptr;    // [Kt]
  double4a* f4 = nullptr;    // [Kt] gather input: fields and one scalar mesh, real parts
  double* bfac = nullptr;    // [3][Kmax]
  double* dbfac = nullptr;   // [3][ncoef][Kmax]
  double* marg = nullptr;    // [3][Kmax]
  double* epart = nullptr;   // [k-space blocks]
  double* cpart = nullptr;   // [atom blocks][ncoef]
  double* R = nullptr;       // [N][3] residual weights
  double* Fw = nullptr;      // [N][3] forces of the loss pass
};

static void hs_free(md_hspme* h) {
  void* p[] = {h->mesh, h->fld, h->bmesh, h->lam, h->f4, h->bfac, h->dbfac, h->marg, h->epart, h->cpart, h->R, h->Fw};
  for (void* x : p) if (x) cudaFree(x);
}

extern "C" int md_hspme_create(md_hspme** out, int natoms, const int K[3], const double L[3], double beta, double CC,
                               int nbin, int bound0, int device) {
  if (!out || natoms < 1 || !K || !L || !(beta > 0) || !(CC > 0) || nbin < 1 || nbin > HS_MAX_NBIN) {
    md_set_error("md_hspme_create: bad arguments");
    return MD_ERR_BADARG;
  }
  const int half = (int)ceil(CC - 1e-12);
  if (2 * half > HS_MAX_S) { md_set_error("md_hspme_create: support CC %g wider than %d grid points", CC, HS_MAX_S); return MD_ERR_BADARG; }
  for (int d = 0; d < 3; ++d)
    if (K[d] < 2 * half + 1 || K[d] > 1024 || !(L[d] > 0)) {
      md_set_error("md_hspme_create: mesh %d or box %g out of range on axis %d", K[d], L[d], d);
      return MD_ERR_BADARG;
    }
  MD_CUDA(cudaSetDevice(device));
  md_hspme* h = new md_hspme();
  h->device = device;
  h->N = natoms;
  HsGeom& g = h->g;
  for (int d = 0; d < 3; ++d) { g.K[d] = K[d]; g.L[d] = L[d]; }
  g.beta = beta;
  g.CC = CC;
  g.nbin = nbin;
  g.h = CC / nbin;
  g.nk = bound0 ? nbin - 1 : nbin;
  g.ncoef = 2 * g.nk;
  g.half = half;
  g.S = 2 * half;
  g.Kt = (long)K[0] * K[1] * K[2];
  h->Kmax = std::max(K[0], std::max(K[1], K[2]));
  const long Kt = g.Kt;
  const long nkb = (Kt + 255) / 256, nab = (natoms + HS_ATOMS - 1) / HS_ATOMS;
  bool ok = cudaMalloc(&h->mesh, sizeof(double2) * Kt) == cudaSuccess &&
            cudaMalloc(&h->fld, sizeof(double2) * 4 * Kt) == cudaSuccess &&
            cudaMalloc(&h->bmesh, sizeof(double2) * 3 * Kt) == cudaSuccess &&
            cudaMalloc(&h->lam, sizeof(double2) * Kt) == cudaSuccess &&
            cudaMalloc(&h->f4, sizeof(double4a) * Kt) == cudaSuccess &&
            cudaMalloc(&h->bfac, sizeof(double) * 3 * h->Kmax) == cudaSuccess &&
            cudaMalloc(&h->dbfac, sizeof(double) * 3 * std::max(g.ncoef, 1) * h->Kmax) == cudaSuccess &&
            cudaMalloc(&h->marg, sizeof(double) * 3 * h->Kmax) == cudaSuccess &&
            cudaMalloc(&h->epart, sizeof(double) * std::max(nkb, nab)) == cudaSuccess &&
            cudaMalloc(&h->cpart, sizeof(double) * nab * std::max(g.ncoef, 1)) == cudaSuccess &&
            cudaMalloc(&h->R, sizeof(double) * 3 * natoms) == cudaSuccess &&
            cudaMalloc(&h->Fw, sizeof(double) * 3 * natoms) == cudaSuccess;
  if (!ok) {
    md_cuda_fail(cudaGetLastError(), "md_hspme_create");
    hs_free(h);
    delete h;
    return MD_ERR_CUDA;
  }
  *out = h;
  return MD_OK;
}

extern "C" int md_hspme_destroy(md_hspme* h) {
  if (!h) return MD_OK;
  cudaSetDevice(h->device);
  hs_free(h);
  delete h;
  return MD_OK;
}

extern "C" int md_hspme_num_coeffs(md_hspme* h, int* out) {
  if (!h || !out) return MD_ERR_BADARG;
  *out = h->g.ncoef;
  return MD_OK;
}

// forward pass of candidate c: factors, spread, transform, k space, the four
// inverse transforms (three field components and the potential)
static int hs_forward(md_hspme* h, const double* q, const double* r, const double* c, cudaStream_t s,
                      bool want_marg) {
  HsGeom& g = h->g;
  const long Kt = g.Kt;
  const int nab = (h->N + HS_ATOMS - 1) / HS_ATOMS;
  const int nkb = (int)((Kt + 255) / 256);
  k_hs_factor<<<dim3((h->Kmax + 63) / 64, 3), 64, 0, s>>>(g, c, h->bfac, h->dbfac, h->Kmax);
  MD_CHECK_LAUNCH("hspme factor");
  MD_CUDA(cudaMemsetAsync(h->mesh, 0, sizeof(double2) * Kt, s));
  k_hs_spread<<<nab, HS_THREADS, 0, s>>>(g, h->N, q, r, c, 0, nullptr, h->mesh);
  MD_CHECK_LAUNCH("hspme spread");
  if (int e = dft3_grid(h->mesh, g.K, -1, 1, s)) return e;
  if (want_marg) MD_CUDA(cudaMemsetAsync(h->marg, 0, sizeof(double) * 3 * h->Kmax, s));
  k_hs_kspace_fwd<<<nkb, 256, 0, s>>>(g, h->mesh, h->bfac, h->Kmax, h->fld, want_marg ? h->marg : nullptr,
                                      h->epart);
  MD_CHECK_LAUNCH("hspme kspace");
  return dft3_grid(h->fld, g.K, +1, 4, s);
}

extern "C" int md_hspme_energy(md_hspme* h, const double* q, const double* r, const double* coeffs, int C,
                               double* energy, double* forces, double* dE_dq, double* dE_dr, double* dE_dc,
                               void* stream) {
  if (!h || !q || !r || !coeffs || C < 1 || !energy) { md_set_error("md_hspme_energy: bad arguments"); return MD_ERR_BADARG; }
  MD_CUDA(cudaSetDevice(h->device));
  cudaStream_t s = (cudaStream_t)stream;
  HsGeom& g = h->g;
  const int N = h->N;
  const int nab = (N + HS_ATOMS - 1) / HS_ATOMS;
  const int nkb = (int)((g.Kt + 255) / 256);
  for (int b = 0; b < C; ++b) {
    const double* c = coeffs + (long)b * g.ncoef;
    if (int e = hs_forward(h, q, r, c, s, dE_dc != nullptr)) return e;
    double* F = forces ? forces + 3L * N * b : h->Fw;
    k_hs_pack4<<<nkb, 256, 0, s>>>(g.Kt, h->fld, h->fld + 3 * g.Kt, h->f4);
    MD_CHECK_LAUNCH("hspme pack");
    k_hs_gather<<<nab, HS_THREADS, 0, s>>>(g, N, q, r, c, 0, h->f4, nullptr, F,
                                           dE_dq ? dE_dq + (long)N * b : nullptr, dE_dr ? dE_dr + 3L * N * b : nullptr,
                                           dE_dc ? h->cpart : nullptr);
    MD_CHECK_LAUNCH("hspme gather");
    // the factor term of dE/dc: 1/2 sum G|Qh|^2 (-2 db/b) = -sum P db / b
    k_hs_coef_finish<<<1, std::max(32, ((g.ncoef + 31) / 32) * 32), 0, s>>>(
        g, h->cpart, nab, h->marg, h->bfac, h->dbfac, h->Kmax, 1.0, dE_dc ? dE_dc + (long)g.ncoef * b : nullptr,
        h->epart, nkb, energy + b);
    MD_CHECK_LAUNCH("hspme finish");
  }
  return MD_OK;
}

extern "C" int md_hspme_force_error(md_hspme* h, const double* q, const double* r, const double* coeffs, int C,
                                    const double* fref, double* loss, double* dL_dq, double* dL_dr, double* dL_dc,
                                    void* stream) {
  if (!h || !q || !r || !coeffs || C < 1 || !fref || !loss) {
    md_set_error("md_hspme_force_error: bad arguments");
    return MD_ERR_BADARG;
  }
  MD_CUDA(cudaSetDevice(h->device));
  cudaStream_t s = (cudaStream_t)stream;
  HsGeom& g = h->g;
  const int N = h->N;
  const long Kt = g.Kt;
  const int nab = (N + HS_ATOMS - 1) / HS_ATOMS;       // spread / gather blocks
  const int nrb = (N + HS_THREADS - 1) / HS_THREADS;   // residual blocks
  const int nkb = (int)((Kt + 255) / 256);
  const bool grads = dL_dq || dL_dr || dL_dc;
  for (int b = 0; b < C; ++b) {
    const double* c = coeffs + (long)b * g.ncoef;
    if (int e = hs_forward(h, q, r, c, s, false)) return e;
    k_hs_pack4<<<nkb, 256, 0, s>>>(Kt, h->fld, h->fld + 3 * Kt, h->f4);
    MD_CHECK_LAUNCH("hspme pack");
    k_hs_gather<<<nab, HS_THREADS, 0, s>>>(g, N, q, r, c, 1, h->f4, nullptr, h->Fw, nullptr, nullptr, nullptr);
    MD_CHECK_LAUNCH("hspme gather");
    k_hs_residual<<<nrb, HS_THREADS, 0, s>>>(N, h->Fw, fref, h->R, h->epart);
    MD_CHECK_LAUNCH("hspme residual");
    k_hs_sum<<<1, 32, 0, s>>>(h->epart, nrb, loss + b);
    MD_CHECK_LAUNCH("hspme loss");
    if (!grads) continue;
    // adjoint: residuals spread, transformed, Lam and the factor marginals
    MD_CUDA(cudaMemsetAsync(h->bmesh, 0, sizeof(double2) * 3 * Kt, s));
    k_hs_spread<<<nab, HS_THREADS, 0, s>>>(g, N, q, r, c, 1, h->R, h->bmesh);
    MD_CHECK_LAUNCH("hspme residual spread");
    if (int e = dft3_grid(h->bmesh, g.K, -1, 3, s)) return e;
    MD_CUDA(cudaMemsetAsync(h->marg, 0, sizeof(double) * 3 * h->Kmax, s));
    k_hs_kspace_adj<<<nkb, 256, 0, s>>>(g, h->mesh, h->bmesh, h->bfac, h->Kmax, h->lam, h->marg);
    MD_CHECK_LAUNCH("hspme adjoint kspace");
    if (int e = dft3_grid(h->lam, g.K, +1, 1, s)) return e;
    k_hs_pack4<<<nkb, 256, 0, s>>>(Kt, h->fld, h->lam, h->f4);
    MD_CHECK_LAUNCH("hspme pack");
    k_hs_gather<<<nab, HS_THREADS, 0, s>>>(g, N, q, r, c, 2, h->f4, h->R, nullptr,
                                           dL_dq ? dL_dq + (long)N * b : nullptr, dL_dr ? dL_dr + 3L * N * b : nullptr,
                                           dL_dc ? h->cpart : nullptr);
    MD_CHECK_LAUNCH("hspme adjoint gather");
    if (dL_dc) {
      // factor term of dL/dc through G: sum_m H(m) dG/dc = -2 sum_d sum_m H_d db/b
      k_hs_coef_finish<<<1, std::max(32, ((g.ncoef + 31) / 32) * 32), 0, s>>>(
          g, h->cpart, nab, h->marg, h->bfac, h->dbfac, h->Kmax, 2.0, dL_dc + (long)g.ncoef * b, nullptr, 0,
          nullptr);
      MD_CHECK_LAUNCH("hspme adjoint finish");
    }
  }
  return MD_OK;
}
