// Smooth particle-mesh Ewald (reciprocal part) and the exact Ewald sum.
// Reference (RE = longRange.hetero/profile.test/template/tools/real.error):
//   calQ spread                      RE/src/EleRecBSpline.cpp:541-619
//   calB / calPsiFPhiF (ik)          RE/src/EleRecBSpline.cpp:729-877
//   applyInteractionCalPotential ik  RE/src/EleRecBSpline.cpp:393-536
//   analytic differentiation         RE/src/EleRecFBSpline.cpp:771-907, 1146-1195
//   exact reciprocal sum (ES)        RE/src/EleRecES.cpp:49-144
//
// Chain of one force evaluation (each step one kernel):
//   spread      charges into a shared-memory tile per block of 64 charges,
//               the tile added to the mesh with 4-wide atomics
//   z pass      R2C along z (real lines -> half-complex lines)
//   y pass      forward C2C along y
//   x pass      forward C2C along x, k-space step (energy and virial in FP64,
//               influence multiply; ik: the three products i(-2 pi m_d) psi Q^,
//               analytic: psi Q^ / 2) and the inverse C2C along x, fused
//   y pass      inverse C2C along y (all products)
//   z pass      C2R along z with the Hermitian completion of an r2c half
//               spectrum (the FFTW c2r convention the reference relies on);
//               for ik the three meshes are written interleaved, one Real4
//               per mesh point
//   gather      order-templated, LPA lanes per atom
// The FFT passes are radix-8 Stockham transforms of whole lines in shared
// memory; a block holds several lines adjacent in memory so that strided
// axes load coalesced.  Mixed precision: mesh, FFT and gather in FP32,
// energy/virial and force accumulation in FP64.  Power-of-two mesh sizes.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <type_traits>
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
  void* G = nullptr;      // convolved real mesh(es): ik Real4 (x, y, z, 0) per point; analytic and adjoint one Real
  void* psi = nullptr;    // influence function on the half spectrum (ik normalisation)
  void* tw[3] = {nullptr, nullptr, nullptr};  // per-axis forward twiddles exp(-2 pi i m / K_d)
  double* bm = nullptr;   // per-axis |b(m)|^2 (k_spme_bmod)
  double4a* frec = nullptr;   // reciprocal forces of a concurrent evaluation (stored, not added)
  double* partials = nullptr; // block partials of the x pass (its own: it may run beside other reductions)
  int max_blocks = 0;
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

// The same recursion with the order a compile-time constant, so that the
// weight arrays stay in registers (a runtime order spills them to local
// memory).  D: also the derivatives dM_n/du.
template <class R, int NO, bool D>
__device__ __forceinline__ void bsp_t(R f, R (&w)[NO], R (&dw)[NO]) {
  w[0] = f;
  w[1] = R(1) - f;
#pragma unroll
  for (int j = 2; j < NO; ++j) w[j] = R(0);
#pragma unroll
  for (int k = 3; k <= NO; ++k) {
    if (D && k == NO) {
#pragma unroll
      for (int j = 0; j < NO; ++j) dw[j] = (j < NO - 1 ? w[j] : R(0)) - (j > 0 ? w[j - 1] : R(0));
    }
    const R inv = R(1) / R(k - 1);
#pragma unroll
    for (int j = k - 1; j >= 0; --j) {
      const R u = f + R(j);
      const R a = (j < k - 1) ? w[j] : R(0);
      const R b = (j > 0) ? w[j - 1] : R(0);
      w[j] = (u * a + (R(k) - u) * b) * inv;
    }
  }
  if (D && NO == 2) { dw[0] = R(1); dw[1] = R(-1); }
}

// Orders with a compiled spread / gather (md_spme_create accepts 2..14).
#define SPME_ORDERS(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14)

// ---------------------------------------------------------------- spread
// A block takes SPREAD_ATOMS consecutive charges (cell order, hence compact
// in space) and spreads them into a shared-memory tile that covers their
// stencils, with shared-memory atomics; the tile is then added to the mesh
// with one 4-wide atomic per 4 z points (binary32) or scalar atomics
// (binary64), skipping empty groups.  Each charge's stencil base is taken in
// the periodic image closest to the block's first charge, so that a block
// next to a periodic face still has a compact tile.  The tile's z origin and
// extent are multiples of 4 (K2 is a power of two >= 4, so a group never
// wraps); rows are padded by one element against bank conflicts.  A block
// whose tile does not fit adds every stencil point with a global atomic.
constexpr int SPREAD_ATOMS = 64;
constexpr int SPREAD_THREADS = 256;
constexpr int SPREAD_TILE_BYTES = 64 * 1024;

template <class R>
__device__ __forceinline__ void mesh_add4(R* dst, R a, R b, R c, R d);
template <>
__device__ __forceinline__ void mesh_add4<float>(float* dst, float a, float b, float c, float d) {
  atomicAdd(reinterpret_cast<float4*>(dst), make_float4(a, b, c, d));
}
template <>
__device__ __forceinline__ void mesh_add4<double>(double* dst, double a, double b, double c, double d) {
  if (a != 0.0) atomicAdd(dst, a);
  if (b != 0.0) atomicAdd(dst + 1, b);
  if (c != 0.0) atomicAdd(dst + 2, c);
  if (d != 0.0) atomicAdd(dst + 3, d);
}

template <class R, int NO>
__global__ void __launch_bounds__(SPREAD_THREADS)
k_spme_spread_t(int N, const typename V4<R>::T* __restrict__ pos, int K0, int K1, int K2,
                const DevState* __restrict__ st, R* __restrict__ Q, int tile_cap) {
  extern __shared__ __align__(16) unsigned char sp_smem[];
  R* tile = reinterpret_cast<R*>(sp_smem);
  __shared__ R sw[3][NO][SPREAD_ATOMS];
  __shared__ R sq[SPREAD_ATOMS];
  __shared__ int sb[3][SPREAD_ATOMS];
  __shared__ int sbox[6];
  const int i0 = blockIdx.x * SPREAD_ATOMS;
  const int na = min(SPREAD_ATOMS, N - i0);
  const int K[3] = {K0, K1, K2};
  if (threadIdx.x < 6) sbox[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;
  __syncthreads();
  if ((int)threadIdx.x < na) {
    const typename V4<R>::T p = pos[i0 + threadIdx.x], p0 = pos[i0];
    const R x[3] = {p.x, p.y, p.z}, x0[3] = {p0.x, p0.y, p0.z};
    const R q = p.w;
    sq[threadIdx.x] = q;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int b, r;
      R f, fr;
      grid_coord<R>(x[d], (R)st->Li[d], K[d], b, f);
      grid_coord<R>(x0[d], (R)st->Li[d], K[d], r, fr);
      const int dv = b - r;
      if (2 * dv > K[d]) b -= K[d];
      else if (2 * dv < -K[d]) b += K[d];
      sb[d][threadIdx.x] = b;
      R w[NO], dw[NO];
      bsp_t<R, NO, false>(f, w, dw);
#pragma unroll
      for (int j = 0; j < NO; ++j) sw[d][j][threadIdx.x] = w[j];
      if (q != R(0)) {
        atomicMin(&sbox[d], b);
        atomicMax(&sbox[3 + d], b);
      }
    }
  }
  __syncthreads();
  if (sbox[0] > sbox[3]) return;  // no charge in this block
  const int o0 = sbox[0] - (NO - 1), o1 = sbox[1] - (NO - 1);
  const int o2 = (sbox[2] - (NO - 1)) & ~3;
  const long e0 = sbox[3] - o0 + 1, e1 = sbox[4] - o1 + 1;
  const long e2 = (sbox[5] - o2 + 4) & ~3;
  const long rs = e2 + 1;
  const int nab = na * NO * NO;
  if (e0 * e1 * rs <= tile_cap) {
    const int tsz = (int)(e0 * e1 * rs), ie1 = (int)e1, irs = (int)rs;
    for (int e = threadIdx.x; e < tsz; e += SPREAD_THREADS) tile[e] = R(0);
    __syncthreads();
    for (int e = threadIdx.x; e < nab; e += SPREAD_THREADS) {
      const int at = e / (NO * NO), ab = e - at * (NO * NO), a = ab / NO, b = ab - a * NO;
      const R q = sq[at];
      if (q == R(0)) continue;
      const R qab = q * sw[0][a][at] * sw[1][b][at];
      R* row = tile + ((sb[0][at] - a - o0) * ie1 + (sb[1][at] - b - o1)) * irs + (sb[2][at] - o2);
#pragma unroll
      for (int c = 0; c < NO; ++c) atomicAdd(row - c, qab * sw[2][c][at]);
    }
    __syncthreads();
    const int g2 = (int)(e2 >> 2), ng = (int)(e0 * e1) * g2;
    for (int g = threadIdx.x; g < ng; g += SPREAD_THREADS) {
      const int z4 = g % g2, xy = g / g2, y = xy % ie1, x = xy / ie1;
      const R* s = tile + (x * ie1 + y) * irs + 4 * z4;
      const R v0 = s[0], v1 = s[1], v2 = s[2], v3 = s[3];
      if (v0 == R(0) && v1 == R(0) && v2 == R(0) && v3 == R(0)) continue;
      const int gx = (o0 + x) & (K0 - 1), gy = (o1 + y) & (K1 - 1), gz = (o2 + 4 * z4) & (K2 - 1);
      mesh_add4<R>(Q + ((size_t)gx * K1 + gy) * K2 + gz, v0, v1, v2, v3);
    }
  } else {
    for (int e = threadIdx.x; e < nab; e += SPREAD_THREADS) {
      const int at = e / (NO * NO), ab = e - at * (NO * NO), a = ab / NO, b = ab - a * NO;
      const R q = sq[at];
      if (q == R(0)) continue;
      const R qab = q * sw[0][a][at] * sw[1][b][at];
      const size_t row = ((size_t)((sb[0][at] - a) & (K0 - 1)) * K1 + ((sb[1][at] - b) & (K1 - 1))) * K2;
#pragma unroll
      for (int c = 0; c < NO; ++c) atomicAdd(Q + row + ((sb[2][at] - c) & (K2 - 1)), qab * sw[2][c][at]);
    }
  }
}

// ---------------------------------------------------------------- FFT
// Stockham transform of whole lines in shared memory, in the formulation of
// Govindaraju et al. (SC'08): with Ns the length already transformed, stage
// (radix R) takes butterfly j < n/R, reads its R inputs at stride n/R,
// multiplies input r by W_n^{r k n/(Ns R)} (k = j mod Ns), applies an R-point
// DFT in registers and writes output r to (j / Ns) Ns R + k + r Ns.  Stages
// of radix 8, then one of radix 4 or 2, cover n = 2^LOGN and leave the line
// in natural order.  One stage reads all its inputs, synchronises and then
// writes, so a single buffer per line suffices.  A block of FFT_THREADS
// threads holds FFT_THREADS / TPL lines (TPL = n/8 threads per line), each
// padded by one element; twiddles come from a per-axis table computed once
// in FP64 (conjugated for the inverse transform).
constexpr int FFT_THREADS = 128;

template <class T2>
__device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <class T2>
__device__ __forceinline__ T2 c_add(T2 a, T2 b) {
  T2 r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <class T2>
__device__ __forceinline__ T2 c_sub(T2 a, T2 b) {
  T2 r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
// a * (SIGN i)
template <int SIGN, class T2>
__device__ __forceinline__ T2 c_mul_si(T2 a) {
  T2 r;
  r.x = SIGN > 0 ? -a.y : a.y;
  r.y = SIGN > 0 ? a.x : -a.x;
  return r;
}

// X_s = sum_r v_r exp(SIGN 2 pi i r s / 4)
template <int SIGN, class T2>
__device__ __forceinline__ void dft4(T2& v0, T2& v1, T2& v2, T2& v3) {
  const T2 s0 = c_add(v0, v2), d0 = c_sub(v0, v2), s1 = c_add(v1, v3), d1 = c_mul_si<SIGN>(c_sub(v1, v3));
  v0 = c_add(s0, s1);
  v2 = c_sub(s0, s1);
  v1 = c_add(d0, d1);
  v3 = c_sub(d0, d1);
}

template <class R, int RR, int SIGN>
__device__ __forceinline__ void dft_reg(typename C2<R>::T (&v)[RR]) {
  typedef typename C2<R>::T T2;
  if constexpr (RR == 2) {
    const T2 a = v[0];
    v[0] = c_add(a, v[1]);
    v[1] = c_sub(a, v[1]);
  } else if constexpr (RR == 4) {
    dft4<SIGN>(v[0], v[1], v[2], v[3]);
  } else {
    // radix 8 = two radix-4 DFTs of the even and odd inputs, odd ones
    // multiplied by W^k, W = exp(SIGN 2 pi i / 8)
    T2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<SIGN>(e0, e1, e2, e3);
    dft4<SIGN>(o0, o1, o2, o3);
    const R h = R(0.70710678118654752440);  // 1/sqrt(2)
    T2 t;
    t.x = (SIGN > 0 ? o1.x - o1.y : o1.x + o1.y) * h;
    t.y = (SIGN > 0 ? o1.y + o1.x : o1.y - o1.x) * h;
    o1 = t;
    o2 = c_mul_si<SIGN>(o2);
    t.x = (SIGN > 0 ? -o3.x - o3.y : -o3.x + o3.y) * h;
    t.y = (SIGN > 0 ? -o3.y + o3.x : -o3.y - o3.x) * h;
    o3 = t;
    v[0] = c_add(e0, o0);
    v[4] = c_sub(e0, o0);
    v[1] = c_add(e1, o1);
    v[5] = c_sub(e1, o1);
    v[2] = c_add(e2, o2);
    v[6] = c_sub(e2, o2);
    v[3] = c_add(e3, o3);
    v[7] = c_sub(e3, o3);
  }
}

template <int LOGN>
struct FftGeom {
  static constexpr int n = 1 << LOGN;
  static constexpr int TPL = n >= 8 ? n / 8 : 1;  // threads per line
  static constexpr int LPB = FFT_THREADS / TPL;   // lines per block
  static constexpr int LS = n + 1;                // padded line stride
  static constexpr int EPT = LPB * n / FFT_THREADS;  // elements per thread
};

// the stages from Ns = 2^LOGNS on, for the line x of this thread (lane tl of
// the line's TPL threads); every thread of the block takes part
template <class R, int LOGN, int LOGNS, int SIGN>
__device__ __forceinline__ void fft_stages(typename C2<R>::T* x, const typename C2<R>::T* tw, int tl) {
  typedef typename C2<R>::T T2;
  constexpr int n = 1 << LOGN, TPL = FftGeom<LOGN>::TPL;
  constexpr int LR = (LOGN - LOGNS) >= 3 ? 3 : (LOGN - LOGNS);
  constexpr int RR = 1 << LR, NS = 1 << LOGNS, NBF = n / RR, BPT = NBF / TPL;
  static_assert(BPT >= 1, "at least one butterfly per thread");
  T2 v[BPT][RR];
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int j = tl + q * TPL;
#pragma unroll
    for (int r = 0; r < RR; ++r) v[q][r] = x[j + r * NBF];
    if constexpr (LOGNS > 0) {
      const int k = j & (NS - 1);
#pragma unroll
      for (int r = 1; r < RR; ++r) v[q][r] = cmul(v[q][r], tw[(r * k) << (LOGN - LOGNS - LR)]);
    }
    dft_reg<R, RR, SIGN>(v[q]);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < BPT; ++q) {
    const int j = tl + q * TPL;
    const int d = ((j >> LOGNS) << (LOGNS + LR)) + (j & (NS - 1));
#pragma unroll
    for (int r = 0; r < RR; ++r) x[d + r * NS] = v[q][r];
  }
  __syncthreads();
  if constexpr (LOGNS + LR < LOGN) fft_stages<R, LOGN, LOGNS + LR, SIGN>(x, tw, tl);
}

// the block barriers of fft_stages<R, LOGN, LOGNS, *> without the work: a
// group with nothing to transform meets the others' barriers
template <int LOGN, int LOGNS>
__device__ __forceinline__ void fft_stage_barriers() {
  constexpr int LR = (LOGN - LOGNS) >= 3 ? 3 : (LOGN - LOGNS);
  __syncthreads();
  __syncthreads();
  if constexpr (LOGNS + LR < LOGN) fft_stage_barriers<LOGN, LOGNS + LR>();
}

template <class R, int SIGN>
__device__ __forceinline__ void load_tw(typename C2<R>::T* tw, const typename C2<R>::T* __restrict__ twg, int n) {
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    typename C2<R>::T w = twg[m];
    if (SIGN > 0) w.y = -w.y;
    tw[m] = w;
  }
}

// One transform pass over lines of one axis.
//   MODE 0: real lines along z (contiguous) -> half-complex lines (n/2+1);
//           the input lines are cleared after they are read
//   MODE 1: complex lines of the half spectrum; line L starts at
//           (L / inner) * outer + L % inner, elements `stride` apart; lines
//           adjacent in memory share a block, so loads coalesce across lines
//   MODE 2: half-complex z lines -> real lines (Hermitian completion, the
//           FFTW c2r convention the reference relies on)
// blockIdx.y selects the batch (in_bs / out_bs apart).  OUT4 (MODE 2): the
// three batches of a line are transformed side by side in one block, by
// three groups of FFT_THREADS threads, and written interleaved, one Real4
// (x, y, z, 0) per mesh point.
template <class R, int LOGN, int MODE, int SIGN, int OUT4>
__global__ void __launch_bounds__(FFT_THREADS * (OUT4 ? 2 : 1))
k_fftp(const void* in, void* out, const typename C2<R>::T* __restrict__ twg, long nlines, long stride, long inner,
       long outer, long in_bs, long out_bs) {
  typedef typename C2<R>::T T2;
  typedef FftGeom<LOGN> G;
  // OUT4: the three Hermitian spectra become the x, y, z of one real
  // 4-vector mesh; group 0 inverts A + iB (the x and y spectra: both results
  // real, they come back as the real and imaginary parts), group 1 the z
  constexpr int n = G::n, LPB = G::LPB, LS = G::LS, NG = OUT4 ? 2 : 1, nh = n / 2 + 1;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  T2* tw = reinterpret_cast<T2*>(fft_smem);
  T2* X = tw + n;
  long* lo = reinterpret_cast<long*>(X + NG * LPB * LS);
  load_tw<R, SIGN>(tw, twg, n);
  // MODE 0: the real lines 2L and 2L + 1 go in as the real and imaginary
  // parts of complex line L, and their half spectra are separated after the
  // transform: A_k = (Z_k + conj Z_{n-k}) / 2, B_k = (Z_k - conj Z_{n-k}) / 2i
  const long nlc = MODE == 0 ? (nlines + 1) / 2 : nlines;  // complex lines
  const long line0 = (long)blockIdx.x * LPB;
  if (threadIdx.x < LPB) {
    const long L = line0 + threadIdx.x;
    lo[threadIdx.x] = MODE == 1 ? (L / inner) * outer + L % inner : L;
  }
  __syncthreads();
  const int grp = NG > 1 ? (int)threadIdx.x / FFT_THREADS : 0;
  const int gt = NG > 1 ? (int)threadIdx.x % FFT_THREADS : (int)threadIdx.x;
  const long batch = OUT4 ? 2 * grp : blockIdx.y;
  T2* Xb = X + grp * LPB * LS;
  {
    // all loads of a thread are issued before any shared-memory store (and,
    // in MODE 0, before the mesh is cleared), so they are in flight together
    T2 vv[G::EPT];
#pragma unroll
    for (int s = 0; s < G::EPT; ++s) {
      const int e = gt + s * FFT_THREADS;
      int l, k;
      if (MODE == 1) { l = e % LPB; k = e / LPB; }
      else { l = e >> LOGN; k = e & (n - 1); }
      const long L = line0 + l;
      T2 v;
      v.x = R(0);
      v.y = R(0);
      if (L < nlc) {
        if (MODE == 0) {
          const R* src = reinterpret_cast<const R*>(in) + batch * in_bs;
          v.x = src[2 * L * n + k];
          if (2 * L + 1 < nlines) v.y = src[(2 * L + 1) * n + k];
        } else if (MODE == 1) {
          v = reinterpret_cast<const T2*>(in)[batch * in_bs + lo[l] + k * stride];
        } else {
          const T2* src = reinterpret_cast<const T2*>(in) + batch * in_bs + L * nh;
          if (k < nh) v = src[k];
          else { const T2 u = src[n - k]; v.x = u.x; v.y = -u.y; }
          if (OUT4 && grp == 0) {
            // + i B, B the spectrum of the next batch.  A real transform
            // ignores the imaginary parts at k = 0 and n/2 (the mirrored half
            // carries the rest); they are dropped here, or they would cross
            // into the other result
            const T2* srb = src + in_bs;
            T2 b;
            if (k < nh) b = srb[k];
            else { const T2 u = srb[n - k]; b.x = u.x; b.y = -u.y; }
            if (k == 0 || k == n / 2) { v.y = R(0); b.y = R(0); }
            v.x -= b.y;
            v.y += b.x;
          }
        }
      }
      vv[s] = v;
    }
#pragma unroll
    for (int s = 0; s < G::EPT; ++s) {
      const int e = gt + s * FFT_THREADS;
      int l, k;
      if (MODE == 1) { l = e % LPB; k = e / LPB; }
      else { l = e >> LOGN; k = e & (n - 1); }
      if (MODE == 0) {
        // the real mesh is consumed: cleared for the next spread
        const long L = line0 + l;
        R* src = reinterpret_cast<R*>(const_cast<void*>(in)) + batch * in_bs;
        if (L < nlc) src[2 * L * n + k] = R(0);
        if (2 * L + 1 < nlines) src[(2 * L + 1) * n + k] = R(0);
      }
      Xb[l * LS + k] = vv[s];
    }
  }
  __syncthreads();
  fft_stages<R, LOGN, 0, SIGN>(Xb + (gt / G::TPL) * LS, tw, gt % G::TPL);
  if (OUT4) {
    typedef typename V4<R>::T R4;
    for (int e = threadIdx.x; e < LPB * n; e += NG * FFT_THREADS) {
      const int l2 = e >> LOGN, k = e & (n - 1);
      const long L = line0 + l2;
      if (L >= nlines) continue;
      R4 o;
      const T2 xy = X[l2 * LS + k];
      o.x = xy.x;
      o.y = xy.y;
      o.z = X[LPB * LS + l2 * LS + k].x;
      o.w = R(0);
      reinterpret_cast<R4*>(out)[L * n + k] = o;
    }
    return;
  }
  for (int e = threadIdx.x; e < LPB * n; e += FFT_THREADS) {
    int l2, k;
    if (MODE == 1) { l2 = e % LPB; k = e / LPB; }
    else { l2 = e >> LOGN; k = e & (n - 1); }
    const long L = line0 + l2;
    if (L >= nlc) continue;
    const T2 v = X[l2 * LS + k];
    if (MODE == 0) {
      if (k < nh) {
        const T2 w = X[l2 * LS + ((n - k) & (n - 1))];
        T2 a, b;
        a.x = R(0.5) * (v.x + w.x);
        a.y = R(0.5) * (v.y - w.y);
        b.x = R(0.5) * (v.y + w.y);
        b.y = R(0.5) * (w.x - v.x);
        T2* dst = reinterpret_cast<T2*>(out) + batch * out_bs;
        dst[2 * L * nh + k] = a;
        if (2 * L + 1 < nlines) dst[(2 * L + 1) * nh + k] = b;
      }
    } else if (MODE == 1) {
      reinterpret_cast<T2*>(out)[batch * out_bs + lo[l2] + k * stride] = v;
    } else {
      reinterpret_cast<R*>(out)[batch * out_bs + L * n + k] = v.x;
    }
  }
}

template <class R>
static size_t fftp_smem(int logn, int nbuf) {
  const int n = 1 << logn, tpl = n >= 8 ? n / 8 : 1, lpb = FFT_THREADS / tpl;
  return sizeof(typename C2<R>::T) * ((size_t)n + (size_t)nbuf * lpb * (n + 1)) + sizeof(long) * lpb;
}

// Forward transform along x, the k-space step and the inverse transform(s)
// along x, in one pass over the x lines (y, kz fixed) of the half spectrum:
//   psi(m) = exp(-pi^2 m^2 / beta^2) / m^2 |b0(i)|^2 |b1(j)|^2 |b2(k)|^2 / (pi V)
//     (calB / calPsiFPhiF), evaluated in FP64 from the per-axis |b|^2
//     tables for the current box, so an NPT box change needs no extra pass,
//   E = 1/2 sum_m psi |Q^|^2 and the diagonal virial (FP64, with_stats),
//   ik (METHOD 0): the three products phi_d = i (-2 pi m_d) psi Q^,
//   (merge = 0: the sums stay in DevState::scratch for a later merge)
//   analytic (METHOD 1): psi Q^ / 2 (FBSpline normalisation),
// each transformed back along x and written to C[1 + d].  Groups of
// FFT_THREADS threads: group 0 runs the forward transform and the k-space
// step (group 1 meets the same barriers), then for ik group 0 inverts phi_x
// and group 1 inverts psi Q^,
// whose transform times -2 pi i m_y and -2 pi i m_z (constant along the
// line) gives phi_y and phi_z.  The last block merges the energy and the
// virial into the statistics slots.
template <class R, int LOGN, int METHOD>
__global__ void __launch_bounds__(FFT_THREADS * (METHOD == 0 ? 3 : 1))
k_fft_x_kspace(typename C2<R>::T* C, const typename C2<R>::T* __restrict__ twg, const double* __restrict__ bm, int K1,
               int K2, double beta, DevState* st, double* partials, int with_stats, int merge) {
  typedef typename C2<R>::T T2;
  typedef FftGeom<LOGN> G;
  // ik: group 0 transforms -2 pi i m_x psi Q^ back; m_y and m_z are constant
  // along an x line, so group 1 transforms psi Q^ once and its result, times
  // -2 pi i m_y and -2 pi i m_z, gives the other two products
  constexpr int n = G::n, LPB = G::LPB, LS = G::LS, EPT = G::EPT, NG = METHOD == 0 ? 2 : 1;
  const int K2h = K2 / 2 + 1;
  const long nlines = (long)K1 * K2h, stride = nlines;
  const size_t nhalf = (size_t)n * nlines;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  T2* twf = reinterpret_cast<T2*>(fft_smem);
  T2* twi = twf + n;
  T2* X = twi + n;
  T2* Y = X + LPB * LS;  // NG buffers
  R* PS = reinterpret_cast<R*>(Y + NG * LPB * LS);
  // psi = exp(-pi^2 m^2 / beta^2) / m^2 * B(m) / (pi V) factors by axis: the
  // x factors exp(-sc m_x^2) b_x(i) for the n points of a line and, per line
  // (j, k), exp(-sc (m_y^2 + m_z^2)) b_y(j) b_z(k) / (pi V) and m_y^2 + m_z^2,
  // worked out once per block (FP64), leaving one reciprocal per point
  double* EX = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(PS + LPB * LS) + 7) & ~(uintptr_t)7);
  double* EJK = EX + n;
  double* MJK = EJK + LPB;
  int* lj = reinterpret_cast<int*>(MJK + LPB);
  int* lk = lj + LPB;
  load_tw<R, -1>(twf, twg, n);
  load_tw<R, 1>(twi, twg, n);
  const long line0 = (long)blockIdx.x * LPB;
  const double sc = M_PI * M_PI / (beta * beta);
  if (threadIdx.x < LPB) {
    const long L = line0 + threadIdx.x;
    const int j = (int)(L / K2h), k = (int)(L % K2h);
    lj[threadIdx.x] = j;
    lk[threadIdx.x] = k;
    const int jp = j <= K1 / 2 ? j : j - K1;
    const double my = jp * st->Li[1], mz = k * st->Li[2], mjk = my * my + mz * mz;
    const double V = st->L[0] * st->L[1] * st->L[2];
    MJK[threadIdx.x] = mjk;
    EJK[threadIdx.x] = exp(-sc * mjk) * (bm[n + j] * bm[n + K1 + k]) / (M_PI * V);
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int ip = i <= n / 2 ? i : i - n;
    const double mx = ip * st->Li[0];
    EX[i] = exp(-sc * mx * mx) * bm[i];
  }
  const int grp = NG > 1 ? (int)threadIdx.x / FFT_THREADS : 0;
  const int gt = NG > 1 ? (int)threadIdx.x % FFT_THREADS : (int)threadIdx.x;
  if (grp == 0) {
    T2 vv[EPT];
#pragma unroll
    for (int s = 0; s < EPT; ++s) {
      const int e = gt + s * FFT_THREADS, l = e % LPB, i = e / LPB;
      const long L = line0 + l;
      vv[s].x = R(0);
      vv[s].y = R(0);
      if (L < nlines) vv[s] = C[L + i * stride];
    }
#pragma unroll
    for (int s = 0; s < EPT; ++s) {
      const int e = gt + s * FFT_THREADS;
      X[(e % LPB) * LS + e / LPB] = vv[s];
    }
  }
  __syncthreads();
  const int l = gt / G::TPL, tl = gt % G::TPL;
  if (grp == 0) fft_stages<R, LOGN, 0, -1>(X + l * LS, twf, tl);
  else fft_stage_barriers<LOGN, 0>();
  double v[4] = {0, 0, 0, 0};
  if (grp == 0) {
#pragma unroll
    for (int s = 0; s < EPT; ++s) {
      const int e = gt + s * FFT_THREADS, le = e % LPB, i = e / LPB;
      const long L = line0 + le;
      const int j = lj[le], k = lk[le];
      const int ip = i <= n / 2 ? i : i - n, jp = j <= K1 / 2 ? j : j - K1;
      const double mx = ip * st->Li[0];
      const double mm = mx * mx + MJK[le];
      const bool live = L < nlines && (ip || jp || k);
      const double inv = live ? 1.0 / mm : 0.0;
      const R ps = live ? (R)(EX[i] * EJK[le] * inv) : R(0);
      PS[le * LS + i] = ps;
      if (with_stats && live) {
        // E = 1/2 sum_m |Q^|^2 psi over the full spectrum: interior z planes count twice
        const T2 q = X[le * LS + i];
        const double wgt = (k == 0 || (2 * k == K2)) ? 1.0 : 2.0;
        const double e2 = 0.5 * wgt * ((double)q.x * q.x + (double)q.y * q.y) * (double)ps;
        // f = 2 (1 + pi^2 m^2 / beta^2) / m^2
        const double f = 2.0 * inv + 2.0 * sc;
        const double m[3] = {mx, jp * st->Li[1], k * st->Li[2]};
        v[0] += e2;
        // pressure tensor V P_aa = sum_m E_m (1 - f m_a^2); the virial slots hold W_aa = -V P_aa
#pragma unroll
        for (int d = 0; d < 3; ++d) v[1 + d] += -e2 * (1.0 - f * m[d] * m[d]);
      }
    }
  }
  __syncthreads();
  T2* Yg = Y + grp * LPB * LS;
#pragma unroll
  for (int s = 0; s < EPT; ++s) {
    const int e = gt + s * FFT_THREADS, le = e % LPB, i = e / LPB;
    const T2 q = X[le * LS + i];
    const R ps = PS[le * LS + i];
    T2 g;
    if (METHOD == 0 && grp == 0) {
      // phi_x = i (-2 pi m_x) psi Q^, m_x = i' / L_x (signed index)
      const int ix = i <= n / 2 ? i : i - n;
      const R c = (R)(-2.0 * M_PI * (ix * st->Li[0])) * ps;
      g.x = -q.y * c;
      g.y = q.x * c;
    } else if (METHOD == 0) {
      g.x = q.x * ps;
      g.y = q.y * ps;
    } else {
      g.x = q.x * (R(0.5) * ps);
      g.y = q.y * (R(0.5) * ps);
    }
    Yg[le * LS + i] = g;
  }
  __syncthreads();
  fft_stages<R, LOGN, 0, 1>(Yg + l * LS, twi, tl);
  if (METHOD == 0 && grp == 1) {
    // phi_y and phi_z = i (-2 pi m_d) times the transform of psi Q^
    T2* outy = C + 2 * nhalf;
    T2* outz = C + 3 * nhalf;
    for (int e = gt; e < LPB * n; e += FFT_THREADS) {
      const int le = e % LPB, i = e / LPB;
      const long L = line0 + le;
      if (L >= nlines) continue;
      const int jp = lj[le] <= K1 / 2 ? lj[le] : lj[le] - K1;
      const R cy = (R)(-2.0 * M_PI * (jp * st->Li[1])), cz = (R)(-2.0 * M_PI * (lk[le] * st->Li[2]));
      const T2 v = Yg[le * LS + i];
      T2 a, b;
      a.x = -v.y * cy;
      a.y = v.x * cy;
      b.x = -v.y * cz;
      b.y = v.x * cz;
      outy[L + i * stride] = a;
      outz[L + i * stride] = b;
    }
  } else {
    T2* out = C + (1 + grp) * nhalf;
    for (int e = gt; e < LPB * n; e += FFT_THREADS) {
      const int le = e % LPB, i = e / LPB;
      const long L = line0 + le;
      if (L < nlines) out[L + i * stride] = Yg[le * LS + i];
    }
  }
  if (with_stats && block_reduce_finish<4>(v, partials, &st->red_counter[RED_SPME], st->scratch, true) && merge) {
    // reciprocal energy into its slot, its diagonal virial added to the virial slots
    st->stats[MD_STAT_ELEC_REC] = st->scratch[0];
    for (int d = 0; d < 3; ++d) st->stats[MD_STAT_VIRIAL_XX + d] += st->scratch[1 + d];
  }
}

template <class R>
static size_t fftx_smem(int logn, int method) {
  const int n = 1 << logn, tpl = n >= 8 ? n / 8 : 1, lpb = FFT_THREADS / tpl, ng = method == 0 ? 2 : 1;
  return sizeof(typename C2<R>::T) * (2 * (size_t)n + (1 + (size_t)ng) * lpb * (n + 1)) +
         sizeof(R) * (size_t)lpb * (n + 1) + 8 + sizeof(double) * ((size_t)n + 2 * lpb) + 2 * sizeof(int) * lpb;
}

// per-axis forward twiddle table exp(-2 pi i m / n), m < n, from FP64
template <class R>
__global__ void k_fft_twiddles(int n, typename C2<R>::T* tw) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  double s, c;
  sincospi(2.0 * m / n, &s, &c);
  tw[m].x = (R)c;
  tw[m].y = (R)(-s);
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
// round trip is needed, and `tab` is updated by k_spme_box_tab afterwards.
// The force chain evaluates psi inside its x pass; this stored copy serves
// the adjoint and md_spme_get_influence.
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

// per-axis |b_d(m)|^2 tables, concatenated: [0, K0) | [0, K1) | [0, K2/2+1)
__global__ void k_spme_bmod(int K0, int K1, int K2, int n, double* bm) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < K0) bm[t] = bmod_d(n, K0, t);
  else if (t < K0 + K1) bm[t] = bmod_d(n, K1, t - K0);
  else if (t < K0 + K1 + K2 / 2 + 1) bm[t] = bmod_d(n, K2, t - K0 - K1);
}

// ---------------------------------------------------------------- gather
// A block takes GATHER_ATOMS consecutive atoms (cell order) with LPA lanes
// each (the power of two >= order, at least 4); lane a takes the stencil
// plane b0 - a and runs over its order^2 points, and the lanes' sums are
// combined by shuffles.  The block first stages the mesh region covering its
// charges' stencils (image-adjusted as in the spread) into shared memory
// with coalesced, independent row loads, then gathers from there; a block
// whose region does not fit reads the mesh directly.
//   MODE 0: ik, the three convolved meshes interleaved, one Real4 per point
//   MODE 1: analytic differentiation of the single convolved mesh
//   MODE 2: adjoint gather of Phi: potential dE/dq_i and exact position
//           gradient dE/dx_i, written in the caller's atom order
// store (MODES 0, 1): force is a separate buffer that receives every atom's
// reciprocal force (zero for neutral atoms) instead of accumulating it.
// MD_SPME_GATHER_TILE_KB: shared-memory budget of the staged region (0: read
// the mesh directly)
#ifndef MD_SPME_GATHER_TILE_KB
#define MD_SPME_GATHER_TILE_KB 64
#endif
constexpr int GATHER_ATOMS = 32;
constexpr int GATHER_TILE_BYTES = MD_SPME_GATHER_TILE_KB * 1024;

__host__ __device__ constexpr int gather_lanes(int order) { return order <= 4 ? 4 : (order <= 8 ? 8 : 16); }

// one stencil row of order points: point c at G[-c] (the staged region) or
// at G[kz[c]] (the mesh, wrapped indices)
template <class R, int NO, int MODE, class GT, class A>
__device__ __forceinline__ void gather_row(const GT* G, R wa, R da, R w1b, R d1b, const R (&w2)[NO],
                                           const R (&d2)[NO], A& s0, A& s1, A& s2, A& s3) {
  const R wab = wa * w1b;
  if constexpr (MODE == 0) {
#pragma unroll
    for (int c = 0; c < NO; ++c) {
      const GT g = G[-c];
      const R w = wab * w2[c];
      s0 += g.x * w;
      s1 += g.y * w;
      s2 += g.z * w;
    }
  } else {
    const R dab = da * w1b, wdb = wa * d1b;
#pragma unroll
    for (int c = 0; c < NO; ++c) {
      const R g = G[-c];
      if (MODE == 1) {
        s0 -= g * dab * w2[c];
        s1 -= g * wdb * w2[c];
        s2 -= g * wab * d2[c];
      } else {
        s0 += (double)(g * wab * w2[c]);
        s1 += (double)(g * dab * w2[c]);
        s2 += (double)(g * wdb * w2[c]);
        s3 += (double)(g * wab * d2[c]);
      }
    }
  }
}

template <class R, int NO, int MODE, class GT, class A>
__device__ __forceinline__ void gather_row_idx(const GT* G, const int (&kz)[NO], R wa, R da, R w1b, R d1b,
                                               const R (&w2)[NO], const R (&d2)[NO], A& s0, A& s1, A& s2, A& s3) {
  const R wab = wa * w1b;
  if constexpr (MODE == 0) {
#pragma unroll
    for (int c = 0; c < NO; ++c) {
      const GT g = G[kz[c]];
      const R w = wab * w2[c];
      s0 += g.x * w;
      s1 += g.y * w;
      s2 += g.z * w;
    }
  } else {
    const R dab = da * w1b, wdb = wa * d1b;
#pragma unroll
    for (int c = 0; c < NO; ++c) {
      const R g = G[kz[c]];
      if (MODE == 1) {
        s0 -= g * dab * w2[c];
        s1 -= g * wdb * w2[c];
        s2 -= g * wab * d2[c];
      } else {
        s0 += (double)(g * wab * w2[c]);
        s1 += (double)(g * dab * w2[c]);
        s2 += (double)(g * wdb * w2[c]);
        s3 += (double)(g * wab * d2[c]);
      }
    }
  }
}

template <class R, int NO, int MODE>
__global__ void __launch_bounds__(GATHER_ATOMS * gather_lanes(NO))
k_spme_gather_t(int N, const typename V4<R>::T* __restrict__ pos, const int* __restrict__ id, int K0, int K1,
                int K2, const DevState* __restrict__ st, const void* __restrict__ Gv, double4a* __restrict__ force,
                double* __restrict__ dq, double* __restrict__ dr, int tile_cap, int store) {
  typedef typename V4<R>::T R4;
  typedef typename std::conditional<MODE == 0, R4, R>::type GT;  // mesh element
  constexpr int LPA = gather_lanes(NO), NT = GATHER_ATOMS * LPA;
  extern __shared__ __align__(32) unsigned char g_smem[];
  GT* tile = reinterpret_cast<GT*>(g_smem);
  __shared__ int sbox[6];
  const int i0 = blockIdx.x * GATHER_ATOMS;
  const int i = i0 + (int)threadIdx.x / LPA, a = threadIdx.x & (LPA - 1);
  const bool act = i < N;
  const int K[3] = {K0, K1, K2};
  if (threadIdx.x < 6) sbox[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;
  R4 p;
  if (act) p = pos[i];
  else { p.x = R(0); p.y = R(0); p.z = R(0); p.w = R(0); }
  const R4 p0 = pos[i0];
  const R x[3] = {p.x, p.y, p.z}, x0[3] = {p0.x, p0.y, p0.z};
  int bb[3];
  R ff[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int r;
    R fr;
    grid_coord<R>(x[d], (R)st->Li[d], K[d], bb[d], ff[d]);
    grid_coord<R>(x0[d], (R)st->Li[d], K[d], r, fr);
    const int dv = bb[d] - r;
    if (2 * dv > K[d]) bb[d] -= K[d];
    else if (2 * dv < -K[d]) bb[d] += K[d];
  }
  // a neutral atom feels no force, but its potential is the adjoint's dE/dq
  const bool live = act && (MODE == 2 || p.w != R(0));
  __syncthreads();
  if (live && a == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      atomicMin(&sbox[d], bb[d]);
      atomicMax(&sbox[3 + d], bb[d]);
    }
  }
  R w0[NO], w1[NO], w2[NO], d0[NO], d1[NO], d2[NO];
  bsp_t<R, NO, MODE != 0>(ff[0], w0, d0);
  bsp_t<R, NO, MODE != 0>(ff[1], w1, d1);
  bsp_t<R, NO, MODE != 0>(ff[2], w2, d2);
  R wa = R(0), da = R(0);
#pragma unroll
  for (int j = 0; j < NO; ++j)
    if (j == a) { wa = w0[j]; da = d0[j]; }
  __syncthreads();
  if (sbox[0] > sbox[3]) {  // no charge in this block
    if (MODE != 2 && store && act && a == 0) force[i] = double4a{0.0, 0.0, 0.0, 0.0};
    return;
  }
  const int o0 = sbox[0] - (NO - 1), o1 = sbox[1] - (NO - 1), o2 = sbox[2] - (NO - 1);
  const long e0 = sbox[3] - o0 + 1, e1 = sbox[4] - o1 + 1, e2 = sbox[5] - o2 + 1;
  // odd plane stride: the lanes of an atom (one x plane each) then fall on
  // different shared-memory banks
  const long ps = (e1 * e2) | 1;
  const bool staged = e0 * ps <= tile_cap;
  const GT* Gm = reinterpret_cast<const GT*>(Gv);
  if (staged) {
    // one mesh row (e2 points along z) per warp pass, lanes along z
    // row (xx, y) = warp + k * (NT / 32), stepped without divisions
    const int nrow = (int)(e0 * e1), ie1 = (int)e1, ie2 = (int)e2, ips = (int)ps;
    constexpr int NWARP = NT >> 5;
    const int w0 = threadIdx.x >> 5;
    int y = w0 % ie1, xx = w0 / ie1;
    for (int row = w0; row < nrow; row += NWARP) {
      const size_t g = ((size_t)((o0 + xx) & (K0 - 1)) * K1 + ((o1 + y) & (K1 - 1))) * K2;
      GT* t = tile + xx * ips + y * ie2;
      for (int z = threadIdx.x & 31; z < ie2; z += 32) t[z] = Gm[g + ((o2 + z) & (K2 - 1))];
      y += NWARP;
      while (y >= ie1) { y -= ie1; ++xx; }
    }
    __syncthreads();
  }
  // the lane's order^2 points are summed in the working precision (FP64 for
  // the adjoint), the lanes in FP64
  typedef typename std::conditional<MODE == 2, double, R>::type A;
  A s0 = A(0), s1 = A(0), s2 = A(0), s3 = A(0);
  if (live && a < NO) {
    if (staged) {
      // row b of plane a starts at tp - b e2; point c of the row at -c
      const int ie2 = (int)e2;
      const GT* tp = tile + (bb[0] - a - o0) * (int)ps + (bb[1] - o1) * ie2 + (bb[2] - o2);
#pragma unroll
      for (int b = 0; b < NO; ++b)
        gather_row<R, NO, MODE>(tp - b * ie2, wa, da, w1[b], d1[b], w2, d2, s0, s1, s2, s3);
    } else {
      int kz[NO];
#pragma unroll
      for (int c = 0; c < NO; ++c) kz[c] = (bb[2] - c) & (K2 - 1);
      const size_t xrow = (size_t)((bb[0] - a) & (K0 - 1)) * K1;
#pragma unroll
      for (int b = 0; b < NO; ++b)
        gather_row_idx<R, NO, MODE>(Gm + (xrow + ((bb[1] - b) & (K1 - 1))) * K2, kz, wa, da, w1[b], d1[b], w2, d2,
                                    s0, s1, s2, s3);
    }
  }
  double F0 = s0, F1 = s1, F2 = s2, F3 = s3;
#pragma unroll
  for (int o = LPA / 2; o > 0; o >>= 1) {
    F0 += __shfl_xor_sync(0xffffffffu, F0, o);
    F1 += __shfl_xor_sync(0xffffffffu, F1, o);
    F2 += __shfl_xor_sync(0xffffffffu, F2, o);
    if (MODE == 2) F3 += __shfl_xor_sync(0xffffffffu, F3, o);
  }
  if (!act || a != 0) return;
  const double q = (double)p.w;
  if (MODE == 2) {
    const int o = id[i];  // results in the caller's atom order
    if (dq) dq[o] = F0;
    if (dr) {
      dr[3 * o] = q * F1 * K0 * st->Li[0];
      dr[3 * o + 1] = q * F2 * K1 * st->Li[1];
      dr[3 * o + 2] = q * F3 * K2 * st->Li[2];
    }
    return;
  }
  double4a f = {0.0, 0.0, 0.0, 0.0};
  if (!live) {
    if (store) force[i] = f;
    return;
  }
  if (!store) f = force[i];
  if (MODE == 0) {
    f.x += q * F0;
    f.y += q * F1;
    f.z += q * F2;
  } else {
    f.x += 2.0 * q * F0 * K0 * st->Li[0];
    f.y += 2.0 * q * F1 * K1 * st->Li[1];
    f.z += 2.0 * q * F2 * K2 * st->Li[2];
  }
  force[i] = f;
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
template <class R, int LOGN>
static const void* fftp_fn_n(int mode, int sign, int out4) {
  if (mode == 0) return (const void*)k_fftp<R, LOGN, 0, -1, 0>;
  if (mode == 1) return sign < 0 ? (const void*)k_fftp<R, LOGN, 1, -1, 0> : (const void*)k_fftp<R, LOGN, 1, 1, 0>;
  return out4 ? (const void*)k_fftp<R, LOGN, 2, 1, 1> : (const void*)k_fftp<R, LOGN, 2, 1, 0>;
}

// line lengths 4 .. 1024
#define FFT_LOGNS(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

template <class R>
static const void* fftp_fn(int logn, int mode, int sign, int out4) {
  switch (logn) {
#define FFT_CASE(L) case L: return fftp_fn_n<R, L>(mode, sign, out4);
    FFT_LOGNS(FFT_CASE)
#undef FFT_CASE
  }
  return nullptr;
}

template <class R>
static const void* fftx_fn(int logn, int method) {
  switch (logn) {
#define FFT_CASE(L) \
  case L: return method == 0 ? (const void*)k_fft_x_kspace<R, L, 0> : (const void*)k_fft_x_kspace<R, L, 1>;
    FFT_LOGNS(FFT_CASE)
#undef FFT_CASE
  }
  return nullptr;
}

template <class R>
static const void* spread_fn(int order) {
  switch (order) {
#define ORDER_CASE(NO) case NO: return (const void*)k_spme_spread_t<R, NO>;
    SPME_ORDERS(ORDER_CASE)
#undef ORDER_CASE
  }
  return nullptr;
}

template <class R>
static const void* gather_fn(int order, int mode) {
  switch (order) {
#define ORDER_CASE(NO)                                                                          \
  case NO:                                                                                      \
    return mode == 0 ? (const void*)k_spme_gather_t<R, NO, 0>                                   \
                     : (mode == 1 ? (const void*)k_spme_gather_t<R, NO, 1> : (const void*)k_spme_gather_t<R, NO, 2>);
    SPME_ORDERS(ORDER_CASE)
#undef ORDER_CASE
  }
  return nullptr;
}

static int ilog2i(int k) {
  int l = 0;
  while ((1 << l) < k) ++l;
  return l;
}
static int fft_lpb(int n) { return FFT_THREADS / (n >= 8 ? n / 8 : 1); }

// one transform pass: mode 0 R2C z, 1 C2C along `axis` (0 x, 1 y), 2 C2R z
// (out4: the three batches interleaved into Real4)
template <class R>
static int fft_launch(md_spme* s, Recorder* rec, const void* in, void* out, int mode, int axis, int sign, int batch,
                      int out4) {
  const int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2], K2h = s->K2h;
  int n;
  long nlines, stride = 1, inner = 1, outer = 0, in_bs = 0, out_bs = 0;
  if (mode == 0 || mode == 2) {
    axis = 2;
    n = K2; nlines = (long)K0 * K1;
    in_bs = (long)s->nhalf; out_bs = (long)s->nreal;
  } else if (axis == 1) {
    n = K1; nlines = (long)K0 * K2h; stride = K2h; inner = K2h; outer = (long)K1 * K2h;
    in_bs = out_bs = (long)s->nhalf;
  } else {
    n = K0; nlines = (long)K1 * K2h; stride = (long)K1 * K2h; inner = (long)K1 * K2h; outer = 0;
    in_bs = out_bs = (long)s->nhalf;
  }
  const int logn = ilog2i(n), lpb = fft_lpb(n);
  const size_t smem = fftp_smem<R>(logn, out4 ? 2 : 1);
  const long nlc = mode == 0 ? (nlines + 1) / 2 : nlines;  // R2C: two real lines per complex transform
  dim3 grid((unsigned)((nlc + lpb - 1) / lpb), out4 ? 1 : batch);
  const void* twg = s->tw[axis];
  void* a[] = {&in, &out, &twg, &nlines, &stride, &inner, &outer, &in_bs, &out_bs};
  return rec_launch(rec, fftp_fn<R>(logn, mode, sign, out4), grid, dim3(FFT_THREADS * (out4 ? 2 : 1)), smem, a);
}

// dynamic shared memory above the default 48 KB needs the opt-in attribute
static int smem_optin(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024) MD_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return MD_OK;
}

template <class R>
static int spme_prepare(md_spme* s) {
  typedef typename C2<R>::T T2;
  cudaStream_t str = s->sys->stream;
  // the real mesh starts cleared; every z pass clears it again after reading
  MD_CUDA(cudaMemsetAsync(s->Q, 0, sizeof(R) * s->nreal, str));
  MD_CUDA(cudaMalloc(&s->frec, sizeof(double4a) * s->sys->N));
  s->max_blocks = ceil_div((long)s->K[1] * s->K2h, fft_lpb(s->K[0]));
  MD_CUDA(cudaMalloc(&s->partials, sizeof(double) * 4 * s->max_blocks));
  const int nbm = s->K[0] + s->K[1] + s->K2h;
  MD_CUDA(cudaMalloc(&s->bm, sizeof(double) * nbm));
  k_spme_bmod<<<ceil_div(nbm, 256), 256, 0, str>>>(s->K[0], s->K[1], s->K[2], s->order, s->bm);
  MD_CHECK_LAUNCH("spme bmod");
  for (int d = 0; d < 3; ++d) {
    MD_CUDA(cudaMalloc(&s->tw[d], sizeof(T2) * s->K[d]));
    k_fft_twiddles<R><<<ceil_div(s->K[d], 256), 256, 0, str>>>(s->K[d], (T2*)s->tw[d]);
    MD_CHECK_LAUNCH("fft twiddles");
  }
  const int l0 = ilog2i(s->K[0]), l1 = ilog2i(s->K[1]), l2 = ilog2i(s->K[2]);
  if (int r = smem_optin(spread_fn<R>(s->order), SPREAD_TILE_BYTES)) return r;
  if (int r = smem_optin(fftp_fn<R>(l2, 0, -1, 0), fftp_smem<R>(l2, 1))) return r;
  if (int r = smem_optin(fftp_fn<R>(l2, 2, 1, 0), fftp_smem<R>(l2, 1))) return r;
  if (int r = smem_optin(fftp_fn<R>(l2, 2, 1, 1), fftp_smem<R>(l2, 2))) return r;
  for (int sg = -1; sg <= 1; sg += 2) {
    if (int r = smem_optin(fftp_fn<R>(l1, 1, sg, 0), fftp_smem<R>(l1, 1))) return r;
    if (int r = smem_optin(fftp_fn<R>(l0, 1, sg, 0), fftp_smem<R>(l0, 1))) return r;
  }
  if (int r = smem_optin(fftx_fn<R>(l0, s->method), fftx_smem<R>(l0, s->method))) return r;
  for (int m = 0; m < 3; ++m)
    if (int r = smem_optin(gather_fn<R>(s->order, m), GATHER_TILE_BYTES)) return r;
  return MD_OK;
}

// stored influence function psi, refreshed only when the box changed
// (adjoint and md_spme_get_influence; the force chain evaluates psi in its
// x pass)
template <class R>
static int influence_launch(md_spme* s, Recorder* rec) {
  int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2], n = s->order;
  R* psi = (R*)s->psi;
  DevState* st = s->sys->st;
  double beta = s->beta;
  {
    void* a[] = {&K0, &K1, &K2, &n, &beta, &st, &psi, &s->d_box_tab};
    if (int r = rec_launch(rec, (const void*)k_spme_influence<R>, dim3((unsigned)((s->nhalf + 255) / 256)),
                           dim3(256), 0, a)) return r;
  }
  void* a[] = {&st, &s->d_box_tab};
  return rec_launch(rec, (const void*)k_spme_box_tab, dim3(1), dim3(1), 0, a);
}

// charges onto the (cleared) real mesh
template <class R>
static int spread_launch(md_spme* s, Recorder* rec) {
  md_system* sys = s->sys;
  int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2], N = sys->N;
  R* Q = (R*)s->Q;
  DevState* st = sys->st;
  const void* pos = sys->pos;
  int cap = SPREAD_TILE_BYTES / (int)sizeof(R);
  void* a[] = {&N, &pos, &K0, &K1, &K2, &st, &Q, &cap};
  return rec_launch(rec, spread_fn<R>(s->order), dim3(ceil_div(N, SPREAD_ATOMS)), dim3(SPREAD_THREADS),
                    SPREAD_TILE_BYTES, a);
}

// spread and the forward transform along z (which clears the real mesh for
// the next spread), y and (with_x) x: C[0] = Q^ on the half spectrum.  Every
// launch goes through the recorder, so the chain is either run on the stream
// or recorded into the step graph of the simulation driver.
template <class R>
static int spme_forward_mesh(md_spme* s, Recorder* rec, bool with_x) {
  typedef typename C2<R>::T T2;
  R* Q = (R*)s->Q;
  T2* C = (T2*)s->C;
  if (int r = spread_launch<R>(s, rec)) return r;
  if (int r = fft_launch<R>(s, rec, Q, C, 0, 2, -1, 1, 0)) return r;
  if (int r = fft_launch<R>(s, rec, C, C, 1, 1, -1, 1, 0)) return r;
  if (with_x)
    if (int r = fft_launch<R>(s, rec, C, C, 1, 0, -1, 1, 0)) return r;
  return MD_OK;
}

template <class R>
static int gather_launch(md_spme* s, Recorder* rec, int mode, double* dq, double* dr, bool store) {
  md_system* sys = s->sys;
  int N = sys->N, K0 = s->K[0], K1 = s->K[1], K2 = s->K[2];
  const void* pos = sys->pos;
  const void* G = s->G;
  DevState* st = sys->st;
  const size_t el = mode == 0 ? sizeof(typename V4<R>::T) : sizeof(R);
  int cap = (int)(GATHER_TILE_BYTES / el);
  double4a* force = store ? s->frec : sys->force;
  int st_ = store ? 1 : 0;
  void* a[] = {&N, &pos, &sys->id, &K0, &K1, &K2, &st, &G, &force, &dq, &dr, &cap, &st_};
  return rec_launch(rec, gather_fn<R>(s->order, mode), dim3(ceil_div(N, GATHER_ATOMS)),
                    dim3(GATHER_ATOMS * gather_lanes(s->order)), GATHER_TILE_BYTES, a);
}

template <class R>
static int spme_run(md_spme* s, bool with_stats, Recorder* rec, bool concurrent) {
  typedef typename C2<R>::T T2;
  md_system* sys = s->sys;
  int K1 = s->K[1], K2 = s->K[2], method = s->method;
  T2* C = (T2*)s->C;
  DevState* st = sys->st;
  if (int r = spme_forward_mesh<R>(s, rec, false)) return r;
  const int l0 = ilog2i(s->K[0]);
  const int nb = ceil_div((long)K1 * s->K2h, fft_lpb(s->K[0]));
  if (with_stats && nb > s->max_blocks) { md_set_error("partials buffer too small for the mesh"); return MD_ERR_BADARG; }
  {
    double beta = s->beta;
    const void* twg = s->tw[0];
    int ws = with_stats ? 1 : 0, merge = concurrent ? 0 : 1;
    void* a[] = {&C, &twg, &s->bm, &K1, &K2, &beta, &st, &s->partials, &ws, &merge};
    if (int r = rec_launch(rec, fftx_fn<R>(l0, method), dim3(nb), dim3(FFT_THREADS * (method == 0 ? 2 : 1)),
                           fftx_smem<R>(l0, method), a)) return r;
  }
  const int nconv = method == 0 ? 3 : 1;
  T2* Cp = C + s->nhalf;
  if (int r = fft_launch<R>(s, rec, Cp, Cp, 1, 1, +1, nconv, 0)) return r;
  if (int r = fft_launch<R>(s, rec, Cp, s->G, 2, 2, +1, nconv, method == 0 ? 1 : 0)) return r;
  return gather_launch<R>(s, rec, method, nullptr, nullptr, concurrent);
}

bool spme_belongs_to(const md_spme* s, const md_system* sys) { return s && s->sys == sys; }

// the chain of one SPME force evaluation, recorded (driver) or launched
int spme_apply_impl(md_spme* s, bool with_stats, Recorder* rec, bool concurrent) {
  return s->sys->prec == MD_PREC_FP64 ? spme_run<double>(s, with_stats, rec, concurrent)
                                      : spme_run<float>(s, with_stats, rec, concurrent);
}

const double4a* spme_force_buffer(const md_spme* s) { return s->frec; }

// energy and gradient: recompute the mesh and its transform, influence
// multiply (energy, dE/dbeta, dE/dpsi), one inverse transform to Phi, gather
__global__ void k_adj_out(const DevState* st, double* energy, double* dbeta) {
  if (energy) *energy = st->scratch[0];
  if (dbeta) *dbeta = st->scratch[1];
}

// dev = true: energy, dq, dr, dbeta are device pointers the results are left
// in (no host copy, no wait); dpsi must then be NULL
template <class R>
static int spme_energy_grad(md_spme* s, double* energy, double* dq, double* dr, double* dbeta, double* dpsi,
                            bool dev = false) {
  typedef typename C2<R>::T T2;
  md_system* sys = s->sys;
  cudaStream_t st_ = sys->stream;
  const int K0 = s->K[0], K1 = s->K[1], K2 = s->K[2];
  T2* C = (T2*)s->C;
  const int nb = (int)((s->nhalf + 255) / 256);
  if (nb > sys->max_partial_blocks) { md_set_error("partials buffer too small for the mesh"); return MD_ERR_BADARG; }
  // device outputs: dq [N], dr [N][3], dpsi [nhalf] (FP64, caller's atom order)
  const size_t nq = dq ? (size_t)sys->N : 0, nr = dr ? 3 * (size_t)sys->N : 0, np = dpsi ? s->nhalf : 0;
  double* d = nullptr;
  if (!dev && nq + nr + np) MD_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * (nq + nr + np), st_));
  double* d_q = dev ? dq : (dq ? d : nullptr);
  double* d_r = dev ? dr : (dr ? d + nq : nullptr);
  double* d_p = dev ? nullptr : (dpsi ? d + nq + nr : nullptr);
  Recorder rec;
  rec.stream = st_;
  if (int r = influence_launch<R>(s, &rec)) return r;
  if (int r = spme_forward_mesh<R>(s, &rec, true)) return r;
  k_spme_adj_kspace<R><<<nb, 256, 0, st_>>>(K0, K1, K2, s->beta, (const R*)s->psi, C, s->nhalf, sys->st,
                                             sys->partials, d_p);
  MD_CHECK_LAUNCH("spme adjoint kspace");
  if (dq || dr) {
    T2* Cp = C + s->nhalf;
    if (int r = fft_launch<R>(s, &rec, Cp, Cp, 1, 0, +1, 1, 0)) return r;
    if (int r = fft_launch<R>(s, &rec, Cp, Cp, 1, 1, +1, 1, 0)) return r;
    if (int r = fft_launch<R>(s, &rec, Cp, s->G, 2, 2, +1, 1, 0)) return r;
    if (int r = gather_launch<R>(s, &rec, 2, d_q, d_r, false)) return r;
  }
  if (dev) {
    k_adj_out<<<1, 1, 0, st_>>>(sys->st, energy, dbeta);
    MD_CHECK_LAUNCH("spme adjoint out");
    return MD_OK;
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
  // G: ik Real4 per mesh point (the adjoint's single mesh fits as well)
  bool ok = cudaMalloc(&s->Q, rs * s->nreal) == cudaSuccess &&
            cudaMalloc(&s->C, 2 * rs * s->nhalf * 4) == cudaSuccess &&
            cudaMalloc(&s->G, sys->r4_size() * s->nreal) == cudaSuccess &&
            cudaMalloc(&s->psi, rs * s->nhalf) == cudaSuccess &&
            cudaMalloc(&s->d_box_tab, sizeof(double) * 3) == cudaSuccess &&
            cudaMemset(s->d_box_tab, 0, sizeof(double) * 3) == cudaSuccess;
  if (!ok) {
    md_cuda_fail(cudaGetLastError(), "md_spme_create");
    md_spme_destroy(s);
    return MD_ERR_CUDA;
  }
  if (int r = sys->prec == MD_PREC_FP64 ? spme_prepare<double>(s) : spme_prepare<float>(s)) {
    md_spme_destroy(s);
    return r;
  }
  *out = s;
  return MD_OK;
}

extern "C" int md_spme_destroy(md_spme* s) {
  if (!s) return MD_OK;
  void* p[] = {s->Q, s->C, s->G, s->psi, s->d_box_tab, s->tw[0], s->tw[1], s->tw[2], s->bm, s->frec, s->partials};
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

// the same with DEVICE outputs (energy and dE_dbeta one double each, dE_dq [N],
// dE_dr [N][3], caller's atom order), asynchronous on the system's stream
extern "C" int md_spme_energy_grad_device(md_spme* s, md_system* sys, double* energy, double* dE_dq, double* dE_dr,
                                          double* dE_dbeta) {
  if (!s || !sys || sys != s->sys) { md_set_error("md_spme_energy_grad_device: bad arguments"); return MD_ERR_BADARG; }
  return sys->prec == MD_PREC_FP64 ? spme_energy_grad<double>(s, energy, dE_dq, dE_dr, dE_dbeta, nullptr, true)
                                   : spme_energy_grad<float>(s, energy, dE_dq, dE_dr, dE_dbeta, nullptr, true);
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
  Recorder rec;
  rec.stream = sys->stream;
  if (int r = sys->prec == MD_PREC_FP64 ? influence_launch<double>(s, &rec) : influence_launch<float>(s, &rec))
    return r;
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

// the charge mesh of the current positions: spread onto the cleared mesh,
// copied out, and cleared again for the next force evaluation
extern "C" int md_spme_get_mesh(md_spme* s, double* Q) {
  if (!s || !Q) return MD_ERR_BADARG;
  md_system* sys = s->sys;
  Recorder rec;
  rec.stream = sys->stream;
  const bool f = sys->prec != MD_PREC_FP64;
  if (int r = f ? spread_launch<float>(s, &rec) : spread_launch<double>(s, &rec)) return r;
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * s->nreal, sys->stream));
  k_mesh_out<<<(unsigned)((s->nreal + 255) / 256), 256, 0, sys->stream>>>(
      s->nreal, f ? (const float*)s->Q : nullptr, f ? nullptr : (const double*)s->Q, d);
  MD_CHECK_LAUNCH("mesh out");
  MD_CUDA(cudaMemsetAsync(s->Q, 0, sys->real_size() * s->nreal, sys->stream));
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

