// Adaptive-cutoff Lennard-Jones non-bonded forces.
// Reference: calNonBondedInteraction_neighbor, statistics variant
// (ENG/src/InteractionEngine_interface.cu:1204-1281), LennardJones6_12::forcePoten
// (ENG/include/NonBondedInteraction.h:867-893), InteractionEngine::
// applyNonBondedInteraction (ENG/src/InteractionEngine_interface.cu:317-380).
//
// G lanes share one atom i and stride through its list row; the pair test is
// the reference's binary32 |d|^2 < rcut_i^2 on the minimum-image vector
// (same rounding as the list criterion), so the interacting pair set is
// exactly the reference's.  Mixed precision: pair forces in FP32, each lane
// keeps Kahan-compensated FP32 partial sums, lanes are combined in FP64 by
// shuffles, the atom force is accumulated in FP64.  Energy and the diagonal
// virial (1/2 sum over the full list, as the reference's per-atom buffers)
// are block-reduced in FP64 and finished by the last block in a fixed order.
// The plain LJ case (one type, no charges) runs its pair arithmetic branch
// free, two entries per packed binary32 (f32x2) instruction, with the same
// binary32 criterion.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>
#include "device_common.cuh"

// LJ 6-12 parameters and the real-space Ewald splitting (EleDir::
// applyInteractionCalPotential, RE/src/EleDir.cpp:43-61):
//   E_ij = q_i q_j erfc(beta r)/r,  F_i = -q_i q_j (erfc(beta r)/r + 2 beta/sqrt(pi) e^{-beta^2 r^2}) / r^2 (r_j - r_i)
struct LJParams {
  float eps4f, sig2f, shiftf, betaf, cbf;
  double eps4, sig2, shift, beta, cb;  // cb = 2 beta / sqrt(pi)
};

// Build options of the mixed kernel (defaults are the measured best):
//   MD_LJ_PREFETCH  1: the plain LJ pass loads the next list line while the
//                   current one is processed
//   MD_LJ_ACC       0: per-lane Kahan-compensated FP32 sums of the per-pass batch
//                      sums; 1: the batch sums added in FP64
#ifndef MD_LJ_PREFETCH
#define MD_LJ_PREFETCH 1
#endif
#ifndef MD_LJ_ACC
#define MD_LJ_ACC 1
#endif
//   MD_LJ_LISTLD    list loads: 0 read-only path, 1 streaming (ld.cs),
//                   2 no L1 allocation, so L1 keeps the position gathers
//                   (each list line is read once per step)
#ifndef MD_LJ_LISTLD
#define MD_LJ_LISTLD 2
#endif
//   MD_LJ_PACKED    1: plain LJ (no charges, one type) through the branch-free
//                   pass with packed binary32 pair arithmetic
#ifndef MD_LJ_PACKED
#define MD_LJ_PACKED 1
#endif

__device__ __forceinline__ int4 load_list4(const int4* p) {
#if MD_LJ_LISTLD == 1
  return __ldcs(p);
#elif MD_LJ_LISTLD == 2
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
#else
  return __ldg(p);
#endif
}

struct Kahan {
#if MD_LJ_ACC == 1
  double s = 0.0;
  __device__ __forceinline__ void add(float x) { s += (double)x; }
  __device__ __forceinline__ double value() const { return s; }
#else
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
#endif
};

template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
  return v;
}

// long-range force correction of the atom (LFC: forcx[ii] += fsumx + fcx[ii],
// FCR/src/InteractionEngine_interface.cu:1118), added to the FP64 sum
__device__ __forceinline__ void add_correction(double4a& f, const double4a& c) {
  f.x += c.x;
  f.y += c.y;
  f.z += c.z;
}

// Typed pairs: the nbForcePoten dispatch of ENG/include/NonBondedInteraction.h:556-600
// over the pair's kind, two 4-vectors per type pair (A, B):
//   LJ 6-12   (1): A = (1, 4 eps, sigma^2, shift)
//                  F = 4 eps (6 s^6 - 12 s^12)/r^2 d,  E = 4 eps (s^12 - s^6) + shift
//   LJ 6-12 B (5): A = (5, eps, sigma^2, shift), B.x = rcut^2 (LennardJones6_12B::forcePoten, :1010-1031)
//                  F = -eps (12 s^12 - 12 s^6)/r^2 d,  E = eps (s^12 - 2 s^6 + shift), 0 beyond rcut
//   CosTail   (3): A = (3, eps, b, rc), B = (rcut, 1/wc, [wc == 0], 0) (CosTail::forcePoten, :1400-1440)
//                  r <= rc: the WCA-shaped core in b; rc < r < rcut: -eps cos^2(pi/2 (r - rc)/wc)
//   none      (0): no force, no energy (mdForceNULL)
// with d = r_j - r_i; the caller has already applied the per-atom cutoff.
template <class R, class V>
__device__ __forceinline__ R typed_pair(const V& A, const V& B, const V& C, R r2, R& e) {
  const int kind = (int)A.x;
  if (kind == 2 || kind == 6) {
    // LennardJones6_12_cap / _12B_cap (:1094-1135, :1271-1312): B = (rcut, cap, capR, pcapR);
    // constant force cap inside capR (a coincident pair takes none here)
    if (kind == 2 ? r2 >= B.x * B.x : r2 > B.x * B.x) { e = R(0); return R(0); }
    if (r2 == R(0)) { e = R(0); return R(0); }
    if (r2 < B.z * B.z) {
      const R s = R(1) / sqrt(r2);
      e = -B.y * (sqrt(r2) - B.z) + B.w;
      return -s * B.y;
    }
    const R ri2 = R(1) / r2, s2 = A.z * ri2, s6 = s2 * s2 * s2;
    if (kind == 2) {
      e = R(4) * A.y * (s6 * s6 - s6) + A.w;
      return -(R(4) * A.y * (R(12) * s6 * s6 - R(6) * s6) * ri2);
    }
    e = A.y * (s6 * s6 - R(2) * s6 + A.w);
    return -(A.y * (R(12) * s6 * s6 - R(12) * s6) * ri2);
  }
  if (kind == 4) {
    // CosTail_cap (:1532-1570): A = (4, eps, b, rc), B = (rcut, 1/wc, [wc == 0], 0),
    // C = (cap, capR, pcapR, 0)
    if (r2 == R(0)) { e = R(0); return R(0); }
    const R ri = R(1) / sqrt(r2);
    if (r2 < C.y * C.y) {
      e = -C.x * (sqrt(r2) - C.y) + C.z;
      return -ri * C.x;
    }
    if (r2 <= A.w * A.w) {
      const R sri = A.z * ri, sri2 = sri * sri, sri6 = sri2 * sri2 * sri2;
      e = R(4) * A.y * (sri6 * sri6 - sri6) + (B.z != R(0) ? A.y : R(0));
      return -R(24) * A.y * (R(2) * sri6 * sri6 - sri6) * ri * ri;
    }
    if (r2 < B.x * B.x) {
      const R pi_ = sizeof(R) == 4 ? R(3.14159265f) : R(M_PI);
      const R term = R(0.5) * pi_ * (r2 * ri - A.w) * B.y;
      const R c = cos(term);
      e = -A.y * c * c;
      return A.y * pi_ * B.y * c * sin(term) * ri;
    }
    e = R(0);
    return R(0);
  }
  if (kind == 1) {
    const R ri2 = R(1) / r2, s2 = A.z * ri2, s6 = s2 * s2 * s2;
    e = A.y * (s6 * s6 - s6) + A.w;
    return A.y * (R(6) * s6 - R(12) * s6 * s6) * ri2;
  }
  if (kind == 5) {
    if (r2 > B.x) { e = R(0); return R(0); }
    const R ri2 = R(1) / r2, s2 = A.z * ri2, s6 = s2 * s2 * s2;
    e = A.y * (s6 * s6 - s6 * R(2) + A.w);
    return -A.y * (R(12) * s6 * s6 - R(12) * s6) * ri2;
  }
  if (kind == 3) {
    const R ri = R(1) / sqrt(r2);
    if (r2 <= A.w * A.w) {
      const R sri = A.z * ri, sri2 = sri * sri, sri6 = sri2 * sri2 * sri2;
      e = R(4) * A.y * (sri6 * sri6 - sri6) + (B.z != R(0) ? A.y : R(0));
      return -R(24) * A.y * (R(2) * sri6 * sri6 - sri6) * ri * ri;
    }
    if (r2 < B.x * B.x) {
      const R pi_ = sizeof(R) == 4 ? R(3.14159265f) : R(M_PI);
      const R term = R(0.5) * pi_ * (r2 * ri - A.w) * B.y;
      const R c = cos(term);
      e = -A.y * c * c;
      return A.y * pi_ * B.y * c * sin(term) * ri;
    }
    e = R(0);
    return R(0);
  }
  e = R(0);
  return R(0);
}

// Statistics of the non-bonded kernels: each warp reduces its lanes' sums
// (shuffles in a fixed order) and lane 0 writes them as one row of
// rows[row][NV], row = warp index in the grid; k_rows_finish (a small grid),
// or in the driver the step's closing kick, sums the rows in a fixed order
// into the statistics slots.  A per-block reduction inside the force kernel
// needed a block barrier, a fence and an atomic per block and a last-block
// pass: 13 us of a 62 us launch on the 65,536-atom slab.
template <int NV>
__device__ __forceinline__ void warp_rows_out(double (&v)[NV], double* __restrict__ rows) {
  warp_sum<NV>(v);
  if ((threadIdx.x & 31) == 0) {
    const size_t r = (size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
#pragma unroll
    for (int k = 0; k < NV; ++k) rows[r * NV + k] = v[k];
  }
}

// The rows added up by a small grid: thread g sums rows g, g + G, ... (G the
// grid's threads), then the blocks combine by the deterministic last-block
// reduction; out[k] is stored (store) or added to.
template <int NV>
__global__ void __launch_bounds__(256) k_rows_finish(int nrows, const double* __restrict__ rows,
                                                     double* __restrict__ out, int store, double* partials,
                                                     unsigned* counter) {
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += rows[(size_t)r * NV + k];
  block_reduce_finish<NV>(acc, partials, counter, out, store != 0);
}

// ---------------------------------------------------------------- mixed
struct MixedAcc {
  Kahan fx, fy, fz;
  float e = 0.f, vx = 0.f, vy = 0.f, vz = 0.f, ec = 0.f;
};

// One pass of a lane over the 4 list entries e4 of row i (one 16-byte load;
// logical entries base + 8u): all position gathers, then the arithmetic, so
// that 4 independent loads are in flight per lane. TAIL: entry u is inside
// the row only when 8u < nvalid (only the last pass of a row).
// The image shift k L of an entry is read from the 64-entry table `shift`
// indexed by the entry's six image bits; the table holds the binary32
// products k_d * L_d (exactly -L_d, +0 or L_d), so d - shift is the same
// binary32 operation as shortestImage's x -= floorf(x/L + 0.5) L.
template <int U, bool TAIL, bool STATS, bool COUL, bool TYPES>
__device__ __forceinline__ void lj_pass_mixed(const int4 e4, int nvalid, const float4* __restrict__ pos, int i,
                                              const float4& pi, float rc2, const float4* shift,
                                              const LJParams& p, MixedAcc& a, const uint8_t* __restrict__ type,
                                              const float4* tab) {
  static_assert(U == 4, "one int4 of list entries per pass");
  int ee[U] = {e4.x, e4.y, e4.z, e4.w};
  float4 pj[U];
  if (TAIL) {
#pragma unroll
    for (int u = 0; u < U; ++u) ee[u] = 8 * u < nvalid ? ee[u] : -1;
  }
#pragma unroll
  // -1 marks "past the end" (a packed entry never has all six image bits set)
  for (int u = 0; u < U; ++u) pj[u] = __ldg(pos + ((!TAIL || ee[u] != -1) ? (ee[u] & 0x03FFFFFF) : i));
  // typed: the pair's (4 eps, sigma^2, shift) from the block's table row of
  // type i (tab points at that row); the j types gathered beside the positions
  int tj[U];
  if (TYPES) {
#pragma unroll
    for (int u = 0; u < U; ++u) tj[u] = __ldg(type + ((!TAIL || ee[u] != -1) ? (ee[u] & 0x03FFFFFF) : i));
  }
  // the U pair forces of this pass are summed in FP32, the pass sum is added
  // to the lane's Kahan-compensated accumulator
  float bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const float4 sh = shift[(unsigned)ee[u] >> 26];
    const float dx = __fsub_rn(__fsub_rn(pj[u].x, pi.x), sh.x);
    const float dy = __fsub_rn(__fsub_rn(pj[u].y, pi.y), sh.y);
    const float dz = __fsub_rn(__fsub_rn(pj[u].z, pi.z), sh.z);
    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if ((!TAIL || ee[u] != -1) && r2 < rc2) {
      const float ri2 = __fdividef(1.0f, r2);
      if (TYPES) {
        float ep = 0.f;
        float fs = typed_pair<float>(tab[3 * tj[u]], tab[3 * tj[u] + 1], tab[3 * tj[u] + 2], r2, ep);
        if (COUL) {
          const float qq = pi.w * pj[u].w;
          const float rinv = rsqrtf(r2);
          const float er = erfcf(p.betaf * r2 * rinv);
          fs -= qq * (er * rinv + p.cbf * __expf(-p.betaf * p.betaf * r2)) * ri2;
          if (STATS) a.ec += qq * er * rinv;
        }
        bx += fs * dx;
        by += fs * dy;
        bz += fs * dz;
        if (STATS) {
          a.e += ep;
          a.vx += fs * dx * dx;
          a.vy += fs * dy * dy;
          a.vz += fs * dz * dz;
        }
      } else {
        const float s2 = p.sig2f * ri2;
        const float s6 = s2 * s2 * s2;
        // 4 eps (6 s^6 - 12 s^12) / r^2 = (4 eps / r^2) s^6 (6 - 12 s^6)
        float fs = (p.eps4f * ri2) * s6 * fmaf(-12.f, s6, 6.f);
        if (COUL) {
          const float qq = pi.w * pj[u].w;
          const float rinv = rsqrtf(r2);
          const float er = erfcf(p.betaf * r2 * rinv);
          fs -= qq * (er * rinv + p.cbf * __expf(-p.betaf * p.betaf * r2)) * ri2;
          if (STATS) a.ec += qq * er * rinv;
        }
        bx += fs * dx;
        by += fs * dy;
        bz += fs * dz;
        if (STATS) {
          a.e += fmaf(p.eps4f, fmaf(s6, s6, -s6), p.shiftf);
          a.vx += fs * dx * dx;
          a.vy += fs * dy * dy;
          a.vz += fs * dz * dz;
        }
      }
    }
  }
  a.fx.add(bx);
  a.fy.add(by);
  a.fz.add(bz);
}

// Accumulators of the packed pass: energy as (pair, pair) halves without the
// shift, which is added once per interacting pair at the end (cnt); virial
// (xx, yy) packed and zz.
struct PackedAcc {
  Kahan fx, fy, fz;
  F2 e2 = {0ull}, vxy = {0ull};
  float vz = 0.f;
  int cnt = 0;
};

__device__ __forceinline__ void acc_stats(const MixedAcc& a, const LJParams&, float& e, float& vx, float& vy,
                                          float& vz, float& ec) {
  e = a.e; vx = a.vx; vy = a.vy; vz = a.vz; ec = a.ec;
}
__device__ __forceinline__ void acc_stats(const PackedAcc& a, const LJParams& p, float& e, float& vx, float& vy,
                                          float& vz, float& ec) {
  float e0, e1;
  f2_split(a.e2, e0, e1);
  e = fmaf((float)a.cnt, p.shiftf, e0 + e1);
  f2_split(a.vxy, vx, vy);
  vz = a.vz;
  ec = 0.f;
}

// Plain LJ 6-12 (no charges, one type) over the 4 entries of a pass, branch
// free: the criterion is the binary32 |d|^2 < rc_i^2 of lj_pass_mixed
// ((x_j - x_i) - k L per axis, (dx^2 + dy^2) + dz^2), computed with x and y
// packed; entries beyond rc_i (and past the row's end) continue with
// r^2 = 1e30, where s^6 = (sigma^2/r^2)^3 underflows to 0 and the pair adds
// exactly zero force, virial and energy.  The pair arithmetic of entries
// (0, 1) and (2, 3) runs packed.
template <bool TAIL, bool STATS>
__device__ __forceinline__ void lj_pass_packed(const int4 e4, int nvalid, const float4* __restrict__ pos, int i,
                                               const float4& pi, float rc2, const float4* shift,
                                               const LJParams& p, PackedAcc& a) {
  int ee[4] = {e4.x, e4.y, e4.z, e4.w};
  if (TAIL) {
#pragma unroll
    for (int u = 0; u < 4; ++u) ee[u] = 8 * u < nvalid ? ee[u] : -1;
  }
  float4 pj[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) pj[u] = __ldg(pos + ((!TAIL || ee[u] != -1) ? (ee[u] & 0x03FFFFFF) : i));
  const F2 pxy = f2(pi.x, pi.y);
  const F2 sig2 = f2(p.sig2f, p.sig2f), eps4 = f2(p.eps4f, p.eps4f);
  const F2 m12 = f2(-12.f, -12.f), six = f2(6.f, 6.f), mone = f2(-1.f, -1.f);
  float bx = 0.f, bz = 0.f, by = 0.f;
  F2 bxy = f2(0.f, 0.f);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    F2 dxy[2];
    float dz[2], r2m[2];
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const int u = 2 * h + v;
      const float4 sh = shift[(unsigned)ee[u] >> 26];
      dxy[v] = f2_sub(f2_sub(f2(pj[u].x, pj[u].y), pxy), f2(sh.x, sh.y));
      dz[v] = __fsub_rn(__fsub_rn(pj[u].z, pi.z), sh.z);
      float sx, sy;
      f2_split(f2_mul(dxy[v], dxy[v]), sx, sy);
      const float r2 = __fadd_rn(__fadd_rn(sx, sy), __fmul_rn(dz[v], dz[v]));
      const bool in = (!TAIL || ee[u] != -1) && r2 < rc2;
      r2m[v] = in ? r2 : 1e30f;
      if (STATS) a.cnt += in ? 1 : 0;
    }
    const F2 ri2 = f2(__fdividef(1.0f, r2m[0]), __fdividef(1.0f, r2m[1]));
    const F2 s2 = f2_mul(sig2, ri2);
    const F2 s6 = f2_mul(f2_mul(s2, s2), s2);
    // 4 eps (6 s^6 - 12 s^12) / r^2 = (4 eps / r^2) s^6 (6 - 12 s^6)
    const F2 fs = f2_mul(f2_mul(f2_mul(eps4, ri2), s6), f2_fma(m12, s6, six));
    float fs0, fs1;
    f2_split(fs, fs0, fs1);
    bxy = f2_fma(f2(fs0, fs0), dxy[0], bxy);
    bz = fmaf(fs0, dz[0], bz);
    bxy = f2_fma(f2(fs1, fs1), dxy[1], bxy);
    bz = fmaf(fs1, dz[1], bz);
    if (STATS) {
      // 4 eps (s^12 - s^6); the shift is added per interacting pair at the end;
      // (dx^2, dy^2) recomputed rather than kept live
      a.e2 = f2_fma(eps4, f2_fma(s6, s6, f2_mul(s6, mone)), a.e2);
      a.vxy = f2_fma(f2(fs0, fs0), f2_mul(dxy[0], dxy[0]), a.vxy);
      a.vz = fmaf(fs0, __fmul_rn(dz[0], dz[0]), a.vz);
      a.vxy = f2_fma(f2(fs1, fs1), f2_mul(dxy[1], dxy[1]), a.vxy);
      a.vz = fmaf(fs1, __fmul_rn(dz[1], dz[1]), a.vz);
    }
  }
  f2_split(bxy, bx, by);
  a.fx.add(bx);
  a.fy.add(by);
  a.fz.add(bz);
}

// threads per block of the non-bonded kernels, and the resident 256-thread
// blocks per SM the plain mixed kernel is compiled for (its register cap)
#ifndef MD_LJ_THREADS
#define MD_LJ_THREADS 256
#endif
#ifndef MD_LJ_MINB
#define MD_LJ_MINB 4
#endif

template <int G, bool STATS, bool COUL, bool TYPES>
__global__ void __launch_bounds__(MD_LJ_THREADS, ((COUL || TYPES) ? 4 : MD_LJ_MINB) * 256 / MD_LJ_THREADS)
k_lj_mixed(int N, const float4* __restrict__ pos, const float* __restrict__ rcut,
           const int* __restrict__ list, const int* __restrict__ nnb, int cap,
           const DevState* __restrict__ st, LJParams p, double4a* __restrict__ force, int overwrite,
           double* partials, unsigned* counter, double* stats, const double4a* __restrict__ corr,
           const int* __restrict__ id, const uint8_t* __restrict__ type, const void* __restrict__ ptab, int nt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / G;
  const int lane = t & (G - 1);
  // image shift table: entry c = (k_x+1) | (k_y+1) << 2 | (k_z+1) << 4
  __shared__ float4 shift[64];
  if (threadIdx.x < 64) {
    const unsigned c = threadIdx.x;
    shift[c] = make_float4(__fmul_rn((float)((int)(c & 3u) - 1), st->Lf[0]),
                           __fmul_rn((float)((int)((c >> 2) & 3u) - 1), st->Lf[1]),
                           __fmul_rn((float)((int)(c >> 4) - 1), st->Lf[2]), 0.f);
  }
  __shared__ float4 tab[TYPES ? 3 * MD_MAX_TYPES * MD_MAX_TYPES : 1];
  if (TYPES)
    for (int c = threadIdx.x; c < 3 * nt * nt; c += blockDim.x) tab[c] = reinterpret_cast<const float4*>(ptab)[c];
  __syncthreads();
  constexpr bool PACK = MD_LJ_PACKED && !COUL && !TYPES;
  typename std::conditional<PACK, PackedAcc, MixedAcc>::type a;
  if (i < N) {
    const float4 pi = pos[i];
    const float4* trow = TYPES ? tab + 3 * nt * (int)type[i] : tab;
    const float rc = rcut[i];
    const float rc2 = __fmul_rn(rc, rc);
    int n = nnb[i];
    n = n < cap ? n : cap;
    // row i as 16-byte vectors: pass q covers the 32-entry line q; with the
    // transposed line layout (nl_slot) the vector of lane l holds logical
    // entries 32q + l + 8u, u = 0..3, so for each u the 8 lanes gather 8
    // consecutive neighbours.  Rows hold whole lines (cap is a multiple of
    // 32), so every vector read stays inside the row.
    static_assert(G * 4 == 32, "8 lanes x 4 entries per pass");
    const int4* row4 = reinterpret_cast<const int4*>(list + (size_t)i * cap);
    const int npass = (n + 31) >> 5;
    // plain LJ: the next pass's vector is loaded before the current pass is
    // processed (the list comes from DRAM, the positions mostly from L1)
    constexpr bool PF = MD_LJ_PREFETCH && PACK;
    int4 nxt = make_int4(0, 0, 0, 0);
    if (PF && npass > 0) nxt = load_list4(row4 + lane);
    for (int q = 0; q < npass; ++q) {
      int4 cur;
      if constexpr (PF) {
        cur = nxt;
        if (q + 1 < npass) nxt = load_list4(row4 + (q + 1) * G + lane);
      } else {
        cur = load_list4(row4 + q * G + lane);
      }
      const int rem = n - (32 * q + lane);  // entry u is inside the row when 8u < rem
      if constexpr (PACK) {
        if (rem > 24) lj_pass_packed<false, STATS>(cur, rem, pos, i, pi, rc2, shift, p, a);
        else if (rem > 0) lj_pass_packed<true, STATS>(cur, rem, pos, i, pi, rc2, shift, p, a);
      } else {
        if (rem > 24) lj_pass_mixed<4, false, STATS, COUL, TYPES>(cur, rem, pos, i, pi, rc2, shift, p, a, type, trow);
        else if (rem > 0) lj_pass_mixed<4, true, STATS, COUL, TYPES>(cur, rem, pos, i, pi, rc2, shift, p, a, type, trow);
      }
    }
  }
  Kahan& fx = a.fx; Kahan& fy = a.fy; Kahan& fz = a.fz;
  float e, vx, vy, vz, ec;
  acc_stats(a, p, e, vx, vy, vz, ec);
  double Fx = group_sum<G>(fx.value()), Fy = group_sum<G>(fy.value()), Fz = group_sum<G>(fz.value());
  if (i < N && lane == 0) {
    double4a f = overwrite ? double4a{0, 0, 0, 0} : force[i];
    f.x += Fx; f.y += Fy; f.z += Fz;
    if (corr) add_correction(f, corr[id[i]]);
    force[i] = f;
  }
  if (STATS) {
    // one row of sums per warp; k_rows_finish, or the driver's closing kick,
    // adds the rows up into the slots NB_ENERGY, VIRIAL_XX..ZZ, ELEC_DIR
    // (stored by the first force term of a step, overwrite, added by later
    // terms)
    double v[5] = {0.5 * (double)e, 0.5 * (double)vx, 0.5 * (double)vy, 0.5 * (double)vz, 0.5 * (double)ec};
    warp_rows_out<5>(v, partials);
  }
}

// ---------------------------------------------------------------- FP64
template <int G, bool STATS, bool COUL, bool TYPES>
__global__ void __launch_bounds__(256)
k_lj_fp64(int N, const double4a* __restrict__ pos, const float* __restrict__ rcut,
          const int* __restrict__ list, const int* __restrict__ nnb, int cap,
          const DevState* __restrict__ st, LJParams p, double4a* __restrict__ force, int overwrite,
          double* partials, unsigned* counter, double* stats, const double4a* __restrict__ corr,
          const int* __restrict__ id, const uint8_t* __restrict__ type, const void* __restrict__ ptab, int nt) {
  __shared__ double4a tab[TYPES ? 3 * MD_MAX_TYPES * MD_MAX_TYPES : 1];
  if (TYPES) {
    const double4a* src = reinterpret_cast<const double4a*>(reinterpret_cast<const float4*>(ptab) +
                                                            3 * MD_MAX_TYPES * MD_MAX_TYPES);
    for (int c = threadIdx.x; c < 3 * nt * nt; c += blockDim.x) tab[c] = src[c];
    __syncthreads();
  }
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / G;
  const int lane = t & (G - 1);
  const double L0 = st->L[0], L1 = st->L[1], L2 = st->L[2];
  double fx = 0, fy = 0, fz = 0, e = 0, vx = 0, vy = 0, vz = 0, ec = 0;
  if (i < N) {
    const double4a pi = pos[i];
    const double rc = (double)rcut[i];
    const double rc2 = rc * rc;
    int n = nnb[i];
    n = n < cap ? n : cap;
    // transposed line layout (nl_slot): the 16-byte vector of lane l in line
    // q holds logical entries 32q + l + 8u, u = 0..3
    const int4* row4 = reinterpret_cast<const int4*>(list + (size_t)i * cap);
    constexpr int U = 4;
    static_assert(G * U == 32, "8 lanes x 4 entries per line");
    for (int k0 = lane; k0 < n; k0 += U * G) {
      int jj[U];
      double4a pq[U];
      const int4 e4 = __ldg(row4 + (k0 >> 5) * G + lane);
      const int ev[U] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int kk = k0 + u * G;
        jj[u] = kk < n ? ev[u] : -1;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) pq[u] = pos[jj[u] != -1 ? (jj[u] & 0x03FFFFFF) : i];
#pragma unroll
      for (int u = 0; u < U; ++u) {
      const double4a pj = pq[u];
      const unsigned code = (unsigned)jj[u] >> 26;
      const double kx = (double)((int)(code & 3u) - 1), ky = (double)((int)((code >> 2) & 3u) - 1),
                   kz = (double)((int)(code >> 4) - 1);
      const double dx = __dsub_rn(__dsub_rn(pj.x, pi.x), __dmul_rn(kx, L0));
      const double dy = __dsub_rn(__dsub_rn(pj.y, pi.y), __dmul_rn(ky, L1));
      const double dz = __dsub_rn(__dsub_rn(pj.z, pi.z), __dmul_rn(kz, L2));
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (jj[u] != -1 && r2 < rc2) {
        const double ri2 = 1.0 / r2;
        double fs, ep = 0.0;
        if (TYPES) {
          const int c = 3 * (nt * (int)type[i] + (int)type[jj[u] & 0x03FFFFFF]);
          fs = typed_pair<double>(tab[c], tab[c + 1], tab[c + 2], r2, ep);
        } else {
          const double s2 = p.sig2 * ri2;
          const double s6 = s2 * s2 * s2;
          fs = p.eps4 * (6.0 * s6 - 12.0 * s6 * s6) * ri2;
          ep = p.eps4 * (s6 * s6 - s6) + p.shift;
        }
        if (COUL) {
          const double qq = pi.w * pj.w;
          const double r = sqrt(r2);
          const double er = erfc(p.beta * r);
          fs -= qq * (er / r + p.cb * exp(-p.beta * p.beta * r2)) * ri2;
          if (STATS) ec += qq * er / r;
        }
        fx += fs * dx;
        fy += fs * dy;
        fz += fs * dz;
        if (STATS) {
          e += ep;
          vx += fs * dx * dx;
          vy += fs * dy * dy;
          vz += fs * dz * dz;
        }
      }
      }
    }
  }
  double Fx = group_sum<G>(fx), Fy = group_sum<G>(fy), Fz = group_sum<G>(fz);
  if (i < N && lane == 0) {
    double4a f = overwrite ? double4a{0, 0, 0, 0} : force[i];
    f.x += Fx; f.y += Fy; f.z += Fz;
    if (corr) add_correction(f, corr[id[i]]);
    force[i] = f;
  }
  if (STATS) {
    double v[5] = {0.5 * e, 0.5 * vx, 0.5 * vy, 0.5 * vz, 0.5 * ec};
    warp_rows_out<5>(v, partials);
  }
}

__global__ void k_clear_force(int N, double4a* f) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) f[k] = double4a{0, 0, 0, 0};
}

static const int kLanes = 8;

// lj6_12_findCapR / lj6_12B_findCapR and the potential there (ENG/include/
// NonBondedInteraction.h:1027-1073, :1204-1250): step the radius down by 0.95
// from 0.95 rcut until the unbounded force reaches the cap, then bisect to
// 1e-4; in the table's precision T
template <class T>
static T cap_force(bool bform, T eps, T sig, T rcut, T r) {
  const T dr2 = r * r;
  if (bform ? dr2 > rcut * rcut : dr2 >= rcut * rcut) return T(0);
  const T ri = T(1) / r, ri2 = ri * ri, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
  return bform ? eps * (T(12) * sri6 * sri6 - T(12) * sri6) * ri : T(4) * eps * (T(12) * sri6 * sri6 - T(6) * sri6) * ri;
}

template <class T>
static void cap_radius(bool bform, T eps, T sig, T shift, T rcut, T cap, T& capR, T& pcapR) {
  T point = T(0.95) * rcut;
  for (int it = 0; it < 4096 && cap_force<T>(bform, eps, sig, rcut, point) < cap; ++it) point *= T(0.95);
  T lower = point, upper = rcut;
  for (int it = 0; it < 200 && std::fabs(upper - lower) > 1e-4; ++it) {
    const T mid = T(0.5) * (upper + lower);
    if (cap_force<T>(bform, eps, sig, rcut, mid) > cap) lower = mid;
    else upper = mid;
  }
  capR = T(0.5) * (upper + lower);
  const T dr2 = capR * capR;
  if (bform ? dr2 > rcut * rcut : dr2 >= rcut * rcut) { pcapR = T(0); return; }
  const T ri = T(1) / capR, ri2 = ri * ri, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
  pcapR = bform ? eps * (sri6 * sri6 - T(2) * sri6 + shift) : T(4) * eps * (sri6 * sri6 - sri6) + shift;
}

// finish_stats = false: the statistics stay as rows in sys->nb_rows for the
// step's closing kick to add up (lj_stat_rows rows)
int lj_apply_impl(md_engine* eng, md_system* sys, md_nlist* nl, bool with_stats, bool overwrite,
                  Recorder* rec, bool finish_stats) {
  if (!eng->has_lj) { md_set_error("no non-bonded interaction registered"); return MD_ERR_BADARG; }
  LJParams p;
  p.eps4 = 4.0 * eng->eps;
  p.sig2 = eng->sigma * eng->sigma;
  p.shift = eng->shift;
  p.eps4f = (float)p.eps4;
  p.sig2f = (float)p.sig2;
  p.shiftf = (float)p.shift;
  p.beta = eng->beta;
  p.cb = 2.0 * eng->beta / sqrt(M_PI);
  p.betaf = (float)p.beta;
  p.cbf = (float)p.cb;
  const bool coul = eng->has_coul;
  int N = sys->N;
  int cap = nl->cap;
  if (cap % 32 != 0) { md_set_error("neighbour-list capacity %d is not a multiple of 32", cap); return MD_ERR_BADARG; }
  int ow = overwrite ? 1 : 0;
  const int threads = MD_LJ_THREADS;
  dim3 grid(ceil_div((long long)N * kLanes, threads));
  // one row of 5 statistics per warp in sys->nb_rows
  if ((long long)grid.x * (threads / 32) > (long long)N / 4 + 1024) {
    md_set_error("statistics rows buffer too small");
    return MD_ERR_BADARG;
  }
  DevState* st = sys->st;
  unsigned* counter = &st->red_counter[RED_LJ];
  double* stats = &st->stats[MD_STAT_NB_ENERGY];
  const double4a* corr = fcorr_values(eng->fcorr);
  // typed pairs: the (4 eps, sigma^2, shift) table, binary32 then binary64 rows
  const bool typed = eng->nt > 0;
  int nt = eng->nt;
  if (typed) {
    if (sys->ntypes > nt) {
      md_set_error("the system has atom types up to %d, the interaction table covers %d", sys->ntypes - 1, nt);
      return MD_ERR_BADARG;
    }
    if (eng->tab_dirty || !eng->d_tab) {
      const size_t nf = 3 * MD_MAX_TYPES * MD_MAX_TYPES;
      if (!eng->d_tab) MD_CUDA(cudaMalloc(&eng->d_tab, nf * (sizeof(float4) + sizeof(double4a))));
      std::vector<float4> tf(nf, make_float4(0.f, 0.f, 0.f, 0.f));
      std::vector<double4a> td(nf, double4a{0, 0, 0, 0});
      for (int a0 = 0; a0 < nt; ++a0)
        for (int a1 = 0; a1 < nt; ++a1) {
          const double* q = eng->nb_param[a0][a1];
          const size_t c = 3 * (size_t)(a0 * nt + a1);
          // derived parameters as the *Parameter::reinit of each kind forms them,
          // in binary32 for the mixed table and binary64 for the FP64 one
          switch (eng->nb_kind[a0][a1]) {
            case MD_NB_LJ6_12: {
              const float sf = (float)q[1];
              tf[c] = make_float4(1.f, 4.f * (float)q[0], sf * sf, (float)q[2]);
              td[c] = double4a{1.0, 4.0 * q[0], q[1] * q[1], q[2]};
              break;
            }
            case MD_NB_LJ6_12B: {
              const float sf = (float)q[1], rf = (float)q[3];
              tf[c] = make_float4(5.f, (float)q[0], sf * sf, (float)q[2]);
              tf[c + 1] = make_float4(rf * rf, 0.f, 0.f, 0.f);
              td[c] = double4a{5.0, q[0], q[1] * q[1], q[2]};
              td[c + 1] = double4a{q[3] * q[3], 0, 0, 0};
              break;
            }
            case MD_NB_COSTAIL: {
              const float ef = (float)q[0], bf = (float)q[1], wf = (float)q[2];
              const float rcf = bf * powf(2.f, 1.f / 6.f);
              tf[c] = make_float4(3.f, ef, bf, rcf);
              tf[c + 1] = make_float4(rcf + wf, wf != 0.f ? 1.f / wf : 0.f, wf == 0.f ? 1.f : 0.f, 0.f);
              const double rcd = q[1] * pow(2.0, 1.0 / 6.0);
              td[c] = double4a{3.0, q[0], q[1], rcd};
              td[c + 1] = double4a{rcd + q[2], q[2] != 0 ? 1.0 / q[2] : 0.0, q[2] == 0 ? 1.0 : 0.0, 0};
              break;
            }
            case MD_NB_LJ6_12_CAP:
            case MD_NB_LJ6_12B_CAP: {
              const bool bform = eng->nb_kind[a0][a1] == MD_NB_LJ6_12B_CAP;
              const float kf = bform ? 6.f : 2.f;
              const float sf = (float)q[1], rcf = (float)q[3], capf = (float)q[4];
              float Rf, Pf;
              cap_radius<float>(bform, (float)q[0], sf, (float)q[2], rcf, capf, Rf, Pf);
              tf[c] = make_float4(kf, (float)q[0], sf * sf, (float)q[2]);
              tf[c + 1] = make_float4(rcf, capf, Rf, Pf);
              double Rd, Pd;
              cap_radius<double>(bform, q[0], q[1], q[2], q[3], q[4], Rd, Pd);
              td[c] = double4a{(double)kf, q[0], q[1] * q[1], q[2]};
              td[c + 1] = double4a{q[3], q[4], Rd, Pd};
              break;
            }
            case MD_NB_COSTAIL_CAP: {
              // CosTail_cap::initParameter: the cap radius of LJ 6-12 (eps, b, shift 0,
              // rcut rc) with the same cap
              const float ef = (float)q[0], bf = (float)q[1], wf = (float)q[2], capf = (float)q[3];
              const float rcf = bf * powf(2.f, 1.f / 6.f);
              float Rf, Pf;
              cap_radius<float>(false, ef, bf, 0.f, rcf, capf, Rf, Pf);
              tf[c] = make_float4(4.f, ef, bf, rcf);
              tf[c + 1] = make_float4(rcf + wf, wf != 0.f ? 1.f / wf : 0.f, wf == 0.f ? 1.f : 0.f, 0.f);
              tf[c + 2] = make_float4(capf, Rf, Pf, 0.f);
              const double rcd = q[1] * pow(2.0, 1.0 / 6.0);
              double Rd, Pd;
              cap_radius<double>(false, q[0], q[1], 0.0, rcd, q[3], Rd, Pd);
              td[c] = double4a{4.0, q[0], q[1], rcd};
              td[c + 1] = double4a{rcd + q[2], q[2] != 0 ? 1.0 / q[2] : 0.0, q[2] == 0 ? 1.0 : 0.0, 0};
              td[c + 2] = double4a{q[3], Rd, Pd, 0};
              break;
            }
            default: break;  // kind 0: no interaction
          }
        }
      MD_CUDA(cudaMemcpy(eng->d_tab, tf.data(), nf * sizeof(float4), cudaMemcpyHostToDevice));
      MD_CUDA(cudaMemcpy(reinterpret_cast<char*>(eng->d_tab) + nf * sizeof(float4), td.data(),
                         nf * sizeof(double4a), cudaMemcpyHostToDevice));
      eng->tab_dirty = false;
    }
  }
  const uint8_t* type = sys->type;
  const void* ptab = eng->d_tab;
  void* a[] = {&N, &sys->pos, &sys->rcut, &nl->list, &nl->nnb, &cap, &st, &p, &sys->force, &ow,
               &sys->nb_rows, &counter, &stats, &corr, &sys->id, &type, &ptab, &nt};
  const void* f;
#define LJ_PICK(K, T)                                                                       \
  (coul ? (with_stats ? (const void*)K<kLanes, true, true, T> : (const void*)K<kLanes, false, true, T>) \
        : (with_stats ? (const void*)K<kLanes, true, false, T> : (const void*)K<kLanes, false, false, T>))
  if (sys->prec == MD_PREC_FP64) f = typed ? LJ_PICK(k_lj_fp64, true) : LJ_PICK(k_lj_fp64, false);
  else f = typed ? LJ_PICK(k_lj_mixed, true) : LJ_PICK(k_lj_mixed, false);
#undef LJ_PICK
  if (int r = rec_launch(rec, f, grid, dim3(threads), 0, a)) return r;
  if (!with_stats || !finish_stats) return MD_OK;
  int nrows = (int)grid.x * (threads / 32);
  void* b[] = {&nrows, &sys->nb_rows, &stats, &ow, &sys->partials, &counter};
  return rec_launch(rec, (const void*)k_rows_finish<5>, dim3(std::min(64, ceil_div(nrows, 256))), dim3(256), 0, b);
}

int lj_stat_rows(const md_system* sys) {
  return ceil_div((long long)sys->N * kLanes, MD_LJ_THREADS) * (MD_LJ_THREADS / 32);
}

// ElectrostaticInteraction_dir: real-space Ewald with splitting beta inside the
// non-bonded kernel (same list and per-atom cutoff as the LJ term)
extern "C" int md_engine_register_coulomb(md_engine* e, double beta) {
  if (!e || !(beta > 0)) { md_set_error("md_engine_register_coulomb: bad arguments"); return MD_ERR_BADARG; }
  e->has_coul = true;
  e->beta = beta;
  return MD_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int md_engine_create(md_engine** out, md_system* sys) {
  if (!out || !sys) { md_set_error("md_engine_create: bad arguments"); return MD_ERR_BADARG; }
  md_engine* e = new md_engine();
  e->sys = sys;
  *out = e;
  return MD_OK;
}

extern "C" int md_engine_destroy(md_engine* e) {
  if (e && e->d_tab) cudaFree(e->d_tab);
  delete e;
  return MD_OK;
}

// SystemNonBondedInteraction::add(type0, type1, LennardJones6_12Parameter(eps, sigma, shift, rc))
// with AtomNBForceTable::calForceIndex (ENG/include/NonBondedInteraction.h:673-683): one
// parameter set per unordered type pair; pairs never given interact with nothing
// (mdForceNULL).  The cutoff stays the per-atom rcut_i.
extern "C" int md_engine_register_nb_pair(md_engine* e, int t0, int t1, int kind, const double* param) {
  if (!e || !param || t0 < 0 || t1 < 0 || t0 >= MD_MAX_TYPES || t1 >= MD_MAX_TYPES) {
    md_set_error("md_engine_register_nb_pair: bad arguments (types 0..%d)", MD_MAX_TYPES - 1);
    return MD_ERR_BADARG;
  }
  bool ok = param[0] >= 0;
  for (int c = 0; c < 6; ++c) ok = ok && std::isfinite(param[c]);
  if (kind == MD_NB_LJ6_12) ok = ok && param[1] > 0;
  else if (kind == MD_NB_LJ6_12B) ok = ok && param[1] > 0 && param[3] > 0;
  else if (kind == MD_NB_COSTAIL) ok = ok && param[1] > 0 && param[2] >= 0;
  else if (kind == MD_NB_LJ6_12_CAP || kind == MD_NB_LJ6_12B_CAP)
    ok = ok && param[0] > 0 && param[1] > 0 && param[3] > 0 && param[4] > 0;
  else if (kind == MD_NB_COSTAIL_CAP) ok = ok && param[0] > 0 && param[1] > 0 && param[2] >= 0 && param[3] > 0;
  else if (kind != MD_NB_NULL) ok = false;
  if (!ok) {
    md_set_error("md_engine_register_nb_pair: kind %d or its parameters out of range", kind);
    return MD_ERR_BADARG;
  }
  for (int k = 0; k < 2; ++k) {
    const int a = k ? t1 : t0, b = k ? t0 : t1;
    for (int c = 0; c < 6; ++c) e->nb_param[a][b][c] = param[c];
    e->nb_kind[a][b] = kind;
  }
  const int need = (t0 > t1 ? t0 : t1) + 1;
  if (need > e->nt) e->nt = need;
  e->has_lj = true;
  e->tab_dirty = true;
  if (e->sys) e->sys->topo_version += 1;  // a recorded step graph picks the typed kernel up
  return MD_OK;
}

extern "C" int md_engine_register_lj_pair(md_engine* e, int t0, int t1, double eps, double sigma, double shift) {
  const double q[6] = {eps, sigma, shift, 0.0, 0.0, 0.0};
  return md_engine_register_nb_pair(e, t0, t1, MD_NB_LJ6_12, q);
}

extern "C" int md_engine_register_lj(md_engine* e, double eps, double sigma, double shift) {
  if (!e || !(eps >= 0) || !(sigma > 0) || !std::isfinite(shift)) { md_set_error("md_engine_register_lj: bad arguments"); return MD_ERR_BADARG; }
  e->has_lj = true;
  e->eps = eps;
  e->sigma = sigma;
  e->shift = shift;
  return MD_OK;
}

extern "C" int md_engine_set_force_correction(md_engine* e, md_fcorr* fc) {
  if (!e) return MD_ERR_BADARG;
  e->fcorr = fc;
  return MD_OK;
}

extern "C" int md_engine_register_bonded(md_engine* e, int n_bonds) {
  if (!e || n_bonds < 0) return MD_ERR_BADARG;
  if (n_bonds != e->n_bonds) {
    md_set_error("registBondedInteraction: %d bonds expected, %d given to md_engine_set_bonds", n_bonds,
                 e->n_bonds);
    return MD_ERR_BADARG;
  }
  return MD_OK;
}

extern "C" int md_engine_clear_forces(md_engine* e, md_system* sys) {
  if (!e || !sys) return MD_ERR_BADARG;
  k_clear_force<<<ceil_div(sys->N, 256), 256, 0, sys->stream>>>(sys->N, sys->force);
  MD_CHECK_LAUNCH("clear force");
  return MD_OK;
}

extern "C" int md_engine_apply_nonbonded(md_engine* e, md_system* sys, md_nlist* nl, int with_stats) {
  if (!e || !sys || !nl || with_stats < 0 || with_stats > 2) return MD_ERR_BADARG;
  if (!nl->built) { md_set_error("neighbour list not built"); return MD_ERR_BADARG; }
  Recorder rec;
  rec.stream = sys->stream;
  return lj_apply_impl(e, sys, nl, with_stats != 0, false, &rec, with_stats != 2);
}

extern "C" int md_engine_finish_nonbonded_stats(md_engine* e, md_system* sys) {
  if (!e || !sys) return MD_ERR_BADARG;
  int nrows = lj_stat_rows(sys);
  double* stats = &sys->st->stats[MD_STAT_NB_ENERGY];
  unsigned* counter = &sys->st->red_counter[RED_LJ];
  int store = 0;
  k_rows_finish<5><<<std::min(64, ceil_div(nrows, 256)), 256, 0, sys->stream>>>(nrows, sys->nb_rows, stats, store,
                                                                                 sys->partials, counter);
  MD_CHECK_LAUNCH("non-bonded statistics");
  return MD_OK;
}
