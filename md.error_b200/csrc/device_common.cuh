// Device helpers: binary32 arithmetic without contraction (for the
// bit-exact cell / neighbour criteria), deterministic last-block
// reductions in FP64, and a counter-based normal generator.
#pragma once
#include "md_internal.cuh"

// ---- binary32 / binary64 arithmetic with no FMA contraction ------------
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float floor_r(float a) { return floorf(a); }
__device__ __forceinline__ double floor_r(double a) { return floor(a); }

// Box accessors in the working precision: binary32 uses the float copies
// (box.size / box.sizei of the reference), binary64 the double ones.
template <class R> __device__ __forceinline__ R boxL(const DevState* s, int d);
template <> __device__ __forceinline__ float boxL<float>(const DevState* s, int d) { return s->Lf[d]; }
template <> __device__ __forceinline__ double boxL<double>(const DevState* s, int d) { return s->L[d]; }
template <class R> __device__ __forceinline__ R boxLi(const DevState* s, int d);
template <> __device__ __forceinline__ float boxLi<float>(const DevState* s, int d) { return s->Lif[d]; }
template <> __device__ __forceinline__ double boxLi<double>(const DevState* s, int d) { return s->Li[d]; }

// shortestImage (ENG/include/BoxGeometry.h:176-179): x -= floorf(x*Li + 0.5)*L
template <class R>
__device__ __forceinline__ R min_image_exact(R x, R L, R Li) {
  R k = floor_r(add_rn(mul_rn(x, Li), R(0.5)));
  return sub_rn(x, mul_rn(k, L));
}

// ---- deterministic reductions ------------------------------------------
template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
}

// Block-reduce v (all threads participate, blockDim.x multiple of 32, <= 1024),
// thread 0 stores the block partial; the last block to finish sums the partials
// in block order (fixed, hence bit-reproducible) and adds them into out[k]
// (or stores when `store`).  `counter` is reset by the last block.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long atom_add_release_u64(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.add.release.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Barrier over every block of a cooperative launch (all blocks resident), on
// one 64-bit counter that each barrier advances by exactly GBAR_EPOCH: every
// block adds 1 with release semantics, block 0 adds GBAR_EPOCH - (blocks - 1),
// and each block waits (acquire loads) for the counter to pass the end of
// the epoch it arrived in.  The counter never needs a reset and stays aligned
// whatever the grid size.  A wait is bounded: past limit_ns (4 s by
// default) the block sets FLAG_TIMEOUT and the call returns false, and the
// caller leaves the kernel (the other blocks' waits then end the same way).
constexpr unsigned long long GBAR_EPOCH = 1ull << 20;  // above any grid size
__device__ __forceinline__ bool grid_barrier(DevState* st, unsigned long long limit_ns = 4000000000ull) {
  __shared__ int gb_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long inc = blockIdx.x == 0 ? GBAR_EPOCH - (gridDim.x - 1) : 1ull;
    const unsigned long long old = atom_add_release_u64(&st->gbar, inc);
    const unsigned long long target = (old & ~(GBAR_EPOCH - 1)) + GBAR_EPOCH;
    int ok = 1;
    const unsigned long long t0 = global_ns();
    while ((long long)(ld_acquire_u64(&st->gbar) - target) < 0) {
      if (global_ns() - t0 > limit_ns) {
        atomicOr(&st->flags, FLAG_TIMEOUT);
        ok = 0;
        break;
      }
    }
    gb_ok = ok;
  }
  __syncthreads();
  return gb_ok != 0;
}

template <int NV>
__device__ bool block_reduce_finish(double (&v)[NV], double* partials, unsigned* counter,
                                    double* out, bool store) {
  __shared__ double sh[32][NV];
  __shared__ bool am_last;
  warp_sum<NV>(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[wid][k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int w = 0; w < nw; ++w)
#pragma unroll
      for (int k = 0; k < NV; ++k) acc[k] += sh[w][k];
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(size_t)blockIdx.x * NV + k] = acc[k];
    // release: this block's partials before its count; acquire: the last
    // block sees every block's partials (its other threads through the
    // barrier below)
    const unsigned prev = atom_add_acq_rel_u32(counter, 1u);
    am_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[(size_t)b * NV + k]);
  warp_sum<NV>(acc);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[wid][k] = acc[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sh[w][k];
      if (store) out[k] = s; else out[k] += s;
    }
    *counter = 0u;  // read again by the next launch only
    return true;
  }
  return false;
}

// ---- Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) -----------------
struct u32x4 { uint32_t a, b, c, d; };
__device__ __forceinline__ void philox_round(u32x4& x, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  uint32_t hi0 = __umulhi(M0, x.a), lo0 = M0 * x.a;
  uint32_t hi1 = __umulhi(M1, x.c), lo1 = M1 * x.c;
  u32x4 y;
  y.a = hi1 ^ x.b ^ k0;
  y.b = lo1;
  y.c = hi0 ^ x.d ^ k1;
  y.d = lo0;
  x = y;
}
__device__ __forceinline__ u32x4 philox4x32_10(u32x4 ctr, uint32_t k0, uint32_t k1) {
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    philox_round(ctr, k0, k1);
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}
// four standard normals (Box-Muller on the two 32-bit pairs) in FP64, for
// the FP64 path (the mixed path draws from the same Philox block in binary32)
__device__ __forceinline__ void normals4(uint64_t seed, uint64_t step, uint32_t id, double out[4]) {
  u32x4 c{id, (uint32_t)step, (uint32_t)(step >> 32), 0x6d646672u};
  u32x4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double inv = 2.3283064365386963e-10;  // 2^-32
  double u1 = ((double)r.a + 0.5) * inv, u2 = ((double)r.b + 0.5) * inv;
  double u3 = ((double)r.c + 0.5) * inv, u4 = ((double)r.d + 0.5) * inv;
  double m1 = sqrt(-2.0 * log(u1)), m2 = sqrt(-2.0 * log(u3));
  double s1, c1, s2, c2;
  sincospi(2.0 * u2, &s1, &c1);
  sincospi(2.0 * u4, &s2, &c2);
  out[0] = m1 * c1; out[1] = m1 * s1; out[2] = m2 * c2; out[3] = m2 * s2;
}

template <class R> __device__ __forceinline__ typename V4<R>::T load4(const void* p, int i) {
  return reinterpret_cast<const typename V4<R>::T*>(p)[i];
}

// Packed binary32 pairs (sm_100 f32x2): one instruction applies the same
// round-to-nearest binary32 operation to both halves, so every half equals
// the scalar .rn result.
struct F2 {
  unsigned long long v;
};
__device__ __forceinline__ F2 f2(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_split(F2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ F2 f2_sub(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 f2_mul(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 f2_fma(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}
