// Langevin integrator pieces shared by the integrator kernels and the
// non-bonded kernel that can close a step (the closing half kick fused into
// its epilogue).  Equations: langevin.npt/writedown/paper.tex:355-369,
// 382-440, 586-600 (see integrate.cu for the splitting).
#pragma once
#include <type_traits>
#include "device_common.cuh"

struct LvDev {
  double dt, kT, c1, c2, c1p, c2p, pref[3], skin_half2;
  int dirs;
  uint64_t seed;
};

// Start of a step, one thread: rebuild accounting and flag reset, step
// counter, and the box part of B(dt/2) A(dt/2) O(dt) A(dt/2).
__device__ __forceinline__ void box_commit(DevState* st) {
  if (!st->box_pending) return;
  for (int d = 0; d < 3; ++d) {
    st->L[d] = st->Lnext[d];
    st->Li[d] = 1.0 / st->Lnext[d];
    st->Lf[d] = (float)st->Lnext[d];
    st->Lif[d] = 1.0f / st->Lf[d];
  }
  st->box_pending = 0;
}

// commit = false: the new box waits in Lnext until the particles of the step
// are moved (k_lv_step1 commits it), so the box read between steps always
// matches the positions
// The box's normals of step s are those of Philox counter (s, 0xffffffff)
// under the seed with 0x5bd1e995 mixed in (box_normals).  xi_pre: the normals
// of the coming step computed ahead by another thread, or null to compute
// them here.
__device__ __forceinline__ void box_normals(const LvDev& p, unsigned long long step, double xi[4]) {
  normals4(p.seed ^ 0x5bd1e995ull, step, 0xffffffffu, xi);
}

__device__ __forceinline__ void box_advance(DevState* st, const LvDev& p, bool commit,
                                            const double* xi_pre = nullptr) {
  const unsigned f = st->flags;
  if (f & FLAG_REBUILD) st->rebuilds += 1ull;
  // a forced rebuild (new cutoff lattice) becomes this step's rebuild
  st->flags = (f & ~(FLAG_REBUILD | FLAG_FORCE_REBUILD)) | ((f & FLAG_FORCE_REBUILD) ? FLAG_REBUILD : 0u);
  st->step += 1ull;
  for (int d = 0; d < 3; ++d) { st->lam1[d] = 1.0; st->lam2[d] = 1.0; }
  if (!p.dirs) return;
  double xi[4];
  if (xi_pre) {
    for (int d = 0; d < 3; ++d) xi[d] = xi_pre[d];
  } else {
    box_normals(p, st->step, xi);
  }
  const double V = st->L[0] * st->L[1] * st->L[2];
  for (int d = 0; d < 3; ++d) st->Lnext[d] = st->L[d];
  for (int d = 0; d < 3; ++d) {
    if (!(p.dirs & (1 << d))) continue;
    const double A = V / st->L[d];
    double ph = st->ph[d];
    const double M = st->Mh[d];
    ph += 0.5 * p.dt * A * (st->Pcur[d] - p.pref[d]);            // B
    const double L0 = st->L[d];
    const double L1 = L0 + 0.5 * p.dt * ph / M;                  // A
    ph = p.c1p * ph + p.c2p * sqrt(M * p.kT) * xi[d];            // O
    const double L2 = L1 + 0.5 * p.dt * ph / M;                  // A
    st->lam1[d] = L1 / L0;
    st->lam2[d] = L2 / L1;
    st->ph[d] = ph;
    st->Lnext[d] = L2;
  }
  st->box_pending = 1;
  if (commit) box_commit(st);
}

// End of a step, one thread, after the kinetic and virial sums are stored:
// P_dd = 2/V (K_dd - W_dd/2) + tail correction (MDStatistic::pressureXX), the
// box momentum's closing half kick (kick) and, with advance, the box part of
// the next step's B A O A.
__device__ __forceinline__ void lv_close(DevState* st, const LvDev& p, int kick, int advance,
                                         const double* xi_pre = nullptr) {
  const double V = st->L[0] * st->L[1] * st->L[2];
  for (int d = 0; d < 3; ++d) {
    const double W = st->stats[MD_STAT_VIRIAL_XX + d];
    const double K = st->stats[MD_STAT_KINETIC_XX + d];
    st->Pcur[d] = 2.0 / V * (K - 0.5 * W) + st->stats[MD_STAT_PRESSURE_CORR_XX + d];
    if (kick && (p.dirs & (1 << d))) st->ph[d] += 0.5 * p.dt * V / st->L[d] * (st->Pcur[d] - p.pref[d]);
  }
  if (advance) box_advance(st, p, false, xi_pre);
}

// The mixed path's particle update in binary32 (FP64 stays for the
// reductions, the box and the error estimates): the same B A O A with the
// box factors and coefficients rounded to binary32, and its three normals
// from the same Philox block by Box-Muller in binary32 on 24-bit uniforms
// (u = (r >> 8) + 1/2) / 2^24, strictly inside (0, 1)).
__device__ __forceinline__ void lv_particle_step1_f32(int k, float4* __restrict__ pos, float4* __restrict__ vel,
                                                      const double4a* __restrict__ force,
                                                      const int* __restrict__ id,
                                                      const float4* __restrict__ backup, DevState* st,
                                                      const LvDev& p) {
  // every load first, so that the thread waits for memory once
  float4 x = pos[k], v = vel[k];
  const double4a f = force[k];
  const uint32_t aid = (uint32_t)id[k];
  const float4 b = backup ? backup[k] : make_float4(0.f, 0.f, 0.f, 0.f);
  const unsigned long long step = st->step;
  const float l1[3] = {(float)st->lam1[0], (float)st->lam1[1], (float)st->lam1[2]};
  const float l2[3] = {(float)st->lam2[0], (float)st->lam2[1], (float)st->lam2[2]};
  const double L[3] = {st->L[0], st->L[1], st->L[2]}, Li[3] = {st->Li[0], st->Li[1], st->Li[2]};
  const float im = v.w;
  const float h = (float)(0.5 * p.dt);
  float vx = v.x + h * (float)f.x * im, vy = v.y + h * (float)f.y * im, vz = v.z + h * (float)f.z * im;  // B
  // A
  x.x = l1[0] * x.x + h * vx; vx /= l1[0];
  x.y = l1[1] * x.y + h * vy; vy /= l1[1];
  x.z = l1[2] * x.z + h * vz; vz /= l1[2];
  // O
  float xi[3];
  {
    u32x4 c{aid, (uint32_t)step, (uint32_t)(step >> 32), 0x6d646672u};
    u32x4 r = philox4x32_10(c, (uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    const float inv = 5.9604644775390625e-8f;  // 2^-24
    const float u1 = ((float)(r.a >> 8) + 0.5f) * inv, u2 = ((float)(r.b >> 8) + 0.5f) * inv;
    const float u3 = ((float)(r.c >> 8) + 0.5f) * inv, u4 = ((float)(r.d >> 8) + 0.5f) * inv;
    const float m1 = sqrtf(-2.0f * logf(u1)), m2 = sqrtf(-2.0f * logf(u3));
    float s1, c1;
    sincospif(2.0f * u2, &s1, &c1);
    xi[0] = m1 * c1;
    xi[1] = m1 * s1;
    xi[2] = m2 * cospif(2.0f * u4);
  }
  const float c1 = (float)p.c1, sd = (float)p.c2 * sqrtf((float)p.kT * im);
  vx = c1 * vx + sd * xi[0];
  vy = c1 * vy + sd * xi[1];
  vz = c1 * vz + sd * xi[2];
  // A
  x.x = l2[0] * x.x + h * vx; vx /= l2[0];
  x.y = l2[1] * x.y + h * vy; vy /= l2[1];
  x.z = l2[2] * x.z + h * vz; vz /= l2[2];
  v.x = vx; v.y = vy; v.z = vz;
  pos[k] = x;
  vel[k] = v;
  // Displacement_max: rebuild when |r - r_backup| > skin/2
  if (backup) {
    const double dx = min_image_exact((double)x.x - (double)b.x, L[0], Li[0]);
    const double dy = min_image_exact((double)x.y - (double)b.y, L[1], Li[1]);
    const double dz = min_image_exact((double)x.z - (double)b.z, L[2], Li[2]);
    const double d2 = dx * dx + dy * dy + dz * dz;
    const bool far = d2 > p.skin_half2;
    const unsigned m = __ballot_sync(__activemask(), far);
    if (m && (int)(threadIdx.x & 31) == __ffs(m) - 1) atomicOr(&st->flags, FLAG_REBUILD);
  }
}

template <class R>
__device__ __forceinline__ void lv_particle_step1(int k, typename V4<R>::T* __restrict__ pos,
                                                  typename V4<R>::T* __restrict__ vel,
                                                  const double4a* __restrict__ force,
                                                  const int* __restrict__ id,
                                                  const typename V4<R>::T* __restrict__ backup,
                                                  DevState* st, const LvDev& p) {
  if constexpr (std::is_same<R, float>::value) {
    lv_particle_step1_f32(k, pos, vel, force, id, backup, st, p);
    return;
  }
  typedef typename V4<R>::T R4;
  // every load first, so that the thread waits for memory once
  R4 x = pos[k], v = vel[k];
  const double4a f = force[k];
  const uint32_t aid = (uint32_t)id[k];
  R4 b{};
  if (backup) b = backup[k];
  const unsigned long long step = st->step;
  const double l1[3] = {st->lam1[0], st->lam1[1], st->lam1[2]};
  const double l2[3] = {st->lam2[0], st->lam2[1], st->lam2[2]};
  const double L[3] = {st->L[0], st->L[1], st->L[2]}, Li[3] = {st->Li[0], st->Li[1], st->Li[2]};
  const double im = (double)v.w;
  const double h = 0.5 * p.dt;
  double vx = v.x + h * f.x * im, vy = v.y + h * f.y * im, vz = v.z + h * f.z * im;  // B
  double rx = x.x, ry = x.y, rz = x.z;
  // A
  rx = l1[0] * rx + h * vx; vx /= l1[0];
  ry = l1[1] * ry + h * vy; vy /= l1[1];
  rz = l1[2] * rz + h * vz; vz /= l1[2];
  // O
  double xi[4];
  normals4(p.seed, step, aid, xi);
  const double sd = p.c2 * sqrt(p.kT * im);
  vx = p.c1 * vx + sd * xi[0];
  vy = p.c1 * vy + sd * xi[1];
  vz = p.c1 * vz + sd * xi[2];
  // A
  rx = l2[0] * rx + h * vx; vx /= l2[0];
  ry = l2[1] * ry + h * vy; vy /= l2[1];
  rz = l2[2] * rz + h * vz; vz /= l2[2];
  x.x = (R)rx; x.y = (R)ry; x.z = (R)rz;
  v.x = (R)vx; v.y = (R)vy; v.z = (R)vz;
  pos[k] = x;
  vel[k] = v;
  // Displacement_max: rebuild when |r - r_backup| > skin/2
  if (backup) {
    const double dx = min_image_exact((double)x.x - (double)b.x, L[0], Li[0]);
    const double dy = min_image_exact((double)x.y - (double)b.y, L[1], Li[1]);
    const double dz = min_image_exact((double)x.z - (double)b.z, L[2], Li[2]);
    const double d2 = dx * dx + dy * dy + dz * dz;
    const bool far = d2 > p.skin_half2;
    const unsigned m = __ballot_sync(__activemask(), far);
    if (m && (int)(threadIdx.x & 31) == __ffs(m) - 1) atomicOr(&st->flags, FLAG_REBUILD);
  }
}

// integrator constants of the system's Langevin parameters (nl: list skin
// for the displacement test, or none)
LvDev make_lv(const md_system* sys, const md_nlist* nl);
