// Langevin integrator pieces shared by the integrator kernels and the
// non-bonded kernel that can close a step (the closing half kick fused into
// its epilogue).  Equations: langevin.npt/writedown/paper.tex:355-369,
// 382-440, 586-600 (see integrate.cu for the splitting).
#pragma once
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

// integrator constants of the system's Langevin parameters (nl: list skin
// for the displacement test, or none)
LvDev make_lv(const md_system* sys, const md_nlist* nl);
