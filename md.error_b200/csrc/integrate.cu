// Integrators: velocity Verlet and Langevin NVT / NPT (BAOAB splitting).
// Reference: velocityVerlet_part1/part2 (ENG/src/Integrator.cu:273-436);
// Langevin equations of motion, langevin.npt/writedown/paper.tex:355-369
// (isotropic), :382-440 (choice of M and gamma_P), :586-600 (anisotropic box).
//
// Box-length Langevin piston for the directions d in npt_dirs (x and y fixed
// for the slab, z free with target P_zz):
//   dL_d/dt = p_d / M_d
//   dp_d/dt = A_d (P_dd - P_ref) - gamma_P p_d + sqrt(2 kT gamma_P M_d) W'
// with A_d = V / L_d (det h h^-T in paper.tex:586-600), and for the particles
//   dr_d/dt = p_d/m + (dL_d/dt / L_d) r_d,  dp_d/dt = F_d - (dL_d/dt / L_d) p_d - gamma_T p_d + noise.
// For fixed box velocity over a sub-step h the drift is solved exactly:
//   L' = L + h v_L, lambda = L'/L, r_d' = lambda r_d + h p_d/m, p_d' = p_d/lambda.
// One step: B(dt/2) A(dt/2) O(dt) A(dt/2) | forces | B(dt/2).  The box part of
// B/A/O runs in a one-thread kernel before the particle update; the closing
// box half kick runs in the last block of the closing particle kick, with
// the pressure computed there from the FP64 kinetic and virial sums.
#include <cmath>
#include <cstring>
#include <type_traits>
#include "langevin.cuh"

__global__ void k_lv_box(DevState* st, LvDev p) { box_advance(st, p, true); }

// Particle part of B(dt/2) A(dt/2) O(dt) A(dt/2) and the rebuild test
// (lv_particle_step1, langevin.cuh).  With use_cond the last block to finish
// writes the rebuild decision into the CUDA graph conditional that guards the
// cell sort + list build.
// threads per block of the Langevin halves the driver launches as separate
// kernels (a multiple of 32, <= 256): with the closing kick's reduction on
// one acquire-release atomic per block, 256 measured 0.7 % more steps/s than
// 128 on the 65,536-atom slab (half the blocks, partials and atomics)
#ifndef MD_LV_THREADS
#define MD_LV_THREADS 256
#endif

template <class R>
__global__ void __launch_bounds__(256)
k_lv_step1(int N, typename V4<R>::T* __restrict__ pos, typename V4<R>::T* __restrict__ vel,
           const double4a* __restrict__ force, const int* __restrict__ id,
           const typename V4<R>::T* __restrict__ backup, DevState* st, LvDev p,
           cudaGraphConditionalHandle cond, int use_cond) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) lv_particle_step1<R>(k, pos, vel, force, id, backup, st, p);
  // the last block to finish (every other block is done reading the box)
  // commits the box of this step and hands the rebuild decision to the graph
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&st->red_counter[RED_DISP], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    box_commit(st);
    const unsigned f = atomicOr(&st->flags, 0u);
    if (use_cond) cudaGraphSetConditional(cond, (f & FLAG_REBUILD) ? 1u : 0u);
    st->red_counter[RED_DISP] = 0u;
    __threadfence();
  }
}

// Closing B(dt/2) (kick = 0: no kick, used to prime the pressure), kinetic
// tensor; the last block computes P, gives the box momentum its half kick
// (with_box) and, with advance, runs box_advance for the next step.
// With nb_rows, the non-bonded kernel's statistics rows (one row of 5 sums
// per warp, nnb rows) are summed here too: thread k takes rows k, k + grid,
// ... in that order, and the rows' totals reach the slots NB_ENERGY,
// VIRIAL_XX..ZZ, ELEC_DIR (stored with nb_store, else added) before the
// reciprocal terms are merged and the pressure is formed.
template <class R>
__global__ void __launch_bounds__(256)
k_lv_step2(int N, typename V4<R>::T* __restrict__ vel, double4a* __restrict__ force,
           DevState* st, LvDev p, double* partials, int with_box, int kick, int advance,
           const double4a* __restrict__ fadd, int merge_rec, const double* __restrict__ nb_rows, int nnb,
           int nb_store) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  // the atom's loads are issued before the rows are read
  typename V4<R>::T v{};
  double4a f{}, g{};
  if (k < N) {
    v = vel[k];
    f = force[k];
    if (fadd) g = fadd[k];
  }
  double kin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (nb_rows)
    for (int r = k; r < nnb; r += gridDim.x * blockDim.x)
#pragma unroll
      for (int q = 0; q < 5; ++q) kin[3 + q] += nb_rows[(size_t)r * 5 + q];
  // The box normals of the coming step do not depend on this step's sums:
  // one thread of block 0 works them out beside the kick, off the serial
  // tail of the last block.  Block 0 signs in at the reduction counter after
  // this store (barrier, fence, atomic), so the last block sees it.
  const bool pre_xi = with_box && advance && p.dirs;
  if (pre_xi && blockIdx.x == 0 && threadIdx.x == (blockDim.x > 32 ? 32u : 0u)) {
    double xi[4];
    box_normals(p, st->step + 1ull, xi);
    for (int d = 0; d < 3; ++d) st->box_xi[d] = xi[d];
    __threadfence();
  }
  if (k < N) {
    if (fadd) {
      f.x += g.x;
      f.y += g.y;
      f.z += g.z;
      force[k] = f;
    }
    const double im = (double)v.w;
    const double h = kick ? 0.5 * p.dt : 0.0;
    double vx = v.x + h * f.x * im, vy = v.y + h * f.y * im, vz = v.z + h * f.z * im;
    v.x = (R)vx; v.y = (R)vy; v.z = (R)vz;
    vel[k] = v;
    const double m = 1.0 / im;
    kin[0] = 0.5 * m * (double)v.x * (double)v.x;
    kin[1] = 0.5 * m * (double)v.y * (double)v.y;
    kin[2] = 0.5 * m * (double)v.z * (double)v.z;
  }
  bool last;
  if (nb_rows) {
    last = block_reduce_finish<8>(kin, partials, &st->red_counter[RED_KIN], st->kick_sums, true);
    if (last) {
      for (int d = 0; d < 3; ++d) st->stats[MD_STAT_KINETIC_XX + d] = st->kick_sums[d];
      for (int q = 0; q < 5; ++q)
        st->stats[MD_STAT_NB_ENERGY + q] = (nb_store ? 0.0 : st->stats[MD_STAT_NB_ENERGY + q]) + st->kick_sums[3 + q];
    }
  } else {
    double kin3[3] = {kin[0], kin[1], kin[2]};
    last = block_reduce_finish<3>(kin3, partials, &st->red_counter[RED_KIN], &st->stats[MD_STAT_KINETIC_XX], true);
  }
  if (last && merge_rec) {
    // reciprocal energy into its slot, its diagonal virial added to the virial slots
    st->stats[MD_STAT_ELEC_REC] = st->scratch[0];
    for (int d = 0; d < 3; ++d) st->stats[MD_STAT_VIRIAL_XX + d] += st->scratch[1 + d];
  }
  if (last && with_box) {
    double xi[3];
    if (pre_xi)
      for (int d = 0; d < 3; ++d) xi[d] = __ldcg(&st->box_xi[d]);
    lv_close(st, p, kick, advance, pre_xi ? xi : nullptr);
  }
}

LvDev make_lv(const md_system* sys, const md_nlist* nl) {
  const md_langevin_params& q = sys->lv;
  LvDev p;
  p.dt = q.dt;
  p.kT = q.temperature;
  p.c1 = exp(-q.gamma_t * q.dt);
  p.c2 = sqrt(1.0 - p.c1 * p.c1);
  double gp = q.tau_p > 0 ? 1.0 / q.tau_p : 0.0;  // gamma_P = 1/tau_P (paper.tex:430)
  p.c1p = exp(-gp * q.dt);
  p.c2p = sqrt(1.0 - p.c1p * p.c1p);
  for (int d = 0; d < 3; ++d) p.pref[d] = q.p_ref[d];
  p.dirs = q.npt_dirs;
  p.seed = q.seed;
  double s = nl ? 0.5 * nl->skin : 1e300;
  p.skin_half2 = s * s;
  return p;
}

// with_box_kernel: launch k_lv_box first (manual stepping); the driver instead
// advances the box in the previous step's closing kick.  cond/use_cond: see
// k_lv_step1.
int langevin_step1_impl(md_system* sys, md_nlist* nl, Recorder* rec, bool with_box_kernel,
                        cudaGraphConditionalHandle cond, int use_cond) {
  LvDev p = make_lv(sys, nl);
  DevState* st = sys->st;
  if (with_box_kernel) {
    void* a[] = {&st, &p};
    if (int r = rec_launch(rec, (const void*)k_lv_box, dim3(1), dim3(1), 0, a)) return r;
  }
  int N = sys->N;
  void* bk = nl ? nl->backup : nullptr;
  void* a[] = {&N, &sys->pos, &sys->vel, &sys->force, &sys->id, &bk, &st, &p, &cond, &use_cond};
  const void* f = sys->prec == MD_PREC_FP64 ? (const void*)k_lv_step1<double> : (const void*)k_lv_step1<float>;
  return rec_launch(rec, f, dim3(ceil_div(N, MD_LV_THREADS)), dim3(MD_LV_THREADS), 0, a);
}

int langevin_step2_impl(md_system* sys, Recorder* rec, int kick, int advance, const double4a* fadd, int merge_rec,
                        int nb_rows, int nb_store) {
  LvDev p = make_lv(sys, nullptr);
  DevState* st = sys->st;
  int N = sys->N;
  int with_box = 1;
  const double* rows = nb_rows > 0 ? sys->nb_rows : nullptr;
  void* a[] = {&N, &sys->vel, &sys->force, &st, &p, &sys->partials, &with_box, &kick, &advance, &fadd, &merge_rec,
               &rows, &nb_rows, &nb_store};
  const void* f = sys->prec == MD_PREC_FP64 ? (const void*)k_lv_step2<double> : (const void*)k_lv_step2<float>;
  return rec_launch(rec, f, dim3(ceil_div(N, MD_LV_THREADS)), dim3(MD_LV_THREADS), 0, a);
}

// ------------------------------------------------------------ velocity Verlet
template <class R>
__global__ void k_vv1(int N, typename V4<R>::T* pos, typename V4<R>::T* vel, const double4a* force, double dt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  typename V4<R>::T x = pos[k], v = vel[k];
  const double4a f = force[k];
  const double hi = 0.5 * dt * (double)v.w;
  v.x = (R)(v.x + hi * f.x); v.y = (R)(v.y + hi * f.y); v.z = (R)(v.z + hi * f.z);
  x.x = (R)(x.x + dt * v.x); x.y = (R)(x.y + dt * v.y); x.z = (R)(x.z + dt * v.z);
  pos[k] = x;
  vel[k] = v;
}

extern "C" int md_vv_step1(md_system* sys, double dt) {
  if (!sys || !(dt > 0)) return MD_ERR_BADARG;
  int nb = ceil_div(sys->N, 256);
  if (sys->prec == MD_PREC_FP64)
    k_vv1<double><<<nb, 256, 0, sys->stream>>>(sys->N, (double4a*)sys->pos, (double4a*)sys->vel, sys->force, dt);
  else
    k_vv1<float><<<nb, 256, 0, sys->stream>>>(sys->N, (float4*)sys->pos, (float4*)sys->vel, sys->force, dt);
  MD_CHECK_LAUNCH("vv step1");
  return MD_OK;
}

extern "C" int md_vv_step2(md_system* sys, double dt, int with_stats) {
  if (!sys || !(dt > 0)) return MD_ERR_BADARG;
  LvDev p;
  memset(&p, 0, sizeof(p));
  p.dt = dt;
  int N = sys->N;
  DevState* st = sys->st;
  int nb = ceil_div(N, 256);
  (void)with_stats;
  if (sys->prec == MD_PREC_FP64)
    k_lv_step2<double><<<nb, 256, 0, sys->stream>>>(N, (double4a*)sys->vel, sys->force, st, p, sys->partials, 0, 1, 0,
                                                     nullptr, 0, nullptr, 0, 0);
  else
    k_lv_step2<float><<<nb, 256, 0, sys->stream>>>(N, (float4*)sys->vel, sys->force, st, p, sys->partials, 0, 1, 0,
                                                    nullptr, 0, nullptr, 0, 0);
  MD_CHECK_LAUNCH("vv step2");
  return MD_OK;
}

// ------------------------------------------------------------ Langevin ABI
__global__ void k_lv_init(DevState* st, double M0, double M1, double M2) {
  st->Mh[0] = M0; st->Mh[1] = M1; st->Mh[2] = M2;
  for (int d = 0; d < 3; ++d) { st->ph[d] = 0.0; st->Pcur[d] = 0.0; st->lam1[d] = st->lam2[d] = 1.0; }
}

extern "C" int md_langevin_setup(md_system* sys, const md_langevin_params* p) {
  if (!sys || !p || !(p->dt > 0) || !(p->temperature >= 0) || !(p->gamma_t >= 0)) {
    md_set_error("md_langevin_setup: bad arguments");
    return MD_ERR_BADARG;
  }
  if (p->npt_dirs && (!(p->tau_p > 0) || !(p->kappa_t > 0))) {
    md_set_error("md_langevin_setup: NPT needs tau_p > 0 and kappa_t > 0");
    return MD_ERR_BADARG;
  }
  sys->lv = *p;
  sys->lv_set = true;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  // M_V = (tau_P / 2pi)^2 / (kappa_T V0) (paper.tex:422-428), carried to a box
  // length: the restoring force on p_d is A_d dP, dP = -dV/(kappa V), dV = A_d dL
  double V = hs.L[0] * hs.L[1] * hs.L[2];
  double M[3];
  for (int d = 0; d < 3; ++d) {
    double A = V / hs.L[d];
    double w = 2.0 * M_PI / (p->tau_p > 0 ? p->tau_p : 1.0);
    M[d] = A * A / (p->kappa_t > 0 ? p->kappa_t * V : 1.0) / (w * w);
  }
  k_lv_init<<<1, 1, 0, sys->stream>>>(sys->st, M[0], M[1], M[2]);
  MD_CHECK_LAUNCH("lv init");
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}

extern "C" int md_langevin_step1(md_system* sys, md_nlist* nl) {
  if (!sys || !sys->lv_set) { md_set_error("md_langevin_step1: call md_langevin_setup first"); return MD_ERR_BADARG; }
  Recorder rec;
  rec.stream = sys->stream;
  return langevin_step1_impl(sys, nl, &rec, true, 0, 0);
}

extern "C" int md_langevin_step2(md_system* sys) {
  if (!sys || !sys->lv_set) { md_set_error("md_langevin_step2: call md_langevin_setup first"); return MD_ERR_BADARG; }
  Recorder rec;
  rec.stream = sys->stream;
  return langevin_step2_impl(sys, &rec, 1, 0);
}

extern "C" int md_langevin_get_state(md_system* sys, double* step, double p_h[3]) {
  if (!sys) return MD_ERR_BADARG;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  if (step) *step = (double)hs.step;
  if (p_h) for (int d = 0; d < 3; ++d) p_h[d] = hs.ph[d];
  return MD_OK;
}
