// Nose-Hoover chain (2 thermostats) with velocity Verlet, NVT.
// Reference: NoseHoover_Chains2 (ENG/include/Thermostat.h:77-120,
// ENG/src/Thermostat.cu:23-304), VelocityVerlet::step1/step2
// (ENG/src/Integrator.cu:300-347), TranslationalFreedomRemover, and the step
// of ENG/app/lj.nhc-xtc.cu:159-200:
//   remove COM velocity; operator_L(dt/2); step1 (kick dt/2, drift dt);
//   rebuild check; forces; step2 (kick dt/2); operator_L(dt/2)
// with operator_L(h) = G2(h/2) vxi1(h/4) G1(h/2) vxi1(h/4) Cv(h) xi(h)
//                      vxi1(h/4) G1(h/2) vxi1(h/4) G2(h/2),
//   G1(t): vxi1 += (2K - 3N T)/Q1 t     G2(t): vxi2 += (Q1 vxi1^2 - T)/Q2 t
//   vxi1(t): vxi1 *= exp(-vxi2 t)       Cv(t): v *= exp(-vxi1 t)
//   xi(t): xi1 += vxi1 t, xi2 += vxi2 t
//   Q1 = tau^2 T 3N / (4 pi^2), Q2 = Q1 / (3N).
// The chain variables are scalars and the velocity map between two kicks is
// v -> s v - w (the chain scalings and the COM shift), so K after each
// scaling is a^2 K (and K - M|u|^2/2 after the COM removal) exactly: the
// whole stretch from the closing kick of one step to the opening kick of the
// next runs in the last block of the closing kick's reduction, and the
// opening kick applies the pending (s, w).  All chain arithmetic in FP64.
#include <cmath>
#include <cstring>
#include "device_common.cuh"

struct NhcDev {
  double xi1, xi2, vxi1, vxi2;
  double Q1, Q2, LL, T;
  double s, w[3];     // pending velocity map v -> s v - w
  double mtot;        // total mass (COM removal)
  double ktensor[3];  // kinetic tensor after the last chain application
  // state right after the closing operator_L of the last step, before the
  // next step's opening half: a_end scales the stored velocities to the
  // reference's end-of-step velocities (see k_nhc_settle)
  double a_end, xi_end[4];
};

__device__ void nhc_G1(NhcDev& c, double K, double t) { c.vxi1 += (2.0 * K - c.LL * c.T) / c.Q1 * t; }
__device__ void nhc_G2(NhcDev& c, double t) { c.vxi2 += (c.Q1 * c.vxi1 * c.vxi1 - c.T) / c.Q2 * t; }
__device__ void nhc_vxi1(NhcDev& c, double t) { c.vxi1 *= exp(-c.vxi2 * t); }

// operator_L(h) on kinetic energy K; returns the velocity scale a of Cv(h)
__device__ double nhc_operator_L(NhcDev& c, double K, double h) {
  nhc_G2(c, 0.5 * h);
  nhc_vxi1(c, 0.25 * h);
  nhc_G1(c, K, 0.5 * h);
  nhc_vxi1(c, 0.25 * h);
  const double a = exp(-c.vxi1 * h);
  c.xi1 += c.vxi1 * h;
  c.xi2 += c.vxi2 * h;
  nhc_vxi1(c, 0.25 * h);
  nhc_G1(c, a * a * K, 0.5 * h);
  nhc_vxi1(c, 0.25 * h);
  nhc_G2(c, 0.5 * h);
  return a;
}

// Closing part of a step, after the kick (kick = 0: none), from the sums
// ktens (kinetic tensor of v) and mom (momentum of v):
//   end:   operator_L(h) -> a1; kinetic tensor a1^2 K into the statistics
//   start: (next step) COM removal and operator_L(h) -> a2
// pending map: v_next = a2 (a1 v - u),  u = a1 mom / M
__device__ void nhc_close(NhcDev& c, const double ktens[3], const double mom[3], double h, bool end,
                          bool start, bool remove_com, DevState* st) {
  double a1 = 1.0;
  const double K = ktens[0] + ktens[1] + ktens[2];
  if (end) a1 = nhc_operator_L(c, K, h);
  for (int d = 0; d < 3; ++d) c.ktensor[d] = a1 * a1 * ktens[d];
  if (end) {
    for (int d = 0; d < 3; ++d) st->stats[MD_STAT_KINETIC_XX + d] = c.ktensor[d];
    c.a_end = a1;
    c.xi_end[0] = c.xi1; c.xi_end[1] = c.xi2; c.xi_end[2] = c.vxi1; c.xi_end[3] = c.vxi2;
  }
  double u[3] = {0, 0, 0};
  double Ks = a1 * a1 * K;
  if (remove_com && start) {
    for (int d = 0; d < 3; ++d) u[d] = a1 * mom[d] / c.mtot;
    Ks -= 0.5 * c.mtot * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  }
  double a2 = 1.0;
  if (start) a2 = nhc_operator_L(c, Ks, h);
  c.s = a2 * a1;
  for (int d = 0; d < 3; ++d) c.w[d] = a2 * u[d];
}

// Opening kick and drift: v = s v - w, v += h F/m, x += dt v; displacement
// test against the list backup.  The last block hands the rebuild decision to
// the graph conditional (use_cond) and does the start-of-step accounting.
template <class R>
__global__ void __launch_bounds__(256)
k_nhc_vv1(int N, typename V4<R>::T* __restrict__ pos, typename V4<R>::T* __restrict__ vel,
          const double4a* __restrict__ force, const typename V4<R>::T* __restrict__ backup, DevState* st,
          const NhcDev* __restrict__ c, double dt, double skin_half2, cudaGraphConditionalHandle cond,
          int use_cond) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) {
    typename V4<R>::T x = pos[k], v = vel[k];
    const double4a f = force[k];
    const double s = c->s, h = 0.5 * dt * (double)v.w;
    double vx = s * (double)v.x - c->w[0] + h * f.x;
    double vy = s * (double)v.y - c->w[1] + h * f.y;
    double vz = s * (double)v.z - c->w[2] + h * f.z;
    v.x = (R)vx; v.y = (R)vy; v.z = (R)vz;
    x.x = (R)((double)x.x + dt * (double)v.x);
    x.y = (R)((double)x.y + dt * (double)v.y);
    x.z = (R)((double)x.z + dt * (double)v.z);
    pos[k] = x;
    vel[k] = v;
    if (backup) {
      const typename V4<R>::T b = backup[k];
      const double dx = min_image_exact((double)x.x - (double)b.x, st->L[0], st->Li[0]);
      const double dy = min_image_exact((double)x.y - (double)b.y, st->L[1], st->Li[1]);
      const double dz = min_image_exact((double)x.z - (double)b.z, st->L[2], st->Li[2]);
      const bool far = dx * dx + dy * dy + dz * dz > skin_half2;
      const unsigned m = __ballot_sync(__activemask(), far);
      if (m && (int)(threadIdx.x & 31) == __ffs(m) - 1) atomicOr(&st->flags, FLAG_REBUILD);
    }
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&st->red_counter[RED_DISP], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const unsigned f = atomicOr(&st->flags, 0u);
    if (use_cond) cudaGraphSetConditional(cond, (f & FLAG_REBUILD) ? 1u : 0u);
    st->red_counter[RED_DISP] = 0u;
    __threadfence();
  }
}

// Closing kick (kick != 0), kinetic tensor and momentum sums; the last block
// runs nhc_close and the rebuild accounting of the next step.
template <class R>
__global__ void __launch_bounds__(256)
k_nhc_vv2(int N, typename V4<R>::T* __restrict__ vel, const double4a* __restrict__ force, DevState* st,
          NhcDev* c, double dt, double* partials, int kick, int end, int start, int remove_com, int account) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double v6[6] = {0, 0, 0, 0, 0, 0};
  if (k < N) {
    typename V4<R>::T v = vel[k];
    const double4a f = force[k];
    const double im = (double)v.w;
    const double h = kick ? 0.5 * dt * im : 0.0;
    v.x = (R)((double)v.x + h * f.x);
    v.y = (R)((double)v.y + h * f.y);
    v.z = (R)((double)v.z + h * f.z);
    vel[k] = v;
    const double m = 1.0 / im;
    v6[0] = 0.5 * m * (double)v.x * (double)v.x;
    v6[1] = 0.5 * m * (double)v.y * (double)v.y;
    v6[2] = 0.5 * m * (double)v.z * (double)v.z;
    v6[3] = m * (double)v.x;
    v6[4] = m * (double)v.y;
    v6[5] = m * (double)v.z;
  }
  const bool last = block_reduce_finish<6>(v6, partials, &st->red_counter[RED_KIN], st->scratch, true);
  if (last) {
    NhcDev cc = *c;
    const double kt[3] = {st->scratch[0], st->scratch[1], st->scratch[2]};
    const double mo[3] = {st->scratch[3], st->scratch[4], st->scratch[5]};
    nhc_close(cc, kt, mo, 0.5 * dt, end != 0, start != 0, remove_com != 0, st);
    *c = cc;
    if (start && account) {
      // rebuild accounting of the coming step (as box_advance)
      const unsigned f = st->flags;
      if (f & FLAG_REBUILD) st->rebuilds += 1ull;
      st->flags = (f & ~(FLAG_REBUILD | FLAG_FORCE_REBUILD)) | ((f & FLAG_FORCE_REBUILD) ? FLAG_REBUILD : 0u);
      st->step += 1ull;
    }
  }
}

// standalone operator_L: sums of the current velocities, chain, then scale
template <class R>
__global__ void __launch_bounds__(256)
k_nhc_apply(int N, typename V4<R>::T* __restrict__ vel, const NhcDev* __restrict__ c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  typename V4<R>::T v = vel[k];
  v.x = (R)(c->s * (double)v.x - c->w[0]);
  v.y = (R)(c->s * (double)v.y - c->w[1]);
  v.z = (R)(c->s * (double)v.z - c->w[2]);
  vel[k] = v;
}

// End of a driver run: bring the stored velocities to the end of the last
// step (v a_end) and the chain back to its state after that step's closing
// operator_L; the next run re-applies the opening half (k_nhc_vv2 with start,
// without the step accounting, which already happened)
template <class R>
__global__ void __launch_bounds__(256)
k_nhc_settle(int N, typename V4<R>::T* __restrict__ vel, const NhcDev* __restrict__ c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  typename V4<R>::T v = vel[k];
  const double a = c->a_end;
  v.x = (R)(a * (double)v.x);
  v.y = (R)(a * (double)v.y);
  v.z = (R)(a * (double)v.z);
  vel[k] = v;
}

__global__ void k_nhc_restore(NhcDev* c) {
  c->xi1 = c->xi_end[0]; c->xi2 = c->xi_end[1]; c->vxi1 = c->xi_end[2]; c->vxi2 = c->xi_end[3];
  c->s = 1.0;
  c->w[0] = c->w[1] = c->w[2] = 0.0;
  c->a_end = 1.0;
}

__global__ void k_nhc_mass(int N, const float4* vf, const double4a* vd, int prec, double* partials,
                           unsigned* counter, NhcDev* c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double m[1] = {0.0};
  if (k < N) m[0] = 1.0 / (prec == MD_PREC_FP64 ? vd[k].w : (double)vf[k].w);
  block_reduce_finish<1>(m, partials, counter, &c->mtot, true);
}

// ------------------------------------------------------------------ host
struct md_nhc {
  md_system* sys = nullptr;
  NhcDev* dev = nullptr;
  double refT = 0, tauT = 0;
  int remove_com = 1;
};

int nhc_vv1_impl(md_nhc* h, md_nlist* nl, double dt, Recorder* rec, cudaGraphConditionalHandle cond,
                 int use_cond) {
  md_system* sys = h->sys;
  int N = sys->N;
  void* bk = nl ? nl->backup : nullptr;
  double sk = nl ? 0.5 * nl->skin : 1e300;
  double skin_half2 = sk * sk;
  DevState* st = sys->st;
  void* a[] = {&N, &sys->pos, &sys->vel, &sys->force, &bk, &st, &h->dev, &dt, &skin_half2, &cond, &use_cond};
  const void* f = sys->prec == MD_PREC_FP64 ? (const void*)k_nhc_vv1<double> : (const void*)k_nhc_vv1<float>;
  return rec_launch(rec, f, dim3(ceil_div(N, 256)), dim3(256), 0, a);
}

int nhc_vv2_impl(md_nhc* h, double dt, Recorder* rec, int kick, int end, int start, int account) {
  md_system* sys = h->sys;
  int N = sys->N;
  DevState* st = sys->st;
  int rc = h->remove_com;
  void* a[] = {&N, &sys->vel, &sys->force, &st, &h->dev, &dt, &sys->partials, &kick, &end, &start, &rc, &account};
  const void* f = sys->prec == MD_PREC_FP64 ? (const void*)k_nhc_vv2<double> : (const void*)k_nhc_vv2<float>;
  return rec_launch(rec, f, dim3(ceil_div(N, 256)), dim3(256), 0, a);
}

int nhc_settle_impl(md_nhc* h) {
  md_system* sys = h->sys;
  const int N = sys->N;
  if (sys->prec == MD_PREC_FP64)
    k_nhc_settle<double><<<ceil_div(N, 256), 256, 0, sys->stream>>>(N, (double4a*)sys->vel, h->dev);
  else
    k_nhc_settle<float><<<ceil_div(N, 256), 256, 0, sys->stream>>>(N, (float4*)sys->vel, h->dev);
  MD_CHECK_LAUNCH("nhc settle");
  k_nhc_restore<<<1, 1, 0, sys->stream>>>(h->dev);
  MD_CHECK_LAUNCH("nhc restore");
  return MD_OK;
}

__global__ void k_nhc_init(NhcDev* c, double Q1, double Q2, double LL, double T) {
  c->xi1 = c->xi2 = 1.0;  // NoseHoover_Chains2::reinit
  c->vxi1 = c->vxi2 = 0.0;
  c->Q1 = Q1; c->Q2 = Q2; c->LL = LL; c->T = T;
  c->s = 1.0;
  c->w[0] = c->w[1] = c->w[2] = 0.0;
  c->ktensor[0] = c->ktensor[1] = c->ktensor[2] = 0.0;
  c->a_end = 1.0;
  c->xi_end[0] = c->xi_end[1] = 1.0;
  c->xi_end[2] = c->xi_end[3] = 0.0;
}

extern "C" int md_nhc_create(md_nhc** out, md_system* sys, double ref_T, double tau_T, int remove_com) {
  if (!out || !sys || !(ref_T > 0) || !(tau_T > 0)) { md_set_error("md_nhc_create: bad arguments"); return MD_ERR_BADARG; }
  md_nhc* h = new md_nhc();
  h->sys = sys;
  h->refT = ref_T;
  h->tauT = tau_T;
  h->remove_com = remove_com ? 1 : 0;
  if (cudaMalloc(&h->dev, sizeof(NhcDev)) != cudaSuccess) {
    delete h;
    return md_cuda_fail(cudaGetLastError(), "md_nhc_create");
  }
  const double LL = 3.0 * sys->N;
  const double Q1 = tau_T * tau_T * ref_T / (4 * M_PI * M_PI) * LL;
  k_nhc_init<<<1, 1, 0, sys->stream>>>(h->dev, Q1, Q1 / LL, LL, ref_T);
  MD_CHECK_LAUNCH("nhc init");
  const int nb = ceil_div(sys->N, 256);
  k_nhc_mass<<<nb, 256, 0, sys->stream>>>(sys->N, (const float4*)sys->vel, (const double4a*)sys->vel, sys->prec,
                                          sys->partials, &sys->st->red_counter[RED_MISC], h->dev);
  MD_CHECK_LAUNCH("nhc mass");
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  *out = h;
  return MD_OK;
}

extern "C" int md_nhc_destroy(md_nhc* h) {
  if (!h) return MD_OK;
  if (h->dev) cudaFree(h->dev);
  delete h;
  return MD_OK;
}

// operator_L(dt) on the current velocities (NoseHoover_Chains2::operator_L):
// one reduction whose last block runs the chain, then the scaling
extern "C" int md_nhc_operator_L(md_nhc* h, md_system* sys, double dt, int with_stats) {
  if (!h || !sys || sys != h->sys || !(dt > 0)) { md_set_error("md_nhc_operator_L: bad arguments"); return MD_ERR_BADARG; }
  Recorder rec;
  rec.stream = sys->stream;
  // nhc_close runs operator_L(dt_step / 2): pass 2 dt; end only, so the COM
  // is left alone
  if (int r = nhc_vv2_impl(h, 2.0 * dt, &rec, 0, 1, 0, 0)) return r;
  const int N = sys->N;
  if (sys->prec == MD_PREC_FP64)
    k_nhc_apply<double><<<ceil_div(N, 256), 256, 0, sys->stream>>>(N, (double4a*)sys->vel, h->dev);
  else
    k_nhc_apply<float><<<ceil_div(N, 256), 256, 0, sys->stream>>>(N, (float4*)sys->vel, h->dev);
  MD_CHECK_LAUNCH("nhc apply");
  (void)with_stats;  // the kinetic tensor slots always receive the scaled tensor
  return MD_OK;
}

// xi1, xi2, vxi1, vxi2 and HamiltonianContribution
// (0.5 Q1 vxi1^2 + 0.5 Q2 vxi2^2 + 3N T xi1 + T xi2)
extern "C" int md_nhc_get_state(md_nhc* h, double out[5]) {
  if (!h || !out) return MD_ERR_BADARG;
  NhcDev c;
  MD_CUDA(cudaMemcpyAsync(&c, h->dev, sizeof(c), cudaMemcpyDeviceToHost, h->sys->stream));
  MD_CUDA(cudaStreamSynchronize(h->sys->stream));
  out[0] = c.xi1; out[1] = c.xi2; out[2] = c.vxi1; out[3] = c.vxi2;
  out[4] = 0.5 * c.Q1 * c.vxi1 * c.vxi1 + 0.5 * c.Q2 * c.vxi2 * c.vxi2 + c.LL * c.T * c.xi1 + c.T * c.xi2;
  return MD_OK;
}

// ===================================================================== NPT
// NoseHoover_Chains2_Isobaric (ENG/include/Barostat.h:90-175,
// ENG/src/Barostat.cu:6-460): one thermostat on particles and barostat,
// isotropic box.  Nf = 3N - 3, Q1 = tau_T^2 T Nf, W = tau_P^2 T Nf,
// ep = ln(V)/3, vep = 0, xi1 = 1, vxi1 = 0.
//   G1(t):  vxi1 += (2K + W vep^2 - (Nf + 1) T)/Q1 t
//   Gep(t): vep  += (6K/Nf + 3V (P - P_ref))/W t,  P = tr(P_dd)/3 + pcorr
//   vep(t): vep  *= exp(-vxi1 t)
//   Cv(t):  v    *= exp(-(vxi1 + (1 + 3/Nf) vep) t)
//   xi(t):  xi1  += vxi1 t
//   L_CP(t) = G1(t/2) vep(t/4) Gep(t/2) vep(t/4) Cv(t) xi(t) vep(t/4) Gep(t/2) vep(t/4) G1(t/2)
//   L_v(t): v += t F/m;  L_r(t): x = e^{vep t} x + t e^{vep t/2} S(vep t/2) v with
//   S(x) = 1 + x^2/6 + x^4/120 + x^6/5040 + x^8/362880 + x^10/39916800;
//   L_box(t): L *= e^{vep t}, ep += vep t.
// The pressure uses the kinetic tensor of the velocities the operator sees
// and the virial slots of the last force evaluation.
struct NhcPDev {
  double ep, vep, xi1, vxi1;
  double Nf, Q1, W, T, Pref, pcorr;
  double a;  // velocity scale of the last Cv
};

__device__ double nhcp_pressure(const NhcPDev& c, const double K[3], const DevState* st) {
  const double V = st->L[0] * st->L[1] * st->L[2];
  double P = 0.0;
  for (int d = 0; d < 3; ++d) P += 2.0 / V * (K[d] - 0.5 * st->stats[MD_STAT_VIRIAL_XX + d]);
  return P / 3.0 + c.pcorr;
}

// L_CP(t) given the kinetic tensor K of the current velocities; returns the
// scale a of Cv and leaves a^2 K in Ko
__device__ double nhcp_L_CP(NhcPDev& c, const double K[3], double t, const DevState* st, double Ko[3]) {
  const double V = st->L[0] * st->L[1] * st->L[2];
  const double Ks = K[0] + K[1] + K[2];
  c.vxi1 += (2.0 * Ks + c.W * c.vep * c.vep - (c.Nf + 1.0) * c.T) / c.Q1 * (0.5 * t);
  c.vep *= exp(-c.vxi1 * 0.25 * t);
  c.vep += (6.0 / c.Nf * Ks + 3.0 * V * (nhcp_pressure(c, K, st) - c.Pref)) / c.W * (0.5 * t);
  c.vep *= exp(-c.vxi1 * 0.25 * t);
  const double a = exp(-(c.vxi1 + (1.0 + 3.0 / c.Nf) * c.vep) * t);
  for (int d = 0; d < 3; ++d) Ko[d] = a * a * K[d];
  const double Ks2 = Ko[0] + Ko[1] + Ko[2];
  c.xi1 += c.vxi1 * t;
  c.vep *= exp(-c.vxi1 * 0.25 * t);
  c.vep += (6.0 / c.Nf * Ks2 + 3.0 * V * (nhcp_pressure(c, Ko, st) - c.Pref)) / c.W * (0.5 * t);
  c.vep *= exp(-c.vxi1 * 0.25 * t);
  c.vxi1 += (2.0 * Ks2 + c.W * c.vep * c.vep - (c.Nf + 1.0) * c.T) / c.Q1 * (0.5 * t);
  return a;
}

template <class R>
__global__ void __launch_bounds__(256)
k_nhcp_cp(int N, const typename V4<R>::T* __restrict__ vel, DevState* st, NhcPDev* c, double t, double* partials) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double kin[3] = {0, 0, 0};
  if (k < N) {
    const typename V4<R>::T v = vel[k];
    const double m = 1.0 / (double)v.w;
    kin[0] = 0.5 * m * (double)v.x * (double)v.x;
    kin[1] = 0.5 * m * (double)v.y * (double)v.y;
    kin[2] = 0.5 * m * (double)v.z * (double)v.z;
  }
  if (block_reduce_finish<3>(kin, partials, &st->red_counter[RED_KIN], st->scratch, true)) {
    NhcPDev cc = *c;
    const double K[3] = {st->scratch[0], st->scratch[1], st->scratch[2]};
    double Ko[3];
    cc.a = nhcp_L_CP(cc, K, t, st, Ko);
    for (int d = 0; d < 3; ++d) st->stats[MD_STAT_KINETIC_XX + d] = Ko[d];
    *c = cc;
  }
}

template <class R>
__global__ void __launch_bounds__(256)
k_nhcp_scale(int N, typename V4<R>::T* __restrict__ vel, const NhcPDev* __restrict__ c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  typename V4<R>::T v = vel[k];
  const double a = c->a;
  v.x = (R)(a * (double)v.x); v.y = (R)(a * (double)v.y); v.z = (R)(a * (double)v.z);
  vel[k] = v;
}

template <class R>
__global__ void __launch_bounds__(256)
k_nhcp_r(int N, typename V4<R>::T* __restrict__ pos, const typename V4<R>::T* __restrict__ vel,
         const NhcPDev* __restrict__ c, double t) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const double xx = c->vep * t * 0.5;
  const double s1 = exp(c->vep * t);
  const double x2 = xx * xx, x4 = x2 * x2, x6 = x4 * x2, x8 = x6 * x2, x10 = x8 * x2;
  const double s2 = t * exp(xx) *
                    (1. + 1. / 6. * x2 + 1. / 120. * x4 + 1. / 5040. * x6 + 1. / 362880. * x8 + 1. / 39916800. * x10);
  typename V4<R>::T x = pos[k];
  const typename V4<R>::T v = vel[k];
  x.x = (R)(s1 * (double)x.x + s2 * (double)v.x);
  x.y = (R)(s1 * (double)x.y + s2 * (double)v.y);
  x.z = (R)(s1 * (double)x.z + s2 * (double)v.z);
  pos[k] = x;
}

__global__ void k_nhcp_box(DevState* st, NhcPDev* c, double t) {
  const double s = exp(c->vep * t);
  c->ep += t * c->vep;
  for (int d = 0; d < 3; ++d) {
    st->L[d] = st->L[d] * s;
    st->Li[d] = 1.0 / st->L[d];
    st->Lf[d] = (float)st->L[d];
    st->Lif[d] = 1.0f / st->Lf[d];
  }
}

__global__ void k_nhcp_init(NhcPDev* c, const DevState* st, double Nf, double Q1, double W, double T, double Pref,
                            double pcorr) {
  c->ep = log(st->L[0] * st->L[1] * st->L[2]) / 3.0;
  c->vep = 0.0;
  c->xi1 = 1.0;
  c->vxi1 = 0.0;
  c->Nf = Nf; c->Q1 = Q1; c->W = W; c->T = T; c->Pref = Pref; c->pcorr = pcorr;
  c->a = 1.0;
}

struct md_nhc_npt {
  md_system* sys = nullptr;
  NhcPDev* dev = nullptr;
};

extern "C" int md_nhc_npt_create(md_nhc_npt** out, md_system* sys, double ref_T, double tau_T, double ref_P,
                                 double tau_P, double pressure_corr) {
  if (!out || !sys || !(ref_T > 0) || !(tau_T > 0) || !(tau_P > 0) || !std::isfinite(ref_P) ||
      !std::isfinite(pressure_corr)) {
    md_set_error("md_nhc_npt_create: bad arguments");
    return MD_ERR_BADARG;
  }
  md_nhc_npt* h = new md_nhc_npt();
  h->sys = sys;
  if (cudaMalloc(&h->dev, sizeof(NhcPDev)) != cudaSuccess) {
    delete h;
    return md_cuda_fail(cudaGetLastError(), "md_nhc_npt_create");
  }
  const double Nf = 3.0 * sys->N - 3.0;
  k_nhcp_init<<<1, 1, 0, sys->stream>>>(h->dev, sys->st, Nf, tau_T * tau_T * ref_T * Nf, tau_P * tau_P * ref_T * Nf,
                                        ref_T, ref_P, pressure_corr);
  MD_CHECK_LAUNCH("nhc npt init");
  *out = h;
  return MD_OK;
}

extern "C" int md_nhc_npt_destroy(md_nhc_npt* h) {
  if (!h) return MD_OK;
  if (h->dev) cudaFree(h->dev);
  delete h;
  return MD_OK;
}

extern "C" int md_nhc_npt_operator_L_CP(md_nhc_npt* h, md_system* sys, double dt) {
  if (!h || !sys || sys != h->sys || !(dt > 0)) { md_set_error("operator_L_CP: bad arguments"); return MD_ERR_BADARG; }
  const int N = sys->N, nb = ceil_div(N, 256);
  if (sys->prec == MD_PREC_FP64) {
    k_nhcp_cp<double><<<nb, 256, 0, sys->stream>>>(N, (const double4a*)sys->vel, sys->st, h->dev, dt, sys->partials);
    k_nhcp_scale<double><<<nb, 256, 0, sys->stream>>>(N, (double4a*)sys->vel, h->dev);
  } else {
    k_nhcp_cp<float><<<nb, 256, 0, sys->stream>>>(N, (const float4*)sys->vel, sys->st, h->dev, dt, sys->partials);
    k_nhcp_scale<float><<<nb, 256, 0, sys->stream>>>(N, (float4*)sys->vel, h->dev);
  }
  MD_CHECK_LAUNCH("operator_L_CP");
  return MD_OK;
}

// L_v(dt): v += dt F/m with the kinetic tensor into the statistic slots
extern "C" int md_nhc_npt_operator_L_v(md_nhc_npt* h, md_system* sys, double dt) {
  if (!h || !sys || sys != h->sys || !(dt > 0)) { md_set_error("operator_L_v: bad arguments"); return MD_ERR_BADARG; }
  // md_vv_step2 kicks by dt/2: pass 2 dt
  return md_vv_step2(sys, 2.0 * dt, 1);
}

extern "C" int md_nhc_npt_operator_L_r(md_nhc_npt* h, md_system* sys, double dt) {
  if (!h || !sys || sys != h->sys || !(dt > 0)) { md_set_error("operator_L_r: bad arguments"); return MD_ERR_BADARG; }
  const int N = sys->N, nb = ceil_div(N, 256);
  if (sys->prec == MD_PREC_FP64)
    k_nhcp_r<double><<<nb, 256, 0, sys->stream>>>(N, (double4a*)sys->pos, (const double4a*)sys->vel, h->dev, dt);
  else
    k_nhcp_r<float><<<nb, 256, 0, sys->stream>>>(N, (float4*)sys->pos, (const float4*)sys->vel, h->dev, dt);
  MD_CHECK_LAUNCH("operator_L_r");
  return MD_OK;
}

extern "C" int md_nhc_npt_operator_L_box(md_nhc_npt* h, md_system* sys, double dt) {
  if (!h || !sys || sys != h->sys || !(dt > 0)) { md_set_error("operator_L_box: bad arguments"); return MD_ERR_BADARG; }
  k_nhcp_box<<<1, 1, 0, sys->stream>>>(sys->st, h->dev, dt);
  MD_CHECK_LAUNCH("operator_L_box");
  return MD_OK;
}

// ep, vep, xi1, vxi1, HamiltonianContribution (W vep^2/2 + Q1 vxi1^2/2 + (Nf+1) T xi1 + P_ref V)
extern "C" int md_nhc_npt_get_state(md_nhc_npt* h, double out[5]) {
  if (!h || !out) return MD_ERR_BADARG;
  NhcPDev c;
  DevState hs;
  MD_CUDA(cudaMemcpyAsync(&c, h->dev, sizeof(c), cudaMemcpyDeviceToHost, h->sys->stream));
  if (int r = h->sys->read_state(hs)) return r;
  const double V = hs.L[0] * hs.L[1] * hs.L[2];
  out[0] = c.ep; out[1] = c.vep; out[2] = c.xi1; out[3] = c.vxi1;
  out[4] = 0.5 * c.W * c.vep * c.vep + 0.5 * c.Q1 * c.vxi1 * c.vxi1 + (c.Nf + 1.0) * c.T * c.xi1 + c.Pref * V;
  return MD_OK;
}

// the step of ENG/app/lj.nhc-xtc.cu with manual stepping: md_nhc_step1 does
// [COM removal] operator_L(dt/2) + step1, md_nhc_step2 step2 + operator_L(dt/2)
extern "C" int md_nhc_step1(md_nhc* h, md_system* sys, md_nlist* nl, double dt) {
  if (!h || !sys || sys != h->sys || !(dt > 0)) { md_set_error("md_nhc_step1: bad arguments"); return MD_ERR_BADARG; }
  Recorder rec;
  rec.stream = sys->stream;
  // start part of the chain (the end part ran in the previous md_nhc_step2)
  if (int r = nhc_vv2_impl(h, dt, &rec, 0, 0, 1, 1)) return r;
  return nhc_vv1_impl(h, nl, dt, &rec, 0, 0);
}

extern "C" int md_nhc_step2(md_nhc* h, md_system* sys, double dt) {
  if (!h || !sys || sys != h->sys || !(dt > 0)) { md_set_error("md_nhc_step2: bad arguments"); return MD_ERR_BADARG; }
  Recorder rec;
  rec.stream = sys->stream;
  if (int r = nhc_vv2_impl(h, dt, &rec, 1, 1, 0, 0)) return r;
  // apply the end scaling now so that the velocities are current between calls
  const int N = sys->N;
  if (sys->prec == MD_PREC_FP64)
    k_nhc_apply<double><<<ceil_div(N, 256), 256, 0, sys->stream>>>(N, (double4a*)sys->vel, h->dev);
  else
    k_nhc_apply<float><<<ceil_div(N, 256), 256, 0, sys->stream>>>(N, (float4*)sys->vel, h->dev);
  MD_CHECK_LAUNCH("nhc apply");
  return MD_OK;
}
