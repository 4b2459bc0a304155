// A-priori Ewald / SPME error estimates, FP64 k-space sums on the GPU; these
// choose the splitting beta and the mesh.
// Reference (RE = longRange.hetero/profile.test/template/tools/real.error):
//   ElectrostaticInteraction::errorEstimatePME (version 3)  RE/src/ElectrostaticInteraction.cpp:349-401
//   ElectrostaticInteraction_rec_BSpline::errorEstimate    RE/src/EleRecBSpline.cpp:154-206
//   EleEcalculator (produce4Item)                          RE/src/EleEcalculator.cpp:100-220
#include <cmath>
#include <vector>
#include "device_common.cuh"

__global__ void k_charge_sq(int N, const float4* pf, const double4a* pd, int prec, double* partials,
                            unsigned* counter, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0};
  if (i < N) {
    const double q = prec == MD_PREC_FP64 ? pd[i].w : (double)pf[i].w;
    v[0] = q * q;
  }
  block_reduce_finish<1>(v, partials, counter, out, true);
}

// sum over |m_d| <= K_d outside the |m_d| <= K_d/2 box of e^{-2 pi^2 m^2/beta^2}/m^2
__global__ void k_est_pme_rec(int K0, int K1, int K2, double beta, const DevState* st, double* partials,
                              unsigned* counter, double* out) {
  const long n0 = 2 * K0 + 1, n1 = 2 * K1 + 1, n2 = 2 * K2 + 1;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double v[1] = {0};
  if (t < n0 * n1 * n2) {
    const int m2 = (int)(t % n2) - K2, m1 = (int)((t / n2) % n1) - K1, m0 = (int)(t / (n2 * n1)) - K0;
    const bool inner = m0 >= -K0 / 2 && m0 <= K0 / 2 && m1 >= -K1 / 2 && m1 <= K1 / 2 && m2 >= -K2 / 2 && m2 <= K2 / 2;
    if (!inner) {
      const double mx = m0 * st->Li[0], my = m1 * st->Li[1], mz = m2 * st->Li[2];
      const double mm = mx * mx + my * my + mz * mz;
      v[0] = exp(-2 * M_PI * M_PI / (beta * beta) * mm) / mm;
    }
  }
  block_reduce_finish<1>(v, partials, counter, out, true);
}

// sum over m in [-K/2, K/2)^3 \ 0 of 2 (2/V)^2 e^{-2 pi^2 m^2/beta^2}/m^2 (ees + eemid)
__global__ void k_est_spme_ik(int K0, int K1, int K2, double beta, const double* e1, const double* e2,
                              const DevState* st, double* partials, unsigned* counter, double* out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double v[1] = {0};
  if (t < (long)K0 * K1 * K2) {
    const int m2 = (int)(t % K2) - K2 / 2, m1 = (int)((t / K2) % K1) - K1 / 2, m0 = (int)(t / ((long)K2 * K1)) - K0 / 2;
    if (m0 || m1 || m2) {
      const double V = st->L[0] * st->L[1] * st->L[2];
      const double mx = m0 * st->Li[0], my = m1 * st->Li[1], mz = m2 * st->Li[2];
      const double mm = mx * mx + my * my + mz * mz;
      // tables: [d][m + K_d/2], d-th block of K_max+1 entries
      const int o0 = m0 + K0 / 2, o1 = 1025 + m1 + K1 / 2, o2 = 2050 + m2 + K2 / 2;
      const double a0 = e1[o0], a1 = e1[o1], a2 = e1[o2];
      const double ees = e2[o0] + e2[o1] + e2[o2] + 2 * a0 * a1 + 2 * a0 * a2 + 2 * a1 * a2;
      const double s = a0 + a1 + a2;
      const double expp = exp(-2 * M_PI * M_PI / (beta * beta) * mm) / mm * 2 / V * 2 / V;
      v[0] = 2 * expp * (ees + s * s);
    }
  }
  block_reduce_finish<1>(v, partials, counter, out, true);
}

static double ipow(int n, double x) {
  double v = 1;
  for (int i = 0; i < n; ++i) v *= x;
  return v;
}

// produce4Item: aliasing sums over |l| = 1..5 (numerator) and |l| <= 7 (denominator)
static void ecal(double x, int n, double& e1, double& e2) {
  if (x == 0) { e1 = e2 = 0; return; }
  auto sum = [&](int nn, int first, int last) {
    double s = 0;
    for (int l = first; l <= last; ++l) {
      if (l == 0) { s += 1. / ipow(nn, x); continue; }
      s += 1. / ipow(nn, x + 2 * M_PI * l) + 1. / ipow(nn, x - 2 * M_PI * l);
    }
    return s;
  };
  const double s6 = sum(n, 1, 5), de = sum(n, 0, 7);
  e1 = -s6 / de;
  e2 = (s6 * s6 + sum(2 * n, 1, 5)) / (de * de);
}

static int charge_sq(md_system* sys, double* c2) {
  k_charge_sq<<<ceil_div(sys->N, 256), 256, 0, sys->stream>>>(sys->N, (float4*)sys->pos, (double4a*)sys->pos,
                                                               sys->prec, sys->partials,
                                                               &sys->st->red_counter[RED_MISC], &sys->st->scratch[4]);
  MD_CHECK_LAUNCH("charge sq");
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  *c2 = hs.scratch[4];
  return MD_OK;
}

extern "C" int md_error_estimate_pme(md_system* sys, const int K[3], double beta, double rcut, double* err_dir,
                                     double* err_rec) {
  if (!sys || !K || !(beta > 0) || !(rcut > 0)) return MD_ERR_BADARG;
  double c2;
  if (int r = charge_sq(sys, &c2)) return r;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  const double V = hs.L[0] * hs.L[1] * hs.L[2];
  if (err_dir) *err_dir = 2 * sqrt(c2 / (double)sys->N) * sqrt(c2 / rcut / V) * exp(-beta * beta * rcut * rcut);
  if (err_rec) {
    const long n = (long)(2 * K[0] + 1) * (2 * K[1] + 1) * (2 * K[2] + 1);
    const int nb = (int)((n + 255) / 256);
    double* part = nullptr;
    MD_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * nb, sys->stream));
    k_est_pme_rec<<<nb, 256, 0, sys->stream>>>(K[0], K[1], K[2], beta, sys->st, part,
                                               &sys->st->red_counter[RED_MISC], &sys->st->scratch[5]);
    MD_CHECK_LAUNCH("est pme");
    MD_CUDA(cudaFreeAsync(part, sys->stream));
    if (int r = sys->read_state(hs)) return r;
    *err_rec = sqrt(hs.scratch[5] / (double)sys->N) * 2 * c2 / V;
  }
  return MD_OK;
}

extern "C" int md_error_estimate_spme_ik(md_system* sys, const int K[3], int order, double beta, double* err) {
  if (!sys || !K || !err || order < 2 || !(beta > 0)) return MD_ERR_BADARG;
  for (int d = 0; d < 3; ++d)
    if (K[d] < 2 || K[d] > 1024) { md_set_error("mesh size out of range"); return MD_ERR_BADARG; }
  double c2;
  if (int r = charge_sq(sys, &c2)) return r;
  std::vector<double> e1(3 * 1025, 0.0), e2(3 * 1025, 0.0);
  for (int d = 0; d < 3; ++d)
    for (int m = -K[d] / 2; m <= K[d] / 2; ++m) ecal(2 * M_PI * m / (double)K[d], order, e1[d * 1025 + m + K[d] / 2], e2[d * 1025 + m + K[d] / 2]);
  double* tab = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&tab, sizeof(double) * 2 * 3 * 1025, sys->stream));
  MD_CUDA(cudaMemcpyAsync(tab, e1.data(), sizeof(double) * 3 * 1025, cudaMemcpyHostToDevice, sys->stream));
  MD_CUDA(cudaMemcpyAsync(tab + 3 * 1025, e2.data(), sizeof(double) * 3 * 1025, cudaMemcpyHostToDevice, sys->stream));
  const long n = (long)K[0] * K[1] * K[2];
  const int nb = (int)((n + 255) / 256);
  double* part = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * nb, sys->stream));
  k_est_spme_ik<<<nb, 256, 0, sys->stream>>>(K[0], K[1], K[2], beta, tab, tab + 3 * 1025, sys->st, part,
                                             &sys->st->red_counter[RED_MISC], &sys->st->scratch[6]);
  MD_CHECK_LAUNCH("est spme");
  MD_CUDA(cudaFreeAsync(part, sys->stream));
  MD_CUDA(cudaFreeAsync(tab, sys->stream));
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  *err = sqrt(hs.scratch[6] * c2 * c2 / (double)sys->N);
  return MD_OK;
}

// ---------------------------------------------------------------------------
// md_error_estimate_spme_ik_noalloc: the ik-SPME interpolation estimate above,
// computed by the same kernel, without any device allocation. The estimate is
// re-evaluated whenever a barostat changes the box or a tuner tries another
// mesh; a caller that reserves all device memory up front in its own pool, or
// that must keep the stream-ordered allocator from growing between steps,
// cannot let each evaluation allocate its aliasing tables and per-block
// partial sums. This variant takes both from one fixed scratch array per
// device instead:
//   [0, 3*1025)            e1 tables of the three axes
//   [3*1025, 6*1025)       e2 tables
//   [6*1025, +max_blocks)  one partial sum per block of k_est_spme_ik
// Nothing in it has to start at zero: the tables are rewritten by every call
// and each block writes its own partial before the last block reads it (the
// completion counter is the system's, reset by that last block). Meshes are
// limited to K0*K1*K2 <= EST_NOALLOC_MAX_BLOCKS * 256 = 4,194,304 points
// (160^3 fits; 256^3 does not) and larger ones are rejected with
// MD_ERR_BADARG. All calls on one device share the scratch: two calls that
// overlap in time (different streams or host threads on one device) race and
// return wrong estimates; calls issued one after the other are safe. The call
// waits for the system's stream (it reads the charges and the result back)
// and copies its tables from pageable host memory, so it must not be issued
// while that stream is being captured into a CUDA graph.
constexpr int EST_TAB = 3 * 1025;
constexpr int EST_NOALLOC_MAX_BLOCKS = 16384;
constexpr int EST_NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) double g_est_scratch[2 * EST_TAB + EST_NOALLOC_MAX_BLOCKS];  // 180 KiB

// Device address of g_est_scratch on `device`, looked up with that device
// current on every call (the lookup is cheap once the module is loaded, and a
// fresh lookup stays valid after a cudaDeviceReset has reloaded the module).
static int est_scratch(int device, double** out) {
  if (device < 0 || device >= EST_NOALLOC_MAX_DEVICES) {
    md_set_error("device %d outside the %d devices the estimate scratch supports", device, EST_NOALLOC_MAX_DEVICES);
    return MD_ERR_BADARG;
  }
  int prev = 0;
  MD_CUDA(cudaGetDevice(&prev));
  if (prev != device) MD_CUDA(cudaSetDevice(device));
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_est_scratch);
  if (prev != device) cudaSetDevice(prev);
  if (e != cudaSuccess) return md_cuda_fail(e, "cudaGetSymbolAddress(g_est_scratch)");
  *out = (double*)p;
  return MD_OK;
}

extern "C" int md_error_estimate_spme_ik_noalloc(md_system* sys, const int K[3], int order, double beta,
                                                 double* err) {
  if (!sys || !K || !err || order < 2 || !(beta > 0)) return MD_ERR_BADARG;
  for (int d = 0; d < 3; ++d)
    if (K[d] < 2 || K[d] > 1024) { md_set_error("mesh size out of range"); return MD_ERR_BADARG; }
  const long n = (long)K[0] * K[1] * K[2];
  const long nb = (n + 255) / 256;
  if (nb > EST_NOALLOC_MAX_BLOCKS) {
    md_set_error("mesh %dx%dx%d has %ld points; the allocation-free estimate handles at most %d",
                 K[0], K[1], K[2], n, EST_NOALLOC_MAX_BLOCKS * 256);
    return MD_ERR_BADARG;
  }
  double* scratch = nullptr;
  if (int r = est_scratch(sys->device, &scratch)) return r;
  double c2;
  if (int r = charge_sq(sys, &c2)) return r;
  std::vector<double> tab(2 * EST_TAB, 0.0);
  for (int d = 0; d < 3; ++d)
    for (int m = -K[d] / 2; m <= K[d] / 2; ++m)
      ecal(2 * M_PI * m / (double)K[d], order, tab[d * 1025 + m + K[d] / 2], tab[EST_TAB + d * 1025 + m + K[d] / 2]);
  MD_CUDA(cudaMemcpyAsync(scratch, tab.data(), sizeof(double) * 2 * EST_TAB, cudaMemcpyHostToDevice, sys->stream));
  k_est_spme_ik<<<(int)nb, 256, 0, sys->stream>>>(K[0], K[1], K[2], beta, scratch, scratch + EST_TAB, sys->st,
                                                  scratch + 2 * EST_TAB, &sys->st->red_counter[RED_MISC],
                                                  &sys->st->scratch[6]);
  MD_CHECK_LAUNCH("est spme (no alloc)");
  DevState hs;
  if (int r = sys->read_state(hs)) return r;  // also keeps tab alive until the copy is done
  *err = sqrt(hs.scratch[6] * c2 * c2 / (double)sys->N);
  return MD_OK;
}

// Splitting parameter for a target real-space error: errorEstimatePME's real-space
// part is decreasing in beta, solved by bisection (FP64).
extern "C" int md_choose_beta(md_system* sys, double rcut, double target, double* beta) {
  if (!sys || !(rcut > 0) || !(target > 0) || !beta) return MD_ERR_BADARG;
  double c2;
  if (int r = charge_sq(sys, &c2)) return r;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  const double V = hs.L[0] * hs.L[1] * hs.L[2];
  auto err = [&](double b) { return 2 * sqrt(c2 / (double)sys->N) * sqrt(c2 / rcut / V) * exp(-b * b * rcut * rcut); };
  double lo = 0.0, hi = 1.0;
  while (err(hi) > target && hi < 1e6) hi *= 2;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (err(mid) > target) lo = mid; else hi = mid;
  }
  *beta = hi;
  return MD_OK;
}
