// Bonded terms and non-bonded exclusions of the interaction engine.
// Reference (shortRange.inhomo/template/tools/simulation.hetero.cutoff):
//   force functions  HarmonicSpring / FENE / FENE2   include/BondInteraction.h:217-372
//                    AngleHarmonic / CosAngle0        include/AngleInteraction.h:365-1216
//   kernels          calBondInteraction / calAngleInteraction
//                    (src/InteractionEngine_interface.cu:1399-1775)
//   topology lists   SystemBondedInteraction::reinit (src/SystemBondedInteraction.cu:100-230),
//                    BondedInteractionList / AngleList / ExclusionList
//
// Per-atom gather, as the reference: every atom sums the forces of its own bonds
// and angles (no atomics; each term is evaluated once per member atom) and adds
// them to its FP64 force.  Energies are shared 1/2 per bond end and 1/3 per
// angle member; the bond virial is 1/2 f.d per end, the angle virial is taken
// on the centre atom, -(f0 d0 - f1 d1).  The topology is kept by original atom
// id in CSR form; slot_of maps an id to its current (cell-sorted) slot and is
// refreshed by every cell sort.  The mixed path evaluates in binary32 from the
// binary32 positions (the reference's ScalorType), the FP64 path in binary64.
// Exclusions leave the neighbour list: after each list build, a pass removes
// the excluded partners from the rows of the atoms that have any, so the
// non-bonded kernels never see them (the reference tests each pair against
// the exclusion list inside the non-bonded kernel, with the same result).
#include <algorithm>
#include <cmath>
#include <vector>
#include "device_common.cuh"

namespace {

template <class R> __device__ __forceinline__ R pi_r();
template <> __device__ __forceinline__ float pi_r<float>() { return 3.14159265f; }  // M_PIF of the reference
template <> __device__ __forceinline__ double pi_r<double>() { return M_PI; }

template <class R> __device__ __forceinline__ R sqrt_r(R x);
template <> __device__ __forceinline__ float sqrt_r<float>(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double sqrt_r<double>(double x) { return sqrt(x); }
template <class R> __device__ __forceinline__ R acos_r(R x);
template <> __device__ __forceinline__ float acos_r<float>(float x) { return acosf(x); }
template <> __device__ __forceinline__ double acos_r<double>(double x) { return acos(x); }
template <class R> __device__ __forceinline__ R log_r(R x);
template <> __device__ __forceinline__ float log_r<float>(float x) { return logf(x); }
template <> __device__ __forceinline__ double log_r<double>(double x) { return log(x); }

// internal parameters from the user ones (the *::initParameter of the reference)
template <class R>
__device__ __forceinline__ void derive(int type, const double* u, R* p) {
  p[0] = (R)u[0];
  p[1] = (R)u[1];
  p[2] = (R)u[2];
  if (type == MD_BOND_FENE) p[1] = p[1] * p[1];
  else if (type == MD_BOND_FENE2) p[1] = p[1] * p[1];
  else if (type == MD_ANGLE_HARMONIC) p[1] = pi_r<R>() - p[1];
}

// bond term on the reference atom, d = r_partner - r_ref (forcePoten of the three types)
template <class R>
__device__ R bond_term(int type, const R* p, R dx, R dy, R dz, R& fx, R& fy, R& fz) {
  if (type == MD_BOND_HARMONIC) {
    R dr = dx * dx + dy * dy + dz * dz;
    const R dri = (R)(1. / (double)sqrt_r(dr));
    dr *= dri;
    const R s = p[0] * (R(1) - p[1] * dri);
    fx = dx * s; fy = dy * s; fz = dz * s;
    return R(0.5) * p[0] * (dr - p[1]) * (dr - p[1]);
  }
  if (type == MD_BOND_FENE) {
    const R dr2 = dx * dx + dy * dy + dz * dz;
    const R core = p[1] / (p[1] - dr2);
    const R s = core * p[0];
    fx = dx * s; fy = dy * s; fz = dz * s;
    const R t = R(1) / core;
    return t <= R(0) ? R(1e10) : R(-0.5) * p[0] * p[1] * log_r(t);
  }
  const R dr = sqrt_r(dx * dx + dy * dy + dz * dz);
  const R rr = dr - p[2];
  const R core = p[1] - rr * rr;
  const R s = p[0] * p[1] * rr / (core * dr);
  fx = dx * s; fy = dy * s; fz = dz * s;
  const R t = core / p[1];
  return t <= R(0) ? R(1e10) : R(-0.5) * p[0] * p[1] * log_r(t);
}

// forcePoten01 of an angle term for the difference vectors a, b
template <class R>
__device__ R angle_term(int type, const R* p, const R (&a)[3], const R (&b)[3], R (&f0)[3], R (&f1)[3]) {
  const R c00 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  const R c01 = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  const R c11 = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
  const R i0 = R(1) / sqrt_r(c00), i1 = R(1) / sqrt_r(c11);
  if (type == MD_ANGLE_COS0) {
    const R t = i0 * i1, cs = c01 * t, s = p[0] * t;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      f0[d] = s * (b[d] - c01 * i0 * i0 * a[d]);
      f1[d] = s * (-a[d] + c01 * i1 * i1 * b[d]);
    }
    return p[0] * (R(1) - cs);
  }
  R e[3], g[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    e[d] = b[d] - c01 * i0 * i0 * a[d];
    g[d] = a[d] - c01 * i1 * i1 * b[d];
  }
  R ct = c01 * i1 * i0;
  if (ct > R(1)) ct = R(1);
  const R th = acos_r(ct);
  const R s = 2 * p[0] * (th - p[1]);
#pragma unroll
  for (int d = 0; d < 3; ++d) { e[d] *= R(1e6); g[d] *= R(1e6); }
  const R t0 = sqrt_r(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
  const R t1 = sqrt_r(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  R s0 = i0 * s, s1 = i1 * s;
#pragma unroll
  for (int d = 0; d < 3; ++d) { f0[d] = R(0); f1[d] = R(0); }
  if (t0 != R(0)) {
    s0 *= (R(1) / t0);
#pragma unroll
    for (int d = 0; d < 3; ++d) f0[d] += s0 * e[d];
  } else {
    f0[0] += s0;
  }
  if (t1 != R(0)) {
    s1 *= (R(1) / t1);
#pragma unroll
    for (int d = 0; d < 3; ++d) f1[d] -= s1 * g[d];
  } else {
    f1[0] -= s1;
  }
  return p[0] * (th - p[1]) * (th - p[1]);
}

struct TopoDev {
  const int* slot_of;
  const int* b_start; const int* b_nbr; const int* b_type; const double* b_param;
  const int* a_start; const int* a_nbr; const int* a_posi; const int* a_type; const double* a_param;
};

template <class R>
__global__ void __launch_bounds__(256)
k_bonded(int N, const typename V4<R>::T* __restrict__ pos, const int* __restrict__ id, TopoDev t,
         const DevState* __restrict__ st, double4a* __restrict__ force, int with_stats, double* partials,
         unsigned* counter, double* stats) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  R L[3], Li[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { L[d] = boxL<R>(st, d); Li[d] = boxLi<R>(st, d); }
  double E = 0, V[3] = {0, 0, 0};
  if (k < N) {
    const int o = id[k];
    const typename V4<R>::T ri = pos[k];
    R F[3] = {R(0), R(0), R(0)};
    const int b1 = t.b_start ? t.b_start[o + 1] : 0;
    for (int b = t.b_start ? t.b_start[o] : 0; b < b1; ++b) {
      const typename V4<R>::T rj = pos[t.slot_of[t.b_nbr[b]]];
      R d[3] = {rj.x - ri.x, rj.y - ri.y, rj.z - ri.z};
#pragma unroll
      for (int c = 0; c < 3; ++c) d[c] = min_image_exact(d[c], L[c], Li[c]);
      R p[3], f[3];
      const int type = t.b_type[b];
      derive<R>(type, t.b_param + 3 * b, p);
      const R e = bond_term<R>(type, p, d[0], d[1], d[2], f[0], f[1], f[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        F[c] += f[c];
        V[c] += 0.5 * (double)(f[c] * d[c]);
      }
      E += 0.5 * (double)e;
    }
    const int a1 = t.a_start ? t.a_start[o + 1] : 0;
    for (int a = t.a_start ? t.a_start[o] : 0; a < a1; ++a) {
      const typename V4<R>::T p0 = pos[t.slot_of[t.a_nbr[2 * a]]];
      const typename V4<R>::T p1 = pos[t.slot_of[t.a_nbr[2 * a + 1]]];
      const bool centre = t.a_posi[a] == 1;
      R d0[3], d1[3];
      if (centre) {
        d0[0] = ri.x - p0.x; d0[1] = ri.y - p0.y; d0[2] = ri.z - p0.z;
        d1[0] = p1.x - ri.x; d1[1] = p1.y - ri.y; d1[2] = p1.z - ri.z;
      } else {
        d0[0] = p0.x - ri.x; d0[1] = p0.y - ri.y; d0[2] = p0.z - ri.z;
        d1[0] = p1.x - p0.x; d1[1] = p1.y - p0.y; d1[2] = p1.z - p0.z;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        d0[c] = min_image_exact(d0[c], L[c], Li[c]);
        d1[c] = min_image_exact(d1[c], L[c], Li[c]);
      }
      R p[3], f0[3], f1[3];
      const int type = t.a_type[a];
      derive<R>(type, t.a_param + 3 * a, p);
      const R e = angle_term<R>(type, p, d0, d1, f0, f1);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (centre) {
          F[c] += f0[c] + f1[c];
          V[c] -= (double)(f0[c] * d0[c] - f1[c] * d1[c]);
        } else {
          F[c] -= f0[c];
        }
      }
      E += (double)e / 3.0;
    }
    double4a f = force[k];
    f.x += (double)F[0];
    f.y += (double)F[1];
    f.z += (double)F[2];
    force[k] = f;
  }
  if (with_stats) {
    // virial slots are added to (the non-bonded term stored them); the bonded
    // energy slot has this kernel as its only writer and is stored
    double v[3] = {V[0], V[1], V[2]};
    block_reduce_finish<3>(v, partials, counter, stats + MD_STAT_VIRIAL_XX, false);
    double e[1] = {E};
    block_reduce_finish<1>(e, partials + 3 * (size_t)gridDim.x, counter + 1, stats + MD_STAT_BOND_ENERGY, true);
  }
}

__global__ void k_slot_of(int N, const int* __restrict__ id, int* __restrict__ slot_of, const DevState* st,
                          int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) slot_of[id[k]] = k;
}

// remove the excluded partners from the list rows of the atoms that have any
__global__ void k_nl_exclude(int N, const int* __restrict__ id, const int* __restrict__ slot_of,
                             const int* __restrict__ x_start, const int* __restrict__ x_nbr, int* list, int* nnb,
                             int cap, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int o = id[k];
  const int x0 = x_start[o], x1 = x_start[o + 1];
  if (x0 == x1) return;
  int n = nnb[k];
  if (n > cap) return;  // an overflowed row is reported and rebuilt larger
  int* row = list + (size_t)k * cap;
  for (int x = x0; x < x1; ++x) {
    const int s = slot_of[x_nbr[x]];
    for (int e = 0; e < n; ++e) {
      if ((row[nl_slot(e)] & 0x03FFFFFF) == s) {  // slot in bits 0-25, image code above
        row[nl_slot(e)] = row[nl_slot(n - 1)];
        --n;
        break;
      }
    }
  }
  nnb[k] = n;
}

}  // namespace

struct md_topo {
  int N = 0;
  int nb = 0, na = 0, nx = 0;
  int* slot_of = nullptr;
  int *b_start = nullptr, *b_nbr = nullptr, *b_type = nullptr;
  double* b_param = nullptr;
  int *a_start = nullptr, *a_nbr = nullptr, *a_posi = nullptr, *a_type = nullptr;
  double* a_param = nullptr;
  int *x_start = nullptr, *x_nbr = nullptr;
};

static void topo_free_bonds(md_topo* t) {
  void* p[] = {t->b_start, t->b_nbr, t->b_type, t->b_param};
  for (void* q : p) if (q) cudaFree(q);
  t->b_start = t->b_nbr = t->b_type = nullptr;
  t->b_param = nullptr;
  t->nb = 0;
}
static void topo_free_angles(md_topo* t) {
  void* p[] = {t->a_start, t->a_nbr, t->a_posi, t->a_type, t->a_param};
  for (void* q : p) if (q) cudaFree(q);
  t->a_start = t->a_nbr = t->a_posi = t->a_type = nullptr;
  t->a_param = nullptr;
  t->na = 0;
}
static void topo_free_excl(md_topo* t) {
  if (t->x_start) cudaFree(t->x_start);
  if (t->x_nbr) cudaFree(t->x_nbr);
  t->x_start = t->x_nbr = nullptr;
  t->nx = 0;
}

void topo_destroy(md_topo* t) {
  if (!t) return;
  topo_free_bonds(t);
  topo_free_angles(t);
  topo_free_excl(t);
  if (t->slot_of) cudaFree(t->slot_of);
  delete t;
}

bool topo_has_terms(const md_topo* t) { return t && (t->nb > 0 || t->na > 0); }

// the system's topology object, created with an identity-free slot map
static int topo_get(md_system* sys, md_topo** out) {
  if (!sys->topo) {
    md_topo* t = new md_topo();
    t->N = sys->N;
    if (cudaMalloc(&t->slot_of, sizeof(int) * sys->N) != cudaSuccess) {
      delete t;
      return md_cuda_fail(cudaGetLastError(), "topology slot map");
    }
    sys->topo = t;
    k_slot_of<<<ceil_div(sys->N, 256), 256, 0, sys->stream>>>(sys->N, sys->id, t->slot_of, sys->st, 0);
    MD_CHECK_LAUNCH("slot map");
  }
  *out = sys->topo;
  return MD_OK;
}

template <class T>
static int upload(T** dst, const std::vector<T>& v, cudaStream_t s) {
  MD_CUDA(cudaMalloc(dst, sizeof(T) * std::max<size_t>(v.size(), 1)));
  if (!v.empty()) MD_CUDA(cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  return MD_OK;
}

static bool bad_param(int type, const double* u) {
  for (int c = 0; c < 3; ++c)
    if (!std::isfinite(u[c])) return true;
  switch (type) {
    case MD_BOND_HARMONIC: return false;
    case MD_BOND_FENE: return !(u[1] > 0);
    case MD_BOND_FENE2: return !(u[1] > 0);
    case MD_ANGLE_HARMONIC: case MD_ANGLE_COS0: return false;
    default: return true;
  }
}

int topo_slot_launch(md_system* sys, Recorder* rec, bool gated) {
  if (!sys->topo) return MD_OK;
  int N = sys->N, gate = gated ? 1 : 0;
  void* a[] = {&N, &sys->id, &sys->topo->slot_of, &sys->st, &gate};
  return rec_launch(rec, (const void*)k_slot_of, dim3(ceil_div(N, 256)), dim3(256), 0, a);
}

int topo_exclude_launch(md_system* sys, md_nlist* nl, Recorder* rec, bool gated) {
  md_topo* t = sys->topo;
  if (!t || t->nx == 0) return MD_OK;
  int N = sys->N, cap = nl->cap, gate = gated ? 1 : 0;
  void* a[] = {&N, &sys->id, &t->slot_of, &t->x_start, &t->x_nbr, &nl->list, &nl->nnb, &cap, &sys->st, &gate};
  return rec_launch(rec, (const void*)k_nl_exclude, dim3(ceil_div(N, 256)), dim3(256), 0, a);
}

int bonded_apply_impl(md_system* sys, Recorder* rec, int with_stats) {
  md_topo* t = sys->topo;
  if (!topo_has_terms(t)) return MD_OK;
  int N = sys->N;
  TopoDev d{t->slot_of, t->b_start, t->b_nbr, t->b_type, t->b_param,
            t->a_start, t->a_nbr, t->a_posi, t->a_type, t->a_param};
  DevState* st = sys->st;
  double4a* f = sys->force;
  double* partials = sys->partials;
  unsigned* counter = st->red_counter + RED_BOND;
  double* stats = st->stats;
  void* a[] = {&N, &sys->pos, &sys->id, &d, &st, &f, &with_stats, &partials, &counter, &stats};
  const void* fn = sys->prec == MD_PREC_FP64 ? (const void*)k_bonded<double> : (const void*)k_bonded<float>;
  return rec_launch(rec, fn, dim3(ceil_div(N, 256)), dim3(256), 0, a);
}

// ------------------------------------------------------------------ C ABI
extern "C" int md_engine_set_bonds(md_engine* e, int n, const int* atoms, const int* type, const double* param) {
  if (!e || !e->sys || n < 0 || (n > 0 && (!atoms || !type || !param))) return MD_ERR_BADARG;
  md_system* sys = e->sys;
  const int N = sys->N;
  for (int b = 0; b < n; ++b) {
    const int i = atoms[2 * b], j = atoms[2 * b + 1];
    if (i < 0 || i >= N || j < 0 || j >= N || i == j) {
      md_set_error("md_engine_set_bonds: bond %d joins atoms %d and %d of %d", b, i, j, N);
      return MD_ERR_BADARG;
    }
    if (type[b] < MD_BOND_HARMONIC || type[b] > MD_BOND_FENE2 || bad_param(type[b], param + 3 * b)) {
      md_set_error("md_engine_set_bonds: bond %d has type %d or parameters out of range", b, type[b]);
      return MD_ERR_BADARG;
    }
  }
  MD_CUDA(cudaSetDevice(sys->device));
  md_topo* t;
  if (int r = topo_get(sys, &t)) return r;
  // per-atom entries in bond order: bond b appears under both of its atoms
  std::vector<int> start(N + 1, 0);
  for (int b = 0; b < n; ++b) { ++start[atoms[2 * b] + 1]; ++start[atoms[2 * b + 1] + 1]; }
  for (int i = 0; i < N; ++i) start[i + 1] += start[i];
  std::vector<int> fill(start.begin(), start.end() - 1), nbr(2 * n), ty(2 * n);
  std::vector<double> par(6 * (size_t)n);
  for (int b = 0; b < n; ++b)
    for (int s = 0; s < 2; ++s) {
      const int me = atoms[2 * b + s], other = atoms[2 * b + 1 - s];
      const int q = fill[me]++;
      nbr[q] = other;
      ty[q] = type[b];
      for (int c = 0; c < 3; ++c) par[3 * (size_t)q + c] = param[3 * b + c];
    }
  topo_free_bonds(t);
  if (int r = upload(&t->b_start, start, sys->stream)) return r;
  if (int r = upload(&t->b_nbr, nbr, sys->stream)) return r;
  if (int r = upload(&t->b_type, ty, sys->stream)) return r;
  if (int r = upload(&t->b_param, par, sys->stream)) return r;
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  t->nb = n;
  sys->topo_version += 1;
  e->n_bonds = n;
  return MD_OK;
}

extern "C" int md_engine_set_angles(md_engine* e, int n, const int* atoms, const int* type, const double* param) {
  if (!e || !e->sys || n < 0 || (n > 0 && (!atoms || !type || !param))) return MD_ERR_BADARG;
  md_system* sys = e->sys;
  const int N = sys->N;
  for (int a = 0; a < n; ++a) {
    const int* m = atoms + 3 * a;
    bool bad = false;
    for (int s = 0; s < 3; ++s) bad |= m[s] < 0 || m[s] >= N;
    bad |= m[0] == m[1] || m[1] == m[2] || m[0] == m[2];
    if (bad) {
      md_set_error("md_engine_set_angles: angle %d has atoms (%d, %d, %d) of %d", a, m[0], m[1], m[2], N);
      return MD_ERR_BADARG;
    }
    if ((type[a] != MD_ANGLE_HARMONIC && type[a] != MD_ANGLE_COS0) || bad_param(type[a], param + 3 * a)) {
      md_set_error("md_engine_set_angles: angle %d has type %d or parameters out of range", a, type[a]);
      return MD_ERR_BADARG;
    }
  }
  MD_CUDA(cudaSetDevice(sys->device));
  md_topo* t;
  if (int r = topo_get(sys, &t)) return r;
  // SystemBondedInteraction.cu:204-219: edge0 sees (centre, edge1) at position 0,
  // the centre (edge0, edge1) at 1, edge1 (centre, edge0) at 2
  std::vector<int> start(N + 1, 0);
  for (int a = 0; a < n; ++a)
    for (int s = 0; s < 3; ++s) ++start[atoms[3 * a + s] + 1];
  for (int i = 0; i < N; ++i) start[i + 1] += start[i];
  std::vector<int> fill(start.begin(), start.end() - 1), nbr(6 * (size_t)n), posi(3 * (size_t)n), ty(3 * (size_t)n);
  std::vector<double> par(9 * (size_t)n);
  for (int a = 0; a < n; ++a) {
    const int e0 = atoms[3 * a], c = atoms[3 * a + 1], e1 = atoms[3 * a + 2];
    const int who[3] = {e0, c, e1};
    const int t0[3] = {c, e0, c}, t1[3] = {e1, e1, e0};
    for (int s = 0; s < 3; ++s) {
      const int q = fill[who[s]]++;
      nbr[2 * (size_t)q] = t0[s];
      nbr[2 * (size_t)q + 1] = t1[s];
      posi[q] = s;
      ty[q] = type[a];
      for (int k = 0; k < 3; ++k) par[3 * (size_t)q + k] = param[3 * a + k];
    }
  }
  topo_free_angles(t);
  if (int r = upload(&t->a_start, start, sys->stream)) return r;
  if (int r = upload(&t->a_nbr, nbr, sys->stream)) return r;
  if (int r = upload(&t->a_posi, posi, sys->stream)) return r;
  if (int r = upload(&t->a_type, ty, sys->stream)) return r;
  if (int r = upload(&t->a_param, par, sys->stream)) return r;
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  t->na = n;
  sys->topo_version += 1;
  return MD_OK;
}

extern "C" int md_engine_set_exclusions(md_engine* e, int n, const int* pairs) {
  if (!e || !e->sys || n < 0 || (n > 0 && !pairs)) return MD_ERR_BADARG;
  md_system* sys = e->sys;
  const int N = sys->N;
  for (int x = 0; x < n; ++x) {
    const int i = pairs[2 * x], j = pairs[2 * x + 1];
    if (i < 0 || i >= N || j < 0 || j >= N || i == j) {
      md_set_error("md_engine_set_exclusions: pair %d is (%d, %d) of %d atoms", x, i, j, N);
      return MD_ERR_BADARG;
    }
  }
  MD_CUDA(cudaSetDevice(sys->device));
  md_topo* t;
  if (int r = topo_get(sys, &t)) return r;
  // both directions, duplicates dropped (a pair listed twice is excluded once)
  std::vector<std::vector<int>> per(N);
  for (int x = 0; x < n; ++x) {
    per[pairs[2 * x]].push_back(pairs[2 * x + 1]);
    per[pairs[2 * x + 1]].push_back(pairs[2 * x]);
  }
  std::vector<int> start(N + 1, 0), nbr;
  for (int i = 0; i < N; ++i) {
    std::sort(per[i].begin(), per[i].end());
    per[i].erase(std::unique(per[i].begin(), per[i].end()), per[i].end());
    start[i + 1] = start[i] + (int)per[i].size();
    nbr.insert(nbr.end(), per[i].begin(), per[i].end());
  }
  topo_free_excl(t);
  if (int r = upload(&t->x_start, start, sys->stream)) return r;
  if (int r = upload(&t->x_nbr, nbr, sys->stream)) return r;
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  t->nx = (int)nbr.size();
  sys->topo_version += 1;
  return MD_OK;
}

extern "C" int md_nlist_apply_exclusions(md_nlist* nl, md_system* sys) {
  if (!nl || !sys) return MD_ERR_BADARG;
  Recorder rec;
  rec.stream = sys->stream;
  if (int r = topo_exclude_launch(sys, nl, &rec, false)) return r;
  MD_CHECK_LAUNCH("exclusions");
  return MD_OK;
}

extern "C" int md_engine_apply_bonded(md_engine* e, md_system* sys) {
  if (!e || !sys || e->sys != sys) return MD_ERR_BADARG;
  Recorder rec;
  rec.stream = sys->stream;
  if (int r = bonded_apply_impl(sys, &rec, 1)) return r;
  MD_CHECK_LAUNCH("bonded");
  return MD_OK;
}
