// md_system: device SoA of the MD system, the C-ABI error channel, and the
// kernel-launch recorder used by the graph-captured driver.
// Reference: MDSystem / DeviceMDData (ENG/include/MDSystem.h:43-78,
// ENG/include/MDSystem_interface.h:18-104), normalizeSystem (ENG/src/BoxGeometry.cu:6-50).
#include <cstdarg>
#include <cmath>
#include <cstring>
#include <vector>
#include "device_common.cuh"

static thread_local char g_err[1024] = "no error";

void md_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int md_cuda_fail(cudaError_t e, const char* what) {
  md_set_error("CUDA error in %s: %s", what, cudaGetErrorString(e));
  return MD_ERR_CUDA;
}

extern "C" const char* md_last_error_message(void) { return g_err; }
extern "C" const char* md_version(void) { return "mdforce-b200 0.1 (sm_100a)"; }

extern "C" int md_device_count(int* out) {
  if (!out) return MD_ERR_BADARG;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *out = n;
  return MD_OK;
}

void box_fill(DevState& s, const double L[3]) {
  for (int d = 0; d < 3; ++d) {
    s.L[d] = L[d];
    s.Li[d] = 1.0 / L[d];
    s.Lf[d] = (float)L[d];
    s.Lif[d] = 1.0f / s.Lf[d];  // setBoxSize: box->sizei.x = 1/x in float
  }
}

int rec_launch(Recorder* r, const void* func, dim3 grid, dim3 block, size_t smem, void** args) {
  if (r && r->graph) {
    cudaKernelNodeParams p;
    memset(&p, 0, sizeof(p));
    p.func = const_cast<void*>(func);
    p.gridDim = grid;
    p.blockDim = block;
    p.sharedMemBytes = (unsigned)smem;
    p.kernelParams = args;
    p.extra = nullptr;
    cudaGraphNode_t node, deps[2];
    size_t nd = 0;
    if (r->has_last) deps[nd++] = r->last;
    if (r->join) deps[nd++] = r->join;
    MD_CUDA(cudaGraphAddKernelNode(&node, r->graph, nd ? deps : nullptr, nd, &p));
    r->last = node;
    r->has_last = true;
    r->join = nullptr;
    return MD_OK;
  }
  cudaStream_t s = r ? r->stream : nullptr;
  MD_CUDA(cudaLaunchKernel(func, grid, block, args, smem, s));
  return MD_OK;
}

int rec_launch_coop(Recorder* r, const void* func, dim3 grid, dim3 block, size_t smem, void** args) {
  if (r && r->graph) {
    if (int e = rec_launch(r, func, grid, block, smem, args)) return e;
    cudaLaunchAttributeValue v;
    memset(&v, 0, sizeof(v));
    v.cooperative = 1;
    MD_CUDA(cudaGraphKernelNodeSetAttribute(r->last, cudaLaunchAttributeCooperative, &v));
    return MD_OK;
  }
  cudaStream_t s = r ? r->stream : nullptr;
  MD_CUDA(cudaLaunchCooperativeKernel(func, grid, block, args, smem, s));
  return MD_OK;
}

int md_system::read_state(DevState& s) {
  MD_CUDA(cudaMemcpyAsync(&s, st, sizeof(DevState), cudaMemcpyDeviceToHost, stream));
  MD_CUDA(cudaStreamSynchronize(stream));
  return MD_OK;
}

// ------------------------------------------------------------------ kernels
template <class R>
__global__ void k_upload(int N, const double* pos, const double* vel, const double* q,
                         const double* m, typename V4<R>::T* p4, typename V4<R>::T* v4,
                         int* id, int4* image, double4a* f, float* rcut) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  typename V4<R>::T a, b;
  a.x = (R)pos[3 * i]; a.y = (R)pos[3 * i + 1]; a.z = (R)pos[3 * i + 2];
  a.w = q ? (R)q[i] : R(0);
  b.x = vel ? (R)vel[3 * i] : R(0);
  b.y = vel ? (R)vel[3 * i + 1] : R(0);
  b.z = vel ? (R)vel[3 * i + 2] : R(0);
  b.w = m ? (R)(1.0 / m[i]) : R(1);
  p4[i] = a;
  v4[i] = b;
  id[i] = i;
  image[i] = make_int4(0, 0, 0, 0);
  f[i] = double4a{0, 0, 0, 0};
  rcut[i] = 0.f;
}

// out[id[k]] = field(k): un-permute to original order
template <class R>
__global__ void k_download(int N, int what, const typename V4<R>::T* p4, const typename V4<R>::T* v4,
                           const double4a* f, const int4* image, const int* id,
                           const DevState* st, double* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  int o = id[k];
  double x, y, z;
  if (what == 0 || what == 3) {
    typename V4<R>::T a = p4[k];
    x = a.x; y = a.y; z = a.z;
    if (what == 3) {
      int4 im = image[k];
      x += im.x * st->L[0]; y += im.y * st->L[1]; z += im.z * st->L[2];
    }
  } else if (what == 1) {
    typename V4<R>::T a = v4[k];
    x = a.x; y = a.y; z = a.z;
  } else {
    double4a a = f[k];
    x = a.x; y = a.y; z = a.z;
  }
  out[3 * o] = x; out[3 * o + 1] = y; out[3 * o + 2] = z;
}

template <class R>
__global__ void k_set_vec(int N, int what, const double* in, const int* id,
                          typename V4<R>::T* p4, typename V4<R>::T* v4) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  int o = id[k];
  typename V4<R>::T* dst = (what == 0) ? p4 : v4;
  typename V4<R>::T a = dst[k];
  a.x = (R)in[3 * o]; a.y = (R)in[3 * o + 1]; a.z = (R)in[3 * o + 2];
  dst[k] = a;
}

// md_system_set_device_view: positions [N][3] and / or charges [N] from device
// memory in the caller's atom order into the cell-ordered arrays
template <class R>
__global__ void k_set_view(int N, const double* __restrict__ pos, const double* __restrict__ q, const int* id,
                           typename V4<R>::T* p4) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const int o = id[k];
  typename V4<R>::T a = p4[k];
  if (pos) { a.x = (R)pos[3 * o]; a.y = (R)pos[3 * o + 1]; a.z = (R)pos[3 * o + 2]; }
  if (q) a.w = (R)q[o];
  p4[k] = a;
}

// charges live in the w component of the position array
template <class R>
__global__ void k_charge_io(int N, int dir, typename V4<R>::T* p4, const int* id, double* host_order) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  if (dir == 0) p4[k].w = (R)host_order[id[k]];
  else host_order[id[k]] = (double)p4[k].w;
}

// masses live in vel.w as 1/m (MDSystem hdata.massi); m given and returned in
// original atom order
template <class R>
__global__ void k_mass_io(int N, int dir, typename V4<R>::T* v4, const int* id, double* host_order) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  if (dir == 0) v4[k].w = (R)(1.0 / host_order[id[k]]);
  else host_order[id[k]] = 1.0 / (double)v4[k].w;
}

__global__ void k_rcut_io(int N, int dir, float* rc, const int* id, float* host_order) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  if (dir == 0) rc[k] = host_order[id[k]];
  else host_order[id[k]] = rc[k];
}

// normalizeSystem / moveParticleToBox (ENG/include/BoxGeometry.h:80-96):
// tmp = floorf(x*sizei); noi += tmp; x -= tmp*size, in binary32 without contraction
template <class R>
__global__ void k_normalize(int N, typename V4<R>::T* p4, int4* image, const DevState* st) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  typename V4<R>::T a = p4[k];
  int4 im = image[k];
  R t;
  t = floor_r(mul_rn(a.x, boxLi<R>(st, 0))); im.x += (int)t; a.x = sub_rn(a.x, mul_rn(t, boxL<R>(st, 0)));
  t = floor_r(mul_rn(a.y, boxLi<R>(st, 1))); im.y += (int)t; a.y = sub_rn(a.y, mul_rn(t, boxL<R>(st, 1)));
  t = floor_r(mul_rn(a.z, boxLi<R>(st, 2))); im.z += (int)t; a.z = sub_rn(a.z, mul_rn(t, boxL<R>(st, 2)));
  p4[k] = a;
  image[k] = im;
}

__global__ void k_clear_stats(DevState* st, int first, int count) {
  int t = threadIdx.x;
  if (t < count) st->stats[first + t] = 0.0;
}

__global__ void k_set_flag(DevState* st, unsigned bits) { st->flags |= bits; }

int clear_stats_impl(md_system* sys, Recorder* rec, int first, int count) {
  DevState* st = sys->st;
  void* args[] = {&st, &first, &count};
  return rec_launch(rec, (const void*)k_clear_stats, dim3(1), dim3(32), 0, args);
}

int set_flag_impl(md_system* sys, unsigned bits, Recorder* rec) {
  DevState* st = sys->st;
  void* args[] = {&st, &bits};
  return rec_launch(rec, (const void*)k_set_flag, dim3(1), dim3(1), 0, args);
}

// ------------------------------------------------------------------ C ABI
static int check_sys(const md_system* s) {
  if (!s) { md_set_error("null md_system"); return MD_ERR_BADARG; }
  return MD_OK;
}

static int ensure_stage(md_system* s, size_t bytes) {
  if (s->h_stage_bytes >= bytes) return MD_OK;
  if (s->h_stage) cudaFreeHost(s->h_stage);
  s->h_stage = nullptr;
  s->h_stage_bytes = 0;
  MD_CUDA(cudaMallocHost(&s->h_stage, bytes));
  s->h_stage_bytes = bytes;
  return MD_OK;
}

__global__ void k_type_slot(int N, const int* __restrict__ id, const uint8_t* __restrict__ by_id,
                            uint8_t* __restrict__ by_slot, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) by_slot[k] = by_id[id[k]];
}

int types_slot_launch(md_system* sys, Recorder* rec, bool gated) {
  if (sys->ntypes <= 1) return MD_OK;  // every slot holds type 0
  int N = sys->N, gate = gated ? 1 : 0;
  void* a[] = {&N, &sys->id, &sys->type_by_id, &sys->type, &sys->st, &gate};
  return rec_launch(rec, (const void*)k_type_slot, dim3(ceil_div(N, 256)), dim3(256), 0, a);
}

extern "C" int md_system_set_types(md_system* s, const int* type) {
  if (!s || !type) return MD_ERR_BADARG;
  int nt = 1;
  for (int i = 0; i < s->N; ++i) {
    if (type[i] < 0 || type[i] >= MD_MAX_TYPES) {
      md_set_error("md_system_set_types: atom %d has type %d (0 <= type < %d)", i, type[i], MD_MAX_TYPES);
      return MD_ERR_BADARG;
    }
    if (type[i] + 1 > nt) nt = type[i] + 1;
  }
  std::vector<uint8_t> t8(type, type + s->N);
  MD_CUDA(cudaSetDevice(s->device));
  MD_CUDA(cudaMemcpyAsync(s->type_by_id, t8.data(), s->N, cudaMemcpyHostToDevice, s->stream));
  s->ntypes = nt;
  k_type_slot<<<ceil_div(s->N, 256), 256, 0, s->stream>>>(s->N, s->id, s->type_by_id, s->type, s->st, 0);
  MD_CHECK_LAUNCH("types");
  MD_CUDA(cudaStreamSynchronize(s->stream));
  s->topo_version += 1;
  return MD_OK;
}

extern "C" int md_system_get_types(md_system* s, int* type) {
  if (!s || !type) return MD_ERR_BADARG;
  std::vector<uint8_t> t8(s->N);
  MD_CUDA(cudaMemcpyAsync(t8.data(), s->type_by_id, s->N, cudaMemcpyDeviceToHost, s->stream));
  MD_CUDA(cudaStreamSynchronize(s->stream));
  for (int i = 0; i < s->N; ++i) type[i] = t8[i];
  return MD_OK;
}

extern "C" int md_system_create(md_system** out, int n, const double box[3], const double* pos,
                                const double* vel, const int* type, const double* charge,
                                const double* mass, int precision, int device) {
  if (!out || n <= 0 || !box || !pos) { md_set_error("md_system_create: bad arguments"); return MD_ERR_BADARG; }
  if (type)
    for (int i = 0; i < n; ++i)
      if (type[i] < 0 || type[i] >= MD_MAX_TYPES) {
        md_set_error("md_system_create: atom %d has type %d (0 <= type < %d)", i, type[i], MD_MAX_TYPES);
        return MD_ERR_BADARG;
      }
  if (precision != MD_PREC_MIXED && precision != MD_PREC_FP64) { md_set_error("bad precision %d", precision); return MD_ERR_BADARG; }
  for (int d = 0; d < 3; ++d)
    if (!(box[d] > 0) || !std::isfinite(box[d])) { md_set_error("md_system_create: bad box"); return MD_ERR_BADARG; }
  for (long long i = 0; i < 3LL * n; ++i)
    if (!std::isfinite(pos[i])) { md_set_error("md_system_create: non-finite position at %lld", i / 3); return MD_ERR_BADARG; }
  if (mass)
    for (int i = 0; i < n; ++i)
      if (!(mass[i] > 0)) { md_set_error("md_system_create: non-positive mass at %d", i); return MD_ERR_BADARG; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    md_set_error("md_system_create: no CUDA device available");
    return MD_ERR_CUDA;
  }
  MD_CUDA(cudaSetDevice(device));
  md_system* s = new md_system();
  s->N = n;
  s->prec = precision;
  s->device = device;
  int rc = MD_OK;
  auto fail = [&](int code) { md_system_destroy(s); return code; };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "stream"));
  s->own_stream = true;
  size_t r4 = s->r4_size();
#define ALLOC(p, bytes) if (cudaMalloc((void**)&(p), (bytes)) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "cudaMalloc " #p))
  ALLOC(s->pos, r4 * n); ALLOC(s->vel, r4 * n); ALLOC(s->force, sizeof(double4a) * n);
  ALLOC(s->image, sizeof(int4) * n); ALLOC(s->id, sizeof(int) * n); ALLOC(s->rcut, sizeof(float) * n);
  ALLOC(s->t_pos, r4 * n); ALLOC(s->t_vel, r4 * n); ALLOC(s->t_force, sizeof(double4a) * n);
  ALLOC(s->t_image, sizeof(int4) * n); ALLOC(s->t_id, sizeof(int) * n); ALLOC(s->t_rcut, sizeof(float) * n);
  ALLOC(s->st, sizeof(DevState));
  s->max_partial_blocks = ceil_div((long long)n * 32, 128) + 1024;
  ALLOC(s->partials, sizeof(double) * 8 * (size_t)s->max_partial_blocks);
  // one row of 5 per warp of the non-bonded kernels (8 lanes per atom)
  ALLOC(s->nb_rows, sizeof(double) * 5 * ((size_t)n / 4 + 1024));
  ALLOC(s->type_by_id, (size_t)n); ALLOC(s->type, (size_t)n);
#undef ALLOC
  DevState hs;
  memset(&hs, 0, sizeof(hs));
  box_fill(hs, box);
  for (int d = 0; d < 3; ++d) { hs.lam1[d] = hs.lam2[d] = 1.0; }
  if (cudaMemcpy(s->st, &hs, sizeof(hs), cudaMemcpyHostToDevice) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "state upload"));
  // stage inputs through device buffers
  size_t bytes = sizeof(double) * (3ull * n * 2 + 2ull * n);
  double* dbuf = nullptr;
  if (cudaMalloc(&dbuf, bytes) != cudaSuccess) return fail(md_cuda_fail(cudaGetLastError(), "stage"));
  double* dpos = dbuf;
  double* dvel = dbuf + 3ull * n;
  double* dq = dbuf + 6ull * n;
  double* dm = dbuf + 7ull * n;
  cudaMemcpy(dpos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
  if (vel) cudaMemcpy(dvel, vel, sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
  if (charge) cudaMemcpy(dq, charge, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (mass) cudaMemcpy(dm, mass, sizeof(double) * n, cudaMemcpyHostToDevice);
  const double* pv = vel ? dvel : nullptr;
  const double* pq = charge ? dq : nullptr;
  const double* pm = mass ? dm : nullptr;
  int nb = ceil_div(n, 256);
  if (s->prec == MD_PREC_FP64)
    k_upload<double><<<nb, 256, 0, s->stream>>>(n, dpos, pv, pq, pm, (double4a*)s->pos, (double4a*)s->vel, s->id, s->image, s->force, s->rcut);
  else
    k_upload<float><<<nb, 256, 0, s->stream>>>(n, dpos, pv, pq, pm, (float4*)s->pos, (float4*)s->vel, s->id, s->image, s->force, s->rcut);
  cudaMemsetAsync(s->type_by_id, 0, (size_t)n, s->stream);
  cudaMemsetAsync(s->type, 0, (size_t)n, s->stream);
  cudaError_t e = cudaStreamSynchronize(s->stream);
  cudaFree(dbuf);
  if (e != cudaSuccess) return fail(md_cuda_fail(e, "upload"));
  if (type)
    if (int r = md_system_set_types(s, type)) return fail(r);
  s->topo_version = 0;
  rc = MD_OK;
  *out = s;
  return rc;
}

extern "C" int md_system_destroy(md_system* s) {
  if (!s) return MD_OK;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  void* ptrs[] = {s->pos, s->vel, s->force, s->image, s->id, s->rcut, s->t_pos, s->t_vel,
                  s->t_force, s->t_image, s->t_id, s->t_rcut, s->st, s->partials, s->nb_rows, s->d_lattice,
                  s->type_by_id, s->type};
  for (void* p : ptrs) if (p) cudaFree(p);
  topo_destroy(s->topo);
  if (s->h_stage) cudaFreeHost(s->h_stage);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return MD_OK;
}

extern "C" int md_system_set_stream(md_system* s, void* stream) {
  if (int r = check_sys(s)) return r;
  MD_CUDA(cudaStreamSynchronize(s->stream));
  if (stream) {
    if (s->own_stream) cudaStreamDestroy(s->stream);
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
  } else if (!s->own_stream) {
    MD_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  return MD_OK;
}

extern "C" int md_system_synchronize(md_system* s) {
  if (int r = check_sys(s)) return r;
  MD_CUDA(cudaStreamSynchronize(s->stream));
  DevState hs;
  if (int r = s->read_state(hs)) return r;
  if (hs.flags & FLAG_NAN) { md_set_error("non-finite coordinates detected"); return MD_ERR_BADARG; }
  return MD_OK;
}

extern "C" int md_system_num_atoms(const md_system* s, int* out) {
  if (int r = check_sys(s)) return r;
  if (!out) return MD_ERR_BADARG;
  *out = s->N;
  return MD_OK;
}

static int download(md_system* s, int what, double* out) {
  if (int r = check_sys(s)) return r;
  if (!out) return MD_ERR_BADARG;
  size_t bytes = sizeof(double) * 3 * (size_t)s->N;
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, bytes, s->stream));
  int nb = ceil_div(s->N, 256);
  if (s->prec == MD_PREC_FP64)
    k_download<double><<<nb, 256, 0, s->stream>>>(s->N, what, (double4a*)s->pos, (double4a*)s->vel, s->force, s->image, s->id, s->st, d);
  else
    k_download<float><<<nb, 256, 0, s->stream>>>(s->N, what, (float4*)s->pos, (float4*)s->vel, s->force, s->image, s->id, s->st, d);
  MD_CHECK_LAUNCH("download");
  if (int r = ensure_stage(s, bytes)) return r;
  MD_CUDA(cudaMemcpyAsync(s->h_stage, d, bytes, cudaMemcpyDeviceToHost, s->stream));
  MD_CUDA(cudaFreeAsync(d, s->stream));
  MD_CUDA(cudaStreamSynchronize(s->stream));
  memcpy(out, s->h_stage, bytes);
  return MD_OK;
}

static int upload_vec(md_system* s, int what, const double* in) {
  if (int r = check_sys(s)) return r;
  if (!in) return MD_ERR_BADARG;
  for (long long i = 0; i < 3LL * s->N; ++i)
    if (!std::isfinite(in[i])) { md_set_error("non-finite input at atom %lld", i / 3); return MD_ERR_BADARG; }
  size_t bytes = sizeof(double) * 3 * (size_t)s->N;
  if (int r = ensure_stage(s, bytes)) return r;
  MD_CUDA(cudaStreamSynchronize(s->stream));
  memcpy(s->h_stage, in, bytes);
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, bytes, s->stream));
  MD_CUDA(cudaMemcpyAsync(d, s->h_stage, bytes, cudaMemcpyHostToDevice, s->stream));
  int nb = ceil_div(s->N, 256);
  if (s->prec == MD_PREC_FP64)
    k_set_vec<double><<<nb, 256, 0, s->stream>>>(s->N, what, d, s->id, (double4a*)s->pos, (double4a*)s->vel);
  else
    k_set_vec<float><<<nb, 256, 0, s->stream>>>(s->N, what, d, s->id, (float4*)s->pos, (float4*)s->vel);
  MD_CHECK_LAUNCH("set vec");
  MD_CUDA(cudaFreeAsync(d, s->stream));
  MD_CUDA(cudaStreamSynchronize(s->stream));
  return MD_OK;
}

extern "C" int md_system_set_positions(md_system* s, const double* pos) { return upload_vec(s, 0, pos); }
extern "C" int md_system_get_positions(md_system* s, double* pos) { return download(s, 0, pos); }
extern "C" int md_system_get_unwrapped_positions(md_system* s, double* pos) { return download(s, 3, pos); }
extern "C" int md_system_set_velocities(md_system* s, const double* v) { return upload_vec(s, 1, v); }
extern "C" int md_system_get_velocities(md_system* s, double* v) { return download(s, 1, v); }
extern "C" int md_system_get_forces(md_system* s, double* f) { return download(s, 2, f); }

// per-atom scalar kept in a w component: what 0 charge (pos.w), 1 mass (vel.w = 1/m)
static int charge_io(md_system* s, int dir, double* q, int what = 0) {
  if (int r = check_sys(s)) return r;
  if (!q) return MD_ERR_BADARG;
  if (dir == 0)
    for (int i = 0; i < s->N; ++i) {
      if (!std::isfinite(q[i])) { md_set_error("non-finite %s at atom %d", what ? "mass" : "charge", i); return MD_ERR_BADARG; }
      if (what == 1 && !(q[i] > 0)) { md_set_error("mass %g of atom %d is not positive", q[i], i); return MD_ERR_BADARG; }
    }
  const size_t bytes = sizeof(double) * (size_t)s->N;
  if (int r = ensure_stage(s, bytes)) return r;
  MD_CUDA(cudaStreamSynchronize(s->stream));
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, bytes, s->stream));
  if (dir == 0) {
    memcpy(s->h_stage, q, bytes);
    MD_CUDA(cudaMemcpyAsync(d, s->h_stage, bytes, cudaMemcpyHostToDevice, s->stream));
  }
  const int nb = ceil_div(s->N, 256);
  if (what == 1) {
    if (s->prec == MD_PREC_FP64)
      k_mass_io<double><<<nb, 256, 0, s->stream>>>(s->N, dir, (double4a*)s->vel, s->id, d);
    else
      k_mass_io<float><<<nb, 256, 0, s->stream>>>(s->N, dir, (float4*)s->vel, s->id, d);
  } else if (s->prec == MD_PREC_FP64) {
    k_charge_io<double><<<nb, 256, 0, s->stream>>>(s->N, dir, (double4a*)s->pos, s->id, d);
  } else {
    k_charge_io<float><<<nb, 256, 0, s->stream>>>(s->N, dir, (float4*)s->pos, s->id, d);
  }
  MD_CHECK_LAUNCH("charge / mass io");
  if (dir == 1) MD_CUDA(cudaMemcpyAsync(s->h_stage, d, bytes, cudaMemcpyDeviceToHost, s->stream));
  MD_CUDA(cudaFreeAsync(d, s->stream));
  MD_CUDA(cudaStreamSynchronize(s->stream));
  if (dir == 1) memcpy(q, s->h_stage, bytes);
  return MD_OK;
}

// Zero-copy input from device tensors: no host copy, no wait; the caller's
// stream must be the system's (md_system_set_stream) or be ordered with it.
extern "C" int md_system_set_device_view(md_system* s, const md_device_view* v) {
  if (int r = check_sys(s)) return r;
  if (!v) return MD_ERR_BADARG;
  if (!v->pos && !v->charge) return MD_OK;
  const int nb = ceil_div(s->N, 256);
  if (s->prec == MD_PREC_FP64)
    k_set_view<double><<<nb, 256, 0, s->stream>>>(s->N, v->pos, v->charge, s->id, (double4a*)s->pos);
  else
    k_set_view<float><<<nb, 256, 0, s->stream>>>(s->N, v->pos, v->charge, s->id, (float4*)s->pos);
  MD_CHECK_LAUNCH("device view");
  return MD_OK;
}

extern "C" int md_system_set_charges(md_system* s, const double* q) { return charge_io(s, 0, const_cast<double*>(q)); }
extern "C" int md_system_get_charges(md_system* s, double* q) { return charge_io(s, 1, q); }
extern "C" int md_system_set_masses(md_system* s, const double* m) { return charge_io(s, 0, const_cast<double*>(m), 1); }
extern "C" int md_system_get_masses(md_system* s, double* m) { return charge_io(s, 1, m, 1); }

extern "C" int md_system_get_box(md_system* s, double box[3]) {
  if (int r = check_sys(s)) return r;
  DevState hs;
  if (int r = s->read_state(hs)) return r;
  for (int d = 0; d < 3; ++d) box[d] = hs.L[d];
  return MD_OK;
}

extern "C" int md_system_set_box(md_system* s, const double box[3]) {
  if (int r = check_sys(s)) return r;
  for (int d = 0; d < 3; ++d)
    if (!(box[d] > 0) || !std::isfinite(box[d])) { md_set_error("bad box"); return MD_ERR_BADARG; }
  DevState hs;
  if (int r = s->read_state(hs)) return r;
  box_fill(hs, box);
  MD_CUDA(cudaMemcpyAsync(s->st, &hs, sizeof(hs), cudaMemcpyHostToDevice, s->stream));
  MD_CUDA(cudaStreamSynchronize(s->stream));
  return MD_OK;
}

static int rcut_io(md_system* s, int dir, float* host) {
  if (int r = check_sys(s)) return r;
  if (!host) return MD_ERR_BADARG;
  float* d = nullptr;
  size_t bytes = sizeof(float) * s->N;
  MD_CUDA(cudaMallocAsync((void**)&d, bytes, s->stream));
  if (dir == 0) MD_CUDA(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, s->stream));
  k_rcut_io<<<ceil_div(s->N, 256), 256, 0, s->stream>>>(s->N, dir, s->rcut, s->id, d);
  MD_CHECK_LAUNCH("rcut io");
  if (dir == 1) MD_CUDA(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, s->stream));
  MD_CUDA(cudaFreeAsync(d, s->stream));
  MD_CUDA(cudaStreamSynchronize(s->stream));
  return MD_OK;
}
extern "C" int md_system_set_rcut(md_system* s, const float* rc) { return rcut_io(s, 0, const_cast<float*>(rc)); }
extern "C" int md_system_get_rcut(md_system* s, float* rc) { return rcut_io(s, 1, rc); }

extern "C" int md_system_normalize(md_system* s) {
  if (int r = check_sys(s)) return r;
  int nb = ceil_div(s->N, 256);
  if (s->prec == MD_PREC_FP64)
    k_normalize<double><<<nb, 256, 0, s->stream>>>(s->N, (double4a*)s->pos, s->image, s->st);
  else
    k_normalize<float><<<nb, 256, 0, s->stream>>>(s->N, (float4*)s->pos, s->image, s->st);
  MD_CHECK_LAUNCH("normalize");
  return MD_OK;
}

extern "C" int md_system_read_stats(md_system* s, double* out) {
  if (int r = check_sys(s)) return r;
  if (!out) return MD_ERR_BADARG;
  DevState hs;
  if (int r = s->read_state(hs)) return r;
  memcpy(out, hs.stats, sizeof(double) * MD_STAT_COUNT);
  return MD_OK;
}

extern "C" int md_system_read_stats_async(md_system* s, double* out) {
  if (int r = check_sys(s)) return r;
  if (!out) return MD_ERR_BADARG;
  MD_CUDA(cudaMemcpyAsync(out, s->st->stats, sizeof(double) * MD_STAT_COUNT, cudaMemcpyDeviceToHost,
                          s->stream));
  return MD_OK;
}

extern "C" int md_system_clear_stats(md_system* s) {
  if (int r = check_sys(s)) return r;
  Recorder rec;
  rec.stream = s->stream;
  return clear_stats_impl(s, &rec, 0, MD_STAT_COUNT);
}
