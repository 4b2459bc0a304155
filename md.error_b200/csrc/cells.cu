// Cell binning and cell-order sort.
// Reference: CellList::DecideNumCell (UNI/src/CellList_interface.cu:147-177),
// naivelyBuildDeviceCellList2 (ENG/src/NeighborList.cu:84-167), the Reshuffle
// permutation (ENG/src/Reshuffle_interface.cu:40-102) and AssignRCut
// (ENG/src/AssignRCut.cu:78-117), which is fused into the gather.
//
// Rebuild = 5 kernels:
//   bin      normalise into the box (moveParticleToBox), cell index with the
//            reference's binary32 formula, warp-aggregated atomic count
//   scan     exclusive scan of the per-cell counts (one block), clears counts
//   scatter  member lists from the atomic ranks
//   order    rank members of each cell by their previous slot (warp per cell),
//            which makes the permutation deterministic
//   gather   permute every per-atom array into cell order (+ per-atom rcut
//            from the lattice when one is set)
// then a copy back into the primary arrays.
#include <cmath>
#include <cstring>
#include "device_common.cuh"

struct CellGeom {
  int nc[3];
  int ntot;
};

// binary32 cell index: IndexType(coord.x * box.sizei.x * ScalorType(NCell.x));
// __float2uint_rz is the saturating conversion the reference's cast compiles to.
template <class R>
__device__ __forceinline__ unsigned cell_coord(R x, R Li, int nc);
template <>
__device__ __forceinline__ unsigned cell_coord<float>(float x, float Li, int nc) {
  return __float2uint_rz(__fmul_rn(__fmul_rn(x, Li), (float)nc));
}
template <>
__device__ __forceinline__ unsigned cell_coord<double>(double x, double Li, int nc) {
  return __double2uint_rz(__dmul_rn(__dmul_rn(x, Li), (double)nc));
}

template <class R>
__global__ void k_bin(int N, typename V4<R>::T* pos, int4* image, DevState* st, CellGeom g,
                      uint32_t* t_cell, uint32_t* slot, uint32_t* count, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < N;
  unsigned cell = 0xffffffffu;
  if (valid) {
    typename V4<R>::T a = pos[i];
    int4 im = image[i];
    const R L0 = boxL<R>(st, 0), L1 = boxL<R>(st, 1), L2 = boxL<R>(st, 2);
    const R I0 = boxLi<R>(st, 0), I1 = boxLi<R>(st, 1), I2 = boxLi<R>(st, 2);
    bool finite = isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
    if (!finite) {
      atomicOr(&st->flags, FLAG_NAN);
      cell = 0;
    } else {
      // moveParticleToBox
      R t;
      t = floor_r(mul_rn(a.x, I0)); im.x += (int)t; a.x = sub_rn(a.x, mul_rn(t, L0));
      t = floor_r(mul_rn(a.y, I1)); im.y += (int)t; a.y = sub_rn(a.y, mul_rn(t, L1));
      t = floor_r(mul_rn(a.z, I2)); im.z += (int)t; a.z = sub_rn(a.z, mul_rn(t, L2));
      unsigned cx = cell_coord<R>(a.x, I0, g.nc[0]);
      unsigned cy = cell_coord<R>(a.y, I1, g.nc[1]);
      unsigned cz = cell_coord<R>(a.z, I2, g.nc[2]);
      // wrap fix of naivelyBuildDeviceCellList2 (NeighborList.cu:110-124)
      if (cx == (unsigned)g.nc[0]) { cx -= g.nc[0]; a.x = sub_rn(a.x, L0); im.x++; }
      if (cy == (unsigned)g.nc[1]) { cy -= g.nc[1]; a.y = sub_rn(a.y, L1); im.y++; }
      if (cz == (unsigned)g.nc[2]) { cz -= g.nc[2]; a.z = sub_rn(a.z, L2); im.z++; }
      if (cx >= (unsigned)g.nc[0] || cy >= (unsigned)g.nc[1] || cz >= (unsigned)g.nc[2]) {
        atomicOr(&st->flags, FLAG_CELL_INDEX);
        cx = min(cx, (unsigned)g.nc[0] - 1); cy = min(cy, (unsigned)g.nc[1] - 1); cz = min(cz, (unsigned)g.nc[2] - 1);
      }
      cell = cz + (unsigned)g.nc[2] * (cy + (unsigned)g.nc[1] * cx);  // D3toD1
      pos[i] = a;
      image[i] = im;
    }
  }
  // warp-aggregated atomic insertion: one atomic per distinct cell per warp
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(active, cell);
  const int leader = __ffs(peers) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(&count[cell], (unsigned)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  slot[i] = base + __popc(peers & ((1u << lane) - 1u));
  t_cell[i] = cell;
}

// single-block exclusive scan (1024 threads, each owns a contiguous chunk);
// zeroes count for the next rebuild
__global__ void __launch_bounds__(1024) k_scan(int n, uint32_t* count, uint32_t* start, DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  // exclusive scan of the cell counts (and their reset) in tiles of 4T cells:
  // thread t of a tile holds cells 4t..4t+3, so each warp reads and writes
  // 512 contiguous bytes; the running total carries from tile to tile
  __shared__ uint32_t wsum[32];
  const int T = blockDim.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = T >> 5;
  uint32_t carry = 0;
  // cells 4t..4t+3 of a tile as one 16-byte load (count and start come from
  // cudaMalloc, so 4t is 16-byte aligned), the next tile's loaded early
  auto load4 = [&](int i0, uint32_t v[4]) {
    if (i0 + 3 < n) {
      const uint4 q = *reinterpret_cast<const uint4*>(count + i0);
      v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] = (i0 + k < n) ? count[i0 + k] : 0u;
    }
  };
  uint32_t nxt[4];
  load4(4 * threadIdx.x, nxt);
  for (int base = 0; base < n; base += 4 * T) {
    const int i0 = base + 4 * threadIdx.x;
    uint32_t v[4] = {nxt[0], nxt[1], nxt[2], nxt[3]};
    if (base + 4 * T < n) load4(i0 + 4 * T, nxt);
    const uint32_t tot = v[0] + v[1] + v[2] + v[3];
    uint32_t x = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t w = lane < nw ? wsum[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    uint32_t run = carry + (wid > 0 ? wsum[wid - 1] : 0u) + x - tot;
    if (i0 + 3 < n) {
      const uint4 st4 = make_uint4(run, run + v[0], run + v[0] + v[1], run + v[0] + v[1] + v[2]);
      *reinterpret_cast<uint4*>(start + i0) = st4;
      *reinterpret_cast<uint4*>(count + i0) = make_uint4(0u, 0u, 0u, 0u);
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (i0 + k < n) {
          start[i0 + k] = run;
          count[i0 + k] = 0u;
        }
        run += v[k];
      }
    }
    carry += wsum[nw - 1];
    __syncthreads();  // wsum is rewritten by the next tile
  }
  if (threadIdx.x == 0) start[n] = carry;
}

__global__ void k_scatter(int N, const uint32_t* t_cell, const uint32_t* slot, const uint32_t* start,
                          uint32_t* members, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  members[start[t_cell[i]] + slot[i]] = (uint32_t)i;
}

// warp per cell: rank each member by its previous slot (ascending)
// Members of a cell are ranked by (cutoff, previous slot): atoms of equal
// cutoff (hence similar list length) become neighbours in memory, so the
// force kernel's warps, which take consecutive atoms, see rows of similar
// length; the previous slot breaks ties, so the order is deterministic.
__global__ void k_order(int ntot, const uint32_t* start, const uint32_t* members, const float* rcut,
                        uint32_t* perm, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= ntot) return;
  const uint32_t s = start[warp], n = start[warp + 1] - s;
  auto key = [&](uint32_t e) -> unsigned long long {
    return ((unsigned long long)__float_as_uint(rcut[e]) << 32) | e;  // rcut >= 0 orders as its bits
  };
  for (uint32_t b = 0; b < n; b += 32) {
    const uint32_t e = (b + lane < n) ? members[s + b + lane] : 0xffffffffu;
    const unsigned long long ke = (b + lane < n) ? key(e) : ~0ull;
    uint32_t rank = 0;
    for (uint32_t b2 = 0; b2 < n; b2 += 32) {
      const unsigned long long v = (b2 + lane < n) ? key(members[s + b2 + lane]) : ~0ull;
#pragma unroll 8
      for (int t = 0; t < 32; ++t) {
        const unsigned long long vt = __shfl_sync(0xffffffffu, v, t);
        rank += (vt < ke) ? 1u : 0u;
      }
    }
    if (b + lane < n) perm[s + rank] = e;
  }
}

// warp per cell, after the gather: the cell's slots ranked by (z, slot), so
// that each cell's z order is at zord[start[c] ..] (slot order itself stays by
// cutoff for the force kernel)
template <class R>
__global__ void k_zorder(int ntot, const uint32_t* start, const typename V4<R>::T* pos, uint32_t* zord,
                         const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= ntot) return;
  const uint32_t s = start[warp], n = start[warp + 1] - s;
  for (uint32_t b = 0; b < n; b += 32) {
    const bool on = b + lane < n;
    const uint32_t e = on ? s + b + lane : 0u;
    const R ze = on ? pos[e].z : R(0);
    uint32_t rank = 0;
    for (uint32_t b2 = 0; b2 < n; b2 += 32) {
      const bool on2 = b2 + lane < n;
      const uint32_t e2 = on2 ? s + b2 + lane : 0xffffffffu;
      const R z2 = on2 ? pos[e2].z : R(0);
#pragma unroll 8
      for (int t = 0; t < 32; ++t) {
        const R zt = __shfl_sync(0xffffffffu, z2, t);
        const uint32_t et = __shfl_sync(0xffffffffu, e2, t);
        rank += (et != 0xffffffffu && (zt < ze || (zt == ze && et < e))) ? 1u : 0u;
      }
    }
    if (on) zord[s + rank] = e;
  }
}

// AssignRCut::assign index (ENG/src/AssignRCut.cu:93-112) in binary32
__device__ __forceinline__ float lattice_rcut(float x, float y, float z, const DevState* st,
                                              const float* lat, int nx, int ny, int nz) {
  const float Lx = st->Lf[0], Ly = st->Lf[1], Lz = st->Lf[2];
  if (x < 0) x = __fadd_rn(x, Lx); else if (x >= Lx) x = __fsub_rn(x, Lx);
  if (y < 0) y = __fadd_rn(y, Ly); else if (y >= Ly) y = __fsub_rn(y, Ly);
  if (z < 0) z = __fadd_rn(z, Lz); else if (z >= Lz) z = __fsub_rn(z, Lz);
  int ix = __float2int_rz(__fdiv_rn(__fmul_rn(x, (float)nx), Lx));
  int iy = __float2int_rz(__fdiv_rn(__fmul_rn(y, (float)ny), Ly));
  int iz = __float2int_rz(__fdiv_rn(__fmul_rn(z, (float)nz), Lz));
  ix = min(max(ix, 0), nx - 1); iy = min(max(iy, 0), ny - 1); iz = min(max(iz, 0), nz - 1);
  return lat[iz + nz * (iy + ny * ix)];
}

template <class R>
__global__ void k_gather(int N, const uint32_t* perm, const uint32_t* t_cell, uint32_t* cell_of,
                         const typename V4<R>::T* pos, const typename V4<R>::T* vel,
                         const double4a* force, const int4* image, const int* id, const float* rcut,
                         typename V4<R>::T* o_pos, typename V4<R>::T* o_vel, double4a* o_force,
                         int4* o_image, int* o_id, float* o_rcut, const float* lat, int nx, int ny,
                         int nz, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const uint32_t o = perm[k];
  typename V4<R>::T p = pos[o];
  o_pos[k] = p;
  o_vel[k] = vel[o];
  o_force[k] = force[o];
  o_image[k] = image[o];
  o_id[k] = id[o];
  o_rcut[k] = lat ? lattice_rcut((float)p.x, (float)p.y, (float)p.z, st, lat, nx, ny, nz) : rcut[o];
  cell_of[k] = t_cell[o];
}

template <class R>
__global__ void k_copyback(int N, const typename V4<R>::T* pos, const typename V4<R>::T* vel,
                           const double4a* force, const int4* image, const int* id, const float* rcut,
                           typename V4<R>::T* o_pos, typename V4<R>::T* o_vel, double4a* o_force,
                           int4* o_image, int* o_id, float* o_rcut, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  o_pos[k] = pos[k];
  o_vel[k] = vel[k];
  o_force[k] = force[k];
  o_image[k] = image[k];
  o_id[k] = id[k];
  o_rcut[k] = rcut[k];
}

template <class R>
static int rebuild_t(md_cell_list* cl, md_system* sys, Recorder* rec, bool gated) {
  typedef typename V4<R>::T T4;
  int N = sys->N;
  int gate = gated ? 1 : 0;
  CellGeom g;
  for (int d = 0; d < 3; ++d) g.nc[d] = cl->ncell[d];
  g.ntot = cl->ntot;
  T4* pos = (T4*)sys->pos;
  T4* vel = (T4*)sys->vel;
  T4* tp = (T4*)sys->t_pos;
  T4* tv = (T4*)sys->t_vel;
  DevState* st = sys->st;
  int nb = ceil_div(N, 256);
  {
    void* a[] = {&N, &pos, &sys->image, &st, &g, &cl->t_cell, &cl->slot, &cl->count, &gate};
    if (int r = rec_launch(rec, (const void*)k_bin<R>, dim3(nb), dim3(256), 0, a)) return r;
  }
  {
    int n = cl->ntot;
    void* a[] = {&n, &cl->count, &cl->start, &st, &gate};
    if (int r = rec_launch(rec, (const void*)k_scan, dim3(1), dim3(1024), 0, a)) return r;
  }
  {
    void* a[] = {&N, &cl->t_cell, &cl->slot, &cl->start, &cl->members, &st, &gate};
    if (int r = rec_launch(rec, (const void*)k_scatter, dim3(nb), dim3(256), 0, a)) return r;
  }
  {
    int n = cl->ntot;
    void* a[] = {&n, &cl->start, &cl->members, &sys->rcut, &cl->perm, &st, &gate};
    if (int r = rec_launch(rec, (const void*)k_order, dim3(ceil_div((long long)n * 32, 256)), dim3(256), 0, a)) return r;
  }
  {
    float* lat = sys->d_lattice;
    int nx = sys->lat_n[0], ny = sys->lat_n[1], nz = sys->lat_n[2];
    void* a[] = {&N, &cl->perm, &cl->t_cell, &cl->cell_of, &pos, &vel, &sys->force, &sys->image,
                 &sys->id, &sys->rcut, &tp, &tv, &sys->t_force, &sys->t_image, &sys->t_id,
                 &sys->t_rcut, &lat, &nx, &ny, &nz, &st, &gate};
    if (int r = rec_launch(rec, (const void*)k_gather<R>, dim3(nb), dim3(256), 0, a)) return r;
  }
  {
    void* a[] = {&N, &tp, &tv, &sys->t_force, &sys->t_image, &sys->t_id, &sys->t_rcut,
                 &pos, &vel, &sys->force, &sys->image, &sys->id, &sys->rcut, &st, &gate};
    if (int r = rec_launch(rec, (const void*)k_copyback<R>, dim3(nb), dim3(256), 0, a)) return r;
  }
  {
    int n = cl->ntot;
    void* a[] = {&n, &cl->start, &pos, &cl->zord, &st, &gate};
    if (int r = rec_launch(rec, (const void*)k_zorder<R>, dim3(ceil_div((long long)n * 32, 256)), dim3(256), 0, a))
      return r;
  }
  return MD_OK;
}

int cells_rebuild_impl(md_cell_list* cl, md_system* sys, Recorder* rec, bool gated) {
  int r = (sys->prec == MD_PREC_FP64) ? rebuild_t<double>(cl, sys, rec, gated)
                                      : rebuild_t<float>(cl, sys, rec, gated);
  if (r == MD_OK) r = topo_slot_launch(sys, rec, gated);  // ids moved: refresh the slot map
  if (r == MD_OK) r = types_slot_launch(sys, rec, gated);  // and the per-slot types
  if (r == MD_OK) cl->built = true;
  return r;
}

// ------------------------------------------------------------------ C ABI
extern "C" int md_cell_list_create(md_cell_list** out, md_system* sys, double cell_size, int bdir,
                                   int divide) {
  if (!out || !sys || !(cell_size > 0) || divide < 1) { md_set_error("md_cell_list_create: bad arguments"); return MD_ERR_BADARG; }
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  md_cell_list* cl = new md_cell_list();
  cl->cell_size = cell_size;
  cl->bdir = bdir;
  cl->divide = divide;
  // DecideNumCell: NCell = floor(L * (1/cellSize)) on the chosen directions, times divide
  double csi = 1.0 / cell_size;
  for (int d = 0; d < 3; ++d) {
    int on = bdir & (1 << d);
    int nc = on ? (int)std::floor(hs.L[d] * csi) : 1;
    if (nc < 1) nc = 1;
    if (on) nc *= divide;
    cl->ncell[d] = nc;
  }
  cl->ntot = cl->ncell[0] * cl->ncell[1] * cl->ncell[2];
  int N = sys->N;
  bool ok = cudaMalloc(&cl->cell_of, sizeof(uint32_t) * N) == cudaSuccess &&
            cudaMalloc(&cl->t_cell, sizeof(uint32_t) * N) == cudaSuccess &&
            cudaMalloc(&cl->slot, sizeof(uint32_t) * N) == cudaSuccess &&
            cudaMalloc(&cl->count, sizeof(uint32_t) * cl->ntot) == cudaSuccess &&
            cudaMalloc(&cl->start, sizeof(uint32_t) * (cl->ntot + 1)) == cudaSuccess &&
            cudaMalloc(&cl->members, sizeof(uint32_t) * N) == cudaSuccess &&
            cudaMalloc(&cl->perm, sizeof(uint32_t) * N) == cudaSuccess &&
            cudaMalloc(&cl->zord, sizeof(uint32_t) * N) == cudaSuccess &&
            cudaMemset(cl->count, 0, sizeof(uint32_t) * cl->ntot) == cudaSuccess;
  if (!ok) {
    md_cuda_fail(cudaGetLastError(), "md_cell_list_create");
    md_cell_list_destroy(cl);
    return MD_ERR_CUDA;
  }
  *out = cl;
  return MD_OK;
}

extern "C" int md_cell_list_destroy(md_cell_list* cl) {
  if (!cl) return MD_OK;
  void* p[] = {cl->cell_of, cl->t_cell, cl->slot, cl->count, cl->start, cl->members, cl->perm, cl->zord};
  for (void* q : p) if (q) cudaFree(q);
  delete cl;
  return MD_OK;
}

extern "C" int md_cell_list_rebuild(md_cell_list* cl, md_system* sys) {
  if (!cl || !sys) return MD_ERR_BADARG;
  Recorder rec;
  rec.stream = sys->stream;
  if (int r = cells_rebuild_impl(cl, sys, &rec, false)) return r;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  if (hs.flags & FLAG_NAN) { md_set_error("non-finite coordinate in cell binning"); return MD_ERR_BADARG; }
  if (hs.flags & FLAG_CELL_INDEX) { md_set_error("cell index overflow"); return MD_ERR_CELL_INDEX; }
  return MD_OK;
}

extern "C" int md_cell_list_get_ncell(md_cell_list* cl, int ncell[3]) {
  if (!cl || !ncell) return MD_ERR_BADARG;
  for (int d = 0; d < 3; ++d) ncell[d] = cl->ncell[d];
  return MD_OK;
}

__global__ void k_cell_out(int N, const uint32_t* cell_of, const int* id, uint32_t* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) out[id[k]] = cell_of[k];
}

extern "C" int md_cell_list_get_cell_index(md_cell_list* cl, md_system* sys, uint32_t* cell) {
  if (!cl || !sys || !cell) return MD_ERR_BADARG;
  if (!cl->built) { md_set_error("cell list not built"); return MD_ERR_BADARG; }
  uint32_t* d = nullptr;
  size_t bytes = sizeof(uint32_t) * sys->N;
  MD_CUDA(cudaMallocAsync((void**)&d, bytes, sys->stream));
  k_cell_out<<<ceil_div(sys->N, 256), 256, 0, sys->stream>>>(sys->N, cl->cell_of, sys->id, d);
  MD_CHECK_LAUNCH("cell out");
  MD_CUDA(cudaMemcpyAsync(cell, d, bytes, cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaFreeAsync(d, sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}

// ------------------------------------------------------------------ AssignRCut
__global__ void k_assign_rcut(int N, const float4* pos4, const double4a* pos8, int prec, float* rc,
                              const float* lat, int nx, int ny, int nz, const DevState* st) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  float x, y, z;
  if (prec == MD_PREC_FP64) { double4a p = pos8[k]; x = (float)p.x; y = (float)p.y; z = (float)p.z; }
  else { float4 p = pos4[k]; x = p.x; y = p.y; z = p.z; }
  rc[k] = lattice_rcut(x, y, z, st, lat, nx, ny, nz);
}

__global__ void k_fill(int N, float* a, float v) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) a[k] = v;
}

extern "C" int md_assign_rcut(md_system* sys, const float* lattice, int nx, int ny, int nz) {
  if (!sys || !lattice || nx < 1 || ny < 1 || nz < 1) { md_set_error("md_assign_rcut: bad arguments"); return MD_ERR_BADARG; }
  for (long long i = 0; i < (long long)nx * ny * nz; ++i)
    if (!(lattice[i] > 0) || !std::isfinite(lattice[i])) { md_set_error("md_assign_rcut: bad lattice value at %lld", i); return MD_ERR_BADARG; }
  size_t n = (size_t)nx * ny * nz;
  if (sys->d_lattice && (size_t)sys->lat_n[0] * sys->lat_n[1] * sys->lat_n[2] != n) {
    cudaFree(sys->d_lattice);
    sys->d_lattice = nullptr;
  }
  if (!sys->d_lattice) MD_CUDA(cudaMalloc(&sys->d_lattice, sizeof(float) * n));
  sys->lat_n[0] = nx; sys->lat_n[1] = ny; sys->lat_n[2] = nz;
  MD_CUDA(cudaMemcpyAsync(sys->d_lattice, lattice, sizeof(float) * n, cudaMemcpyHostToDevice, sys->stream));
  k_assign_rcut<<<ceil_div(sys->N, 256), 256, 0, sys->stream>>>(
      sys->N, (float4*)sys->pos, (double4a*)sys->pos, sys->prec, sys->rcut, sys->d_lattice, nx, ny, nz, sys->st);
  MD_CHECK_LAUNCH("assign rcut");
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}

extern "C" int md_set_rcut_uniform(md_system* sys, float rc) {
  if (!sys || !(rc > 0)) { md_set_error("md_set_rcut_uniform: bad arguments"); return MD_ERR_BADARG; }
  if (sys->d_lattice) { cudaFree(sys->d_lattice); sys->d_lattice = nullptr; }
  sys->lat_n[0] = sys->lat_n[1] = sys->lat_n[2] = 0;
  k_fill<<<ceil_div(sys->N, 256), 256, 0, sys->stream>>>(sys->N, sys->rcut, rc);
  MD_CHECK_LAUNCH("fill rcut");
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}
