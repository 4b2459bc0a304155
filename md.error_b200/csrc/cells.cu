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
#include "cells_dev.cuh"

// ------------------------------------------------------------ kernels
template <class R>
__global__ void k_bin(int N, typename V4<R>::T* pos, int4* image, DevState* st, CellGeom g,
                      uint32_t* t_cell, uint32_t* slot, uint32_t* count, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bin_atom<R>(i, i < N, pos, image, st, g, t_cell, slot, count);
}

__global__ void __launch_bounds__(1024) k_scan(int n, uint32_t* count, uint32_t* start, DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  scan_block<4>(n, count, start);
}

__global__ void k_scatter(int N, const uint32_t* t_cell, const uint32_t* slot, const uint32_t* start,
                          uint32_t* members, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) scatter_atom(i, t_cell, slot, start, members);
}

__global__ void k_order(int ntot, const uint32_t* start, const uint32_t* members, const float* rcut,
                        uint32_t* perm, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp < ntot) order_cell(warp, threadIdx.x & 31, start, members, rcut, perm);
}

template <class R>
__global__ void k_zorder(int ntot, const uint32_t* start, const typename V4<R>::T* pos, uint32_t* zord,
                         const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp < ntot) zorder_cell<R>(warp, threadIdx.x & 31, start, pos, zord);
}

template <class R>
__global__ void k_gather(int N, const uint32_t* perm, const uint32_t* t_cell, uint32_t* cell_of,
                         const typename V4<R>::T* pos, const typename V4<R>::T* vel,
                         const double4a* force, const int4* image, const int* id, const float* rcut,
                         typename V4<R>::T* o_pos, typename V4<R>::T* o_vel, double4a* o_force,
                         int4* o_image, int* o_id, float* o_rcut, const float* lat, int nx, int ny,
                         int nz, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N)
    gather_atom<R>(k, perm, t_cell, cell_of, pos, vel, force, image, id, rcut, o_pos, o_vel, o_force, o_image, o_id,
                   o_rcut, lat, nx, ny, nz, st);
}

template <class R>
__global__ void k_copyback(int N, const typename V4<R>::T* pos, const typename V4<R>::T* vel,
                           const double4a* force, const int4* image, const int* id, const float* rcut,
                           typename V4<R>::T* o_pos, typename V4<R>::T* o_vel, double4a* o_force,
                           int4* o_image, int* o_id, float* o_rcut, const DevState* st, int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) copyback_atom<R>(k, pos, vel, force, image, id, rcut, o_pos, o_vel, o_force, o_image, o_id, o_rcut);
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
            cudaMalloc(&cl->busy, sizeof(uint32_t) * cl->ntot) == cudaSuccess &&
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
  void* p[] = {cl->cell_of, cl->t_cell, cl->slot, cl->count, cl->start, cl->members, cl->perm, cl->zord, cl->busy};
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
