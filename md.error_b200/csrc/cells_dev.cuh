// Cell binning and cell-order sort, per atom / per cell / per block: the
// bodies shared by the one-kernel-per-phase chain (cells.cu) and the fused,
// flag-gated rebuild kernel (nlist.cu).  References as in cells.cu.
#pragma once
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

// atom i of a warp-uniform pass (valid = i < N; every lane of the warp calls)
template <class R>
__device__ __forceinline__ void bin_atom(int i, bool valid, typename V4<R>::T* pos, int4* image, DevState* st,
                                         const CellGeom& g, uint32_t* t_cell, uint32_t* slot, uint32_t* count) {
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

// single-block exclusive scan (each thread owns 4 cells of a tile); zeroes
// count for the next rebuild
// one block, any multiple of 32 threads
__device__ __forceinline__ void scan_block(int n, uint32_t* count, uint32_t* start) {
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

__device__ __forceinline__ void scatter_atom(int i, const uint32_t* t_cell, const uint32_t* slot,
                                             const uint32_t* start, uint32_t* members) {
  members[start[t_cell[i]] + slot[i]] = (uint32_t)i;
}

// warp per cell: rank each member by its previous slot (ascending)
// Members of a cell are ranked by (cutoff, previous slot): atoms of equal
// cutoff (hence similar list length) become neighbours in memory, so the
// force kernel's warps, which take consecutive atoms, see rows of similar
// length; the previous slot breaks ties, so the order is deterministic.
__device__ __forceinline__ void order_cell(int cell, int lane, const uint32_t* start, const uint32_t* members,
                                           const float* rcut, uint32_t* perm) {
  const uint32_t s = start[cell], n = start[cell + 1] - s;
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
__device__ __forceinline__ void zorder_cell(int cell, int lane, const uint32_t* start,
                                            const typename V4<R>::T* pos, uint32_t* zord) {
  const uint32_t s = start[cell], n = start[cell + 1] - s;
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
__device__ __forceinline__ void gather_atom(int k, const uint32_t* perm, const uint32_t* t_cell, uint32_t* cell_of,
                                            const typename V4<R>::T* pos, const typename V4<R>::T* vel,
                                            const double4a* force, const int4* image, const int* id,
                                            const float* rcut, typename V4<R>::T* o_pos,
                                            typename V4<R>::T* o_vel, double4a* o_force, int4* o_image,
                                            int* o_id, float* o_rcut, const float* lat, int nx, int ny, int nz,
                                            const DevState* st) {
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
__device__ __forceinline__ void copyback_atom(int k, const typename V4<R>::T* pos, const typename V4<R>::T* vel,
                                              const double4a* force, const int4* image, const int* id,
                                              const float* rcut, typename V4<R>::T* o_pos,
                                              typename V4<R>::T* o_vel, double4a* o_force, int4* o_image,
                                              int* o_id, float* o_rcut) {
  o_pos[k] = pos[k];
  o_vel[k] = vel[k];
  o_force[k] = force[k];
  o_image[k] = image[k];
  o_id[k] = id[k];
  o_rcut[k] = rcut[k];
}
