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

// single-block exclusive scan of the cell counts (each thread owns PER
// consecutive cells of a tile of PER * blockDim cells, read and written as
// 16-byte vectors: count and start come from cudaMalloc and PER is a multiple
// of 4, so every vector is aligned); zeroes count for the next rebuild.  One
// block, any multiple of 32 threads; the running total carries from tile to
// tile and the next tile is loaded early.
template <int PER>
__device__ __forceinline__ void scan_block(int n, uint32_t* count, uint32_t* start) {
  static_assert(PER % 4 == 0, "whole 16-byte vectors per thread");
  __shared__ uint32_t wsum[32];
  const int T = blockDim.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = T >> 5;
  uint32_t carry = 0;
  auto loadv = [&](int i0, uint32_t (&v)[PER]) {
#pragma unroll
    for (int q = 0; q < PER / 4; ++q) {
      const int j = i0 + 4 * q;
      if (j + 3 < n) {
        const uint4 u = *reinterpret_cast<const uint4*>(count + j);
        v[4 * q] = u.x; v[4 * q + 1] = u.y; v[4 * q + 2] = u.z; v[4 * q + 3] = u.w;
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[4 * q + k] = (j + k < n) ? count[j + k] : 0u;
      }
    }
  };
  uint32_t nxt[PER];
  loadv(PER * threadIdx.x, nxt);
  for (int base = 0; base < n; base += PER * T) {
    const int i0 = base + PER * threadIdx.x;
    uint32_t v[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) v[k] = nxt[k];
    if (base + PER * T < n) loadv(i0 + PER * T, nxt);
    uint32_t tot = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) tot += v[k];
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
#pragma unroll
    for (int q = 0; q < PER / 4; ++q) {
      const int j = i0 + 4 * q;
      if (j + 3 < n) {
        const uint32_t s0 = run, s1 = s0 + v[4 * q], s2 = s1 + v[4 * q + 1], s3 = s2 + v[4 * q + 2];
        *reinterpret_cast<uint4*>(start + j) = make_uint4(s0, s1, s2, s3);
        *reinterpret_cast<uint4*>(count + j) = make_uint4(0u, 0u, 0u, 0u);
        run = s3 + v[4 * q + 3];
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (j + k < n) {
            start[j + k] = run;
            count[j + k] = 0u;
          }
          run += v[4 * q + k];
        }
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

// order_cell and, from the same members, the z order zorder_cell gives after
// the gather: member e goes to slot s + rank(e) (perm), and its z there is
// the binned pos[e].z, so ranking (z, new slot) here gives zord without a
// pass over the gathered arrays.  Up to 32 members stay in registers; a
// fuller cell reads its new order back from perm.
template <class R>
__device__ __forceinline__ void order_zorder_cell(int cell, int lane, const uint32_t* start, const uint32_t* members,
                                                  const float* rcut, const typename V4<R>::T* pos, uint32_t* perm,
                                                  uint32_t* zord) {
  const uint32_t s = start[cell], n = start[cell + 1] - s;
  if (n == 0) return;
  if (n > 32) {
    order_cell(cell, lane, start, members, rcut, perm);
    __syncwarp();  // the warp's perm stores are visible to the warp
    for (uint32_t b = 0; b < n; b += 32) {
      const bool on = b + lane < n;
      const uint32_t e = on ? s + b + lane : 0u;
      const R ze = on ? pos[perm[e]].z : R(0);
      uint32_t rank = 0;
      for (uint32_t b2 = 0; b2 < n; b2 += 32) {
        const bool on2 = b2 + lane < n;
        const uint32_t e2 = on2 ? s + b2 + lane : 0xffffffffu;
        const R z2 = on2 ? pos[perm[e2]].z : R(0);
#pragma unroll 8
        for (int t = 0; t < 32; ++t) {
          const R zt = __shfl_sync(0xffffffffu, z2, t);
          const uint32_t et = __shfl_sync(0xffffffffu, e2, t);
          rank += (et != 0xffffffffu && (zt < ze || (zt == ze && et < e))) ? 1u : 0u;
        }
      }
      if (on) zord[s + rank] = e;
    }
    return;
  }
  const bool on = (uint32_t)lane < n;
  const uint32_t m = on ? members[s + lane] : 0u;
  const unsigned long long km = on ? (((unsigned long long)__float_as_uint(rcut[m]) << 32) | m) : ~0ull;
  const R zm = on ? pos[m].z : R(0);
  uint32_t rank = 0;
#pragma unroll 8
  for (int t = 0; t < 32; ++t) {
    const unsigned long long kt = __shfl_sync(0xffffffffu, km, t);
    rank += (kt < km) ? 1u : 0u;
  }
  const uint32_t e = on ? s + rank : 0xffffffffu;  // the member's slot after the gather
  if (on) perm[e] = m;
  uint32_t rz = 0;
#pragma unroll 8
  for (int t = 0; t < 32; ++t) {
    const R zt = __shfl_sync(0xffffffffu, zm, t);
    const uint32_t et = __shfl_sync(0xffffffffu, e, t);
    rz += (et != 0xffffffffu && (zt < zm || (zt == zm && et < e))) ? 1u : 0u;
  }
  if (on) zord[s + rz] = e;
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
