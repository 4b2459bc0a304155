// Verlet neighbour-list build with skin, displacement check and export.
// Reference: buildDeviceNeighborList_AllPair (ENG/src/NeighborList.cu:327-420),
// buildDeviceNeighborList_DeviceCellList (UNI/src/NeighborList_interface.cu:361-491),
// NeighborList::mallocDeviceNeighborList (UNI/src/NeighborList_interface.cu:187-208),
// Displacement_max (ENG/src/Displacement_interface.cu:80-126).
//
// One block per home cell.  The candidate cells of the home cell (every cell
// whose box comes within the largest list radius of the home-cell box, or the
// reference's c +- 1 stencil in cell-shift mode) are enumerated as (x, y)
// columns of contiguous z runs -- each run one contiguous slice of the
// cell-sorted arrays -- and staged into a shared-memory tile.  Each warp then
// takes one home atom i at a time; its 32 lanes test 32 tile entries at once,
// skipping runs whose box lies beyond rlist_i, and a ballot compacts the
// accepted ones into row i of the list.  When the tile would not fit, the same
// loop reads the runs from global memory.
// The acceptance test repeats the reference's binary32 operations exactly
// (no FMA contraction), so the neighbour SETS are bit-identical to the
// reference criterion; only the enumeration (and list order) is ours.
// List layout: list[i*cap + k], k < nnb[i]; each entry packs the slot index j
// (bits 0-25) and the periodic image k_d = floorf(d_d/L_d + 0.5) in {-1,0,1}
// of the minimum-image vector, 2 bits per axis (bits 26-31, stored k+1), so
// the force loop forms d - k L with the reference's exact operations.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include "cells_dev.cuh"
#include "langevin.cuh"

struct NlGeom {
  int nc[3];
};

#define NL_TILE_CAP 2304
#define NL_MAX_RUNS 160
#define NL_RUN_MAXZ 7   // z cells of a run with per-atom z windows (longer runs are scanned whole)

// Runs of a home cell, one array per field (the 32 lanes of a warp read the
// fields of 32 different runs at once, which a struct per run would turn
// into 16-way shared-memory bank conflicts)
struct RunTable {
  int jb[NL_MAX_RUNS], cnt[NL_MAX_RUNS], off[NL_MAX_RUNS];  // global start, length, tile offset
  int sx[NL_MAX_RUNS], sy[NL_MAX_RUNS], sz[NL_MAX_RUNS];    // periodic images of the run
  float b0[3][NL_MAX_RUNS], b1[3][NL_MAX_RUNS];             // run box (unwrapped frame of the home cell)
  int zc0[NL_MAX_RUNS], nz[NL_MAX_RUNS];  // first z cell (unwrapped); z cells with offsets in zoff (0 = none)
  // zoff[k][r]: offset in run r of the first atom of its k-th z cell (k = nz: cnt)
  unsigned short zoff[NL_RUN_MAXZ + 1][NL_MAX_RUNS];
};

__device__ __forceinline__ int img_code(int kx, int ky, int kz) {
  return ((kx + 1) << 26) | ((ky + 1) << 28) | ((kz + 1) << 30);
}

// the slot index carried in the w component of a staged position (bit copy)
template <class R> __device__ __forceinline__ R slot_as_w(int j);
template <> __device__ __forceinline__ float slot_as_w<float>(int j) { return __int_as_float(j); }
template <> __device__ __forceinline__ double slot_as_w<double>(int j) { return __longlong_as_double((long long)j); }
template <class R> __device__ __forceinline__ int slot_of_w(R w);
template <> __device__ __forceinline__ int slot_of_w<float>(float w) { return __float_as_int(w); }
template <> __device__ __forceinline__ int slot_of_w<double>(double w) { return (int)__double_as_longlong(w); }

// The lists of the atoms of home cell c, by one block of 8 warps.  Every
// exit is uniform over the block; the shared state is first written after a
// block barrier, so a block may run this for one cell after another.
template <class R, int MODE>
__device__ __forceinline__ void nl_build_cell(int c, const typename V4<R>::T* __restrict__ pos,
                                              const float* __restrict__ rcut, const uint32_t* __restrict__ start,
                                              const uint32_t* __restrict__ zord, NlGeom g,
                                              const DevState* __restrict__ st, double rlist_uniform, double skin,
                                              int cap, int* __restrict__ list, int* __restrict__ nnb,
                                              typename V4<R>::T* __restrict__ backup, int force_minimage,
                                              DevState* stw) {
  typedef typename V4<R>::T T4;
  extern __shared__ __align__(16) unsigned char nl_smem[];
  T4* tile = reinterpret_cast<T4*>(nl_smem);  // w carries the atom's slot (charges are not needed here)
  __shared__ RunTable rt;
  __shared__ int nruns, tile_n, use_global;
  __shared__ float rl_max_sh;
  const int i0 = (int)start[c], i1 = (int)start[c + 1];
  if (i0 == i1) return;  // empty home cell (uniform exit for the whole block)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const R L[3] = {boxL<R>(st, 0), boxL<R>(st, 1), boxL<R>(st, 2)};
  const R Li[3] = {boxLi<R>(st, 0), boxLi<R>(st, 1), boxLi<R>(st, 2)};
  const bool minimg = (MODE == MD_NL_MINIMAGE) || force_minimage;
  const int hc[3] = {c / (g.nc[2] * g.nc[1]), (c / g.nc[2]) % g.nc[1], c % g.nc[2]};

  // largest list radius among the home atoms
  if (threadIdx.x == 0) rl_max_sh = 0.f;
  __syncthreads();
  if (MODE == MD_NL_MINIMAGE) {
    float m = 0.f;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) m = fmaxf(m, __fadd_rn(rcut[i], (float)skin));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) atomicMax((int*)&rl_max_sh, __float_as_int(m));  // non-negative floats order as ints
  } else if (threadIdx.x == 0) {
    rl_max_sh = (float)rlist_uniform;
  }
  __syncthreads();

  // the stencil of the home cell (cells per axis whose box comes within the
  // largest radius), worked out once by thread 0
  __shared__ double s_h[3];
  __shared__ int s_lo[3], s_hi[3], s_full[3];
  if (threadIdx.x == 0) {
    const double rle = (double)rl_max_sh * (1.0 + 1e-6) + 2e-3;
    for (int d = 0; d < 3; ++d) {
      const double hd = st->L[d] / g.nc[d];
      s_h[d] = hd;
      if (!minimg) {
        const int reach = (hd >= rlist_uniform) ? 1 : (int)ceil(rlist_uniform / hd);
        s_lo[d] = hc[d] - reach; s_hi[d] = hc[d] + reach; s_full[d] = 0;
      } else {
        int a = (int)floor((hc[d] * hd - rle) / hd), b = (int)floor(((hc[d] + 1) * hd + rle) / hd);
        s_full[d] = (b - a + 1) >= g.nc[d];
        if (s_full[d]) { a = 0; b = g.nc[d] - 1; }
        s_lo[d] = a; s_hi[d] = b;
      }
    }
  }
  __syncthreads();
  // runs of candidate cells: one thread per (x, y) column of the stencil
  // computes its (at most 3) z segments; block-wide exclusive scans give
  // each run its slot and tile offset in column order
  const double h[3] = {s_h[0], s_h[1], s_h[2]};
  const int lo[3] = {s_lo[0], s_lo[1], s_lo[2]}, hi[3] = {s_hi[0], s_hi[1], s_hi[2]};
  const bool full[3] = {s_full[0] != 0, s_full[1] != 0, s_full[2] != 0};
  __shared__ int scan_r[32], scan_a[32];
  __shared__ int base_r, base_a, overflow_runs;
  if (threadIdx.x == 0) { base_r = 0; base_a = 0; overflow_runs = 0; }
  __syncthreads();
  const int ncy = hi[1] - lo[1] + 1;
  const int ncols = (hi[0] - lo[0] + 1) * ncy;
  for (int col0 = 0; col0 < ncols; col0 += blockDim.x) {
    const int col = col0 + threadIdx.x;
    int jb_s[3], cnt_s[3], rs[3], rz0[3], len_s[3], ra_s[3], nseg = 0;
    int ix = 0, iy = 0, sx = 0, sy = 0, colbase = 0;
    if (col < ncols) {
      ix = lo[0] + col / ncy;
      iy = lo[1] + col % ncy;
      int cx = ix, cy = iy;
      if (cx < 0) { cx += g.nc[0]; sx = 1; } else if (cx >= g.nc[0]) { cx -= g.nc[0]; sx = -1; }
      if (cy < 0) { cy += g.nc[1]; sy = 1; } else if (cy >= g.nc[1]) { cy -= g.nc[1]; sy = -1; }
      colbase = g.nc[2] * (cy + g.nc[1] * cx);
      int ra[3], rb[3], ns = 0;
      if (full[2]) { ra[0] = 0; rb[0] = g.nc[2] - 1; rs[0] = 0; rz0[0] = 0; ns = 1; }
      else {
        const int zlo = lo[2], zhi = hi[2];
        if (zlo < 0) { ra[ns] = zlo + g.nc[2]; rb[ns] = g.nc[2] - 1; rs[ns] = 1; rz0[ns] = zlo; ++ns; }
        const int a = max(zlo, 0), b = min(zhi, g.nc[2] - 1);
        if (a <= b) { ra[ns] = a; rb[ns] = b; rs[ns] = 0; rz0[ns] = a; ++ns; }
        if (zhi >= g.nc[2]) { ra[ns] = 0; rb[ns] = zhi - g.nc[2]; rs[ns] = -1; rz0[ns] = g.nc[2]; ++ns; }
      }
      for (int s = 0; s < ns; ++s) {
        const int jb = (int)start[colbase + ra[s]], je = (int)start[colbase + rb[s] + 1];
        if (je == jb) continue;
        jb_s[nseg] = jb; cnt_s[nseg] = je - jb; len_s[nseg] = rb[s] - ra[s];
        rs[nseg] = rs[s]; rz0[nseg] = rz0[s]; ra_s[nseg] = ra[s];
        ++nseg;
      }
    }
    int atoms = 0;
    for (int s = 0; s < nseg; ++s) atoms += cnt_s[s];
    // inclusive warp scans of (runs, atoms), then across warps
    int ir = nseg, ia = atoms;
    for (int o = 1; o < 32; o <<= 1) {
      const int vr = __shfl_up_sync(0xffffffffu, ir, o), va = __shfl_up_sync(0xffffffffu, ia, o);
      if (lane >= o) { ir += vr; ia += va; }
    }
    if (lane == 31) { scan_r[warp] = ir; scan_a[warp] = ia; }
    __syncthreads();
    int wr = base_r, wa = base_a;
    for (int w = 0; w < warp; ++w) { wr += scan_r[w]; wa += scan_a[w]; }
    int r_off = wr + ir - nseg, a_off = wa + ia - atoms;
    for (int s = 0; s < nseg; ++s) {
      if (r_off >= NL_MAX_RUNS) { overflow_runs = 1; break; }
      const int q = r_off;
      rt.jb[q] = jb_s[s]; rt.cnt[q] = cnt_s[s]; rt.off[q] = a_off;
      rt.sx[q] = sx; rt.sy[q] = sy; rt.sz[q] = rs[s];
      const int zc0 = rz0[s], zc1 = rz0[s] + len_s[s];
      rt.b0[0][q] = full[0] ? -1e30f : (float)(ix * h[0]); rt.b1[0][q] = full[0] ? 1e30f : (float)((ix + 1) * h[0]);
      rt.b0[1][q] = full[1] ? -1e30f : (float)(iy * h[1]); rt.b1[1][q] = full[1] ? 1e30f : (float)((iy + 1) * h[1]);
      rt.b0[2][q] = full[2] ? -1e30f : (float)(zc0 * h[2]); rt.b1[2][q] = full[2] ? 1e30f : (float)((zc1 + 1) * h[2]);
      // per-cell offsets for the per-atom z window (runs that do not wrap the
      // whole z axis and have at most NL_RUN_MAXZ cells)
      rt.zc0[q] = zc0;
      const int nzq = (!full[2] && len_s[s] + 1 <= NL_RUN_MAXZ && cnt_s[s] <= 65535) ? len_s[s] + 1 : 0;
      rt.nz[q] = nzq;
      for (int k = 0; k < nzq; ++k)
        rt.zoff[k][q] = (unsigned short)((int)start[colbase + ra_s[s] + k] - jb_s[s]);
      if (nzq) rt.zoff[nzq][q] = (unsigned short)cnt_s[s];
      ++r_off;
      a_off += cnt_s[s];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 0; w < nwarp; ++w) { base_r += scan_r[w]; base_a += scan_a[w]; }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    nruns = min(base_r, NL_MAX_RUNS);
    tile_n = base_a;
    use_global = (base_a > NL_TILE_CAP) ? 1 : 0;
    if (overflow_runs) atomicOr(&stw->flags, FLAG_NL_OVERFLOW);
  }
  __syncthreads();
  const int nr = nruns;
  // stage the runs into the tile, one warp per run; a home cell with fewer
  // than 4 atoms reads its candidates from L2 instead (staging would cost
  // more than the few reads it saves)
  const bool stage = !use_global && (i1 - i0) >= 4;
  // a run's cells are staged in their z order (zord), so each cell of the run
  // is a z-sorted slice of the tile
  if (stage) {
    for (int r = warp; r < nr; r += nwarp) {
      const int c = rt.cnt[r], o = rt.off[r], jb = rt.jb[r];
      for (int t = lane; t < c; t += 32) {
        const int j = (int)zord[jb + t];
        T4 v = pos[j];
        v.w = slot_as_w<R>(j);
        tile[o + t] = v;
      }
    }
  }
  __syncthreads();
  const bool glob = !stage;
  const unsigned ltmask = (1u << lane) - 1u;
  const unsigned lemask = (2u << lane) - 1u;  // lanes 0..lane (all 32 for lane 31)
  // per-warp table of the current run group's non-empty runs (rank order)
  __shared__ int wdelta[8][32];
  __shared__ T4 wshift[8][32];
  // When the stencil spans less than the box along every axis, each cell
  // appears in exactly one run, at that run's periodic image k_run, and
  // 2 rlist < L.  For any pair within rlist the reference's image
  // floor((r_j - r_i)/L + 1/2) is then k_run (it can differ only where
  // |d| is within rounding of L/2 > rlist, where both reject), so
  // d = (r_j - r_i) - k_run L repeats the reference's binary32 operations and
  // the image code is the run's.
  const bool runshift = minimg && !full[0] && !full[1] && !full[2];
  const float hz = (float)h[2], hzi = 1.0f / hz;
  const float Lzf = (float)st->L[2];
  // z of entry t of a run (z order) in the stored, wrapped frame
  auto zat = [&](int roff, int rjb, int t) -> float {
    return glob ? (float)pos[zord[rjb + t]].z : (float)tile[roff + t].z;
  };

  for (int i = i0 + warp; i < i1; i += nwarp) {
    const T4 pi = pos[i];
    R rl;
    if (MODE == MD_NL_MINIMAGE) rl = add_rn((R)rcut[i], (R)skin);
    else rl = (R)rlist_uniform;
    const R rl2 = mul_rn(rl, rl);
    // enumeration coordinates of i in the home cell's frame
    float xe[3];
    {
      const double xi[3] = {(double)pi.x, (double)pi.y, (double)pi.z};
      for (int d = 0; d < 3; ++d) {
        double w = xi[d] - floor(xi[d] * st->Li[d]) * st->L[d];
        if (!(w >= 0.0) || w >= st->L[d]) w = 0.0;
        xe[d] = (float)w;
      }
    }
    const float rle_i = (float)rl * (1.0f + 1e-5f) + 2e-3f;
    int n = 0;
    int* rowp = list + (size_t)i * cap;
    // the 32 lanes test 32 runs at a time against i's box distance and z
    // window, then the surviving runs are walked in order
    for (int rb = 0; rb < nr; rb += 32) {
      bool keep = false;
      int tbl = 0, tel = 0;
      if (rb + lane < nr) {
        const int r = rb + lane;
        keep = true;
        float wz = rle_i;  // z half-window of i in this run's (x, y) column
        if (minimg) {
          float dxy = 0.f;
          for (int d = 0; d < 2; ++d) {
            const float e = fmaxf(0.f, fmaxf(rt.b0[d][r] - xe[d], xe[d] - rt.b1[d][r]));
            dxy += e * e;
          }
          const float ez = fmaxf(0.f, fmaxf(rt.b0[2][r] - xe[2], xe[2] - rt.b1[2][r]));
          keep = dxy + ez * ez <= rle_i * rle_i;
          wz = sqrtf(fmaxf(rle_i * rle_i - dxy, 0.f));
        }
        // the cells of the run that meet i's z window [z - wz, z + wz]; the
        // first and last of them are cut to the window by binary search in
        // their z order (the middle ones lie inside it whole)
        tbl = 0;
        tel = rt.cnt[r];
        const int nzr = rt.nz[r];
        if (keep && minimg && nzr) {
          const int zc0 = rt.zc0[r];
          // (a product with 1/h_z: its rounding, ~1e-5 cell, stays inside the
          // window's 2e-3 margin)
          const int k0 = max((int)floorf((xe[2] - wz) * hzi) - zc0, 0);
          const int k1 = min((int)floorf((xe[2] + wz) * hzi) - zc0, nzr - 1);
          keep = k0 <= k1;
          if (keep) {
            const int roff = rt.off[r], rjb = rt.jb[r];
            // window in the stored frame: z_stored = z_run + sz L_z
            const float shift = (float)rt.sz[r] * Lzf;
            const float zlo = xe[2] - wz - 1e-3f + shift, zhi = xe[2] + wz + 1e-3f + shift;
            int lo = rt.zoff[k0][r], hi = rt.zoff[k0 + 1][r];  // first index with z >= zlo
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (zat(roff, rjb, mid) < zlo) lo = mid + 1; else hi = mid;
            }
            tbl = lo;
            lo = rt.zoff[k1][r];  // first index with z > zhi
            hi = rt.zoff[k1 + 1][r];
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (zat(roff, rjb, mid) <= zhi) lo = mid + 1; else hi = mid;
            }
            tel = lo;
            keep = tbl < tel;
          }
        }
      }
      // the candidate ranges of the surviving runs, packed end to end into
      // 32-lane chunks: lane l of a chunk takes candidate c = t0 + l, owned by
      // the last non-empty run whose range starts at or before c.  The
      // non-empty runs are compacted (in run order) into the warp's table:
      // the offset taking c to its tile (or zord) index, and the run's image
      // shift k L with its code.  Within a chunk the owner's rank is the number
      // of non-empty runs starting before the chunk plus those starting inside
      // it at or before c (a 32-bit start mask).
      const int len = keep ? tel - tbl : 0;
      int incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      const int excl = incl - len;
      const bool ne = len > 0;
      const unsigned nem = __ballot_sync(0xffffffffu, ne);
      __syncwarp();  // the previous group's table has been read
      if (ne) {
        const int r = rb + lane;
        const int k = __popc(nem & ltmask);
        wdelta[warp][k] = (glob ? rt.jb[r] : rt.off[r]) + tbl - excl;
        const int rsx = rt.sx[r], rsy = rt.sy[r], rsz = rt.sz[r];
        wshift[warp][k] = T4{mul_rn((R)rsx, L[0]), mul_rn((R)rsy, L[1]), mul_rn((R)rsz, L[2]),
                             slot_as_w<R>(img_code(rsx, rsy, rsz))};
      }
      __syncwarp();
      int before = 0;  // non-empty runs starting before the chunk
      for (int t0 = 0; t0 < total; t0 += 32) {
        const int cidx = t0 + lane;
        const unsigned smask =
            __reduce_or_sync(0xffffffffu, (ne && excl >= t0 && excl < t0 + 32) ? (1u << (excl - t0)) : 0u);
        const int k = before + __popc(smask & lemask) - 1;
        before += __popc(smask);
        bool ok = false;
        int j = 0, code = 0;
        if (cidx < total) {
          const int x = cidx + wdelta[warp][k];
          T4 pj;
          if (glob) {
            j = (int)zord[x];
            pj = pos[j];
          } else {
            pj = tile[x];
            j = slot_of_w<R>(pj.w);
          }
          const T4 sh = wshift[warp][k];
          R dx, dy, dz, d2;
          if (runshift) {
            dz = sub_rn(sub_rn(pj.z, pi.z), sh.z);
            if constexpr (std::is_same<R, float>::value) {
              // x and y as one packed binary32 pair: the same roundings
              const F2 dxy = f2_sub(f2_sub(f2(pj.x, pj.y), f2(pi.x, pi.y)), f2(sh.x, sh.y));
              float sx, sy;
              f2_split(f2_mul(dxy, dxy), sx, sy);
              d2 = __fadd_rn(__fadd_rn(sx, sy), __fmul_rn(dz, dz));
            } else {
              dx = sub_rn(sub_rn(pj.x, pi.x), sh.x);
              dy = sub_rn(sub_rn(pj.y, pi.y), sh.y);
              d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
            }
            code = slot_of_w<R>(sh.w);
          } else {
            const R rx = sub_rn(pj.x, pi.x), ry = sub_rn(pj.y, pi.y), rz = sub_rn(pj.z, pi.z);
            const R kx = floor_r(add_rn(mul_rn(rx, Li[0]), R(0.5)));
            const R ky = floor_r(add_rn(mul_rn(ry, Li[1]), R(0.5)));
            const R kz = floor_r(add_rn(mul_rn(rz, Li[2]), R(0.5)));
            if (minimg) {
              dx = sub_rn(rx, mul_rn(kx, L[0]));
              dy = sub_rn(ry, mul_rn(ky, L[1]));
              dz = sub_rn(rz, mul_rn(kz, L[2]));
            } else {
              dx = sub_rn(sub_rn(pj.x, sh.x), pi.x);
              dy = sub_rn(sub_rn(pj.y, sh.y), pi.y);
              dz = sub_rn(sub_rn(pj.z, sh.z), pi.z);
            }
            code = img_code((int)kx, (int)ky, (int)kz);
            d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
          }
          ok = (d2 < rl2) && (j != i);
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (ok) {
          const int p = n + __popc(m & ltmask);
          if (p < cap) rowp[nl_slot(p)] = j | code;
        }
        n += __popc(m);
      }
    }
    if (lane == 0) {
      nnb[i] = n;
      backup[i] = pi;
      if (n > cap) atomicOr(&stw->flags, FLAG_NL_OVERFLOW);
      atomicMax(&stw->max_nnb, n);
    }
  }
}

template <class R, int MODE>
__global__ void __launch_bounds__(256, 4)
k_nl_build(int N, const typename V4<R>::T* __restrict__ pos, const float* __restrict__ rcut,
           const uint32_t* __restrict__ start, const uint32_t* __restrict__ zord, NlGeom g,
           const DevState* __restrict__ st, double rlist_uniform, double skin, int cap, int* __restrict__ list,
           int* __restrict__ nnb, typename V4<R>::T* __restrict__ backup, int force_minimage, DevState* stw,
           int gate) {
  if (gate && !(st->flags & FLAG_REBUILD)) return;
  nl_build_cell<R, MODE>(blockIdx.x, pos, rcut, start, zord, g, st, rlist_uniform, skin, cap, list, nnb, backup,
                         force_minimage, stw);
}

template <class R, int MODE>
static const void* nl_kernel() {
  static bool attr = false;
  const void* f = (const void*)k_nl_build<R, MODE>;
  if (!attr) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(NL_TILE_CAP * sizeof(typename V4<R>::T)));
    attr = true;
  }
  return f;
}

// cell-list criterion needs >= 4 cells per direction (DecideNumCell), else the
// reference falls back to the all-pair (minimum image) kernel
static int nl_force_minimage(const md_nlist* nl, md_system* sys, const md_cell_list* cl, int* force_mi) {
  *force_mi = 0;
  if (nl->mode != MD_NL_CELLSHIFT) return MD_OK;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  for (int d = 0; d < 3; ++d) {
    if (cl->ncell[d] < 4) *force_mi = 1;
    double h = hs.L[d] / cl->ncell[d];
    int reach = (h >= nl->rlist) ? 1 : (int)std::ceil(nl->rlist / h);
    if (2 * reach + 1 > cl->ncell[d]) *force_mi = 1;
  }
  return MD_OK;
}

int nlist_build_impl(md_nlist* nl, md_system* sys, md_cell_list* cl, Recorder* rec, bool gated) {
  int N = sys->N;
  if (N >= (1 << 26)) { md_set_error("neighbour lists hold at most 2^26 atoms"); return MD_ERR_BADARG; }
  NlGeom g;
  for (int d = 0; d < 3; ++d) g.nc[d] = cl->ncell[d];
  int gate = gated ? 1 : 0;
  int force_mi = 0;
  if (int r = nl_force_minimage(nl, sys, cl, &force_mi)) return r;
  double rl = nl->rlist, skin = nl->skin;
  DevState* st = sys->st;
  int cap = nl->cap;
  dim3 grid(cl->ntot), block(256);
  void* a[] = {&N, &sys->pos, &sys->rcut, &cl->start, &cl->zord, &g, &st, &rl, &skin, &cap, &nl->list,
               &nl->nnb, &nl->backup, &force_mi, &st, &gate};
  const void* f;
  size_t smem;
  if (sys->prec == MD_PREC_FP64) {
    f = nl->mode == MD_NL_MINIMAGE ? nl_kernel<double, MD_NL_MINIMAGE>() : nl_kernel<double, MD_NL_CELLSHIFT>();
    smem = NL_TILE_CAP * sizeof(double4a);
  } else {
    f = nl->mode == MD_NL_MINIMAGE ? nl_kernel<float, MD_NL_MINIMAGE>() : nl_kernel<float, MD_NL_CELLSHIFT>();
    smem = NL_TILE_CAP * sizeof(float4);
  }
  if (int r = rec_launch(rec, f, grid, block, smem, a)) return r;
  if (int r = topo_exclude_launch(sys, nl, rec, gated)) return r;
  nl->built = true;
  return MD_OK;
}

// ------------------------------------------------------- fused rebuild
// The rebuild chain of cells.cu (bin, scan, scatter, order, gather, copy
// back, z order) and the list build as the phases of one cooperative kernel,
// separated by grid barriers, that returns at once unless the rebuild flag is
// set.  Inside a captured step it replaces the conditional node around the
// chain: a node that returns at once costs a few microseconds, the
// conditional node around eight kernels about ten.  Each phase does exactly
// the work of its kernel (the same device functions), so the sorted arrays
// and the lists are the same bit for bit.
template <class R>
struct RebuildArgs {
  typedef typename V4<R>::T T4;
  int N, ntot;
  CellGeom cg;
  NlGeom ng;
  T4 *pos, *vel, *t_pos, *t_vel;
  double4a *force, *t_force;
  int4 *image, *t_image;
  int *id, *t_id;
  float *rcut, *t_rcut;
  uint32_t *t_cell, *slot, *count, *start, *members, *perm, *cell_of, *zord, *busy;
  const float* lat;
  int lat_n[3];
  const uint8_t* type_by_id;  // null with one atom type
  uint8_t* type;
  DevState* st;
  double rlist, skin;
  int cap, force_mi;
  int *list, *nnb;
  T4* backup;
};

// resident blocks per SM the kernels are built for: the list tile of the
// FP64 path (72 KB) leaves room for two
template <class R> constexpr int rebuild_min_blocks() { return sizeof(R) == 4 ? 4 : 2; }

// the atoms of this block in the per-atom phases: a contiguous share of
// ceil(N / blocks), so that every block (and every SM) takes part
__device__ __forceinline__ void block_atoms(int N, int& k0, int& k1) {
  const int per = (N + (int)gridDim.x - 1) / (int)gridDim.x;
  k0 = min(N, (int)blockIdx.x * per);
  k1 = min(N, k0 + per);
}

// the phases, from the cell of every atom to the lists; every block calls
template <class R, int MODE>
__device__ __forceinline__ void rebuild_phases(const RebuildArgs<R>& a) {
  DevState* st = a.st;
  const int lane = threadIdx.x & 31;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const int gw = gt >> 5, nw = gs >> 5;
  int k0, k1;
  block_atoms(a.N, k0, k1);
  // 1. cell of every atom (warp-uniform passes for the warp-aggregated count)
  if (gt == 0) { st->red_counter[RED_NLWORK] = 0u; st->ncell_busy = 0u; st->ncell_light = 0u; }
  for (int b = k0 + (int)(threadIdx.x & ~31u); b < k1; b += blockDim.x)
    bin_atom<R>(b + lane, b + lane < k1, a.pos, a.image, st, a.cg, a.t_cell, a.slot, a.count);
  if (!grid_barrier(st)) return;
  // 2. cell starts
  if (blockIdx.x == 0) scan_block<16>(a.ntot, a.count, a.start);
  if (!grid_barrier(st)) return;
  // 3. member lists; the non-empty cells listed for the list build, cells of
  // 4 atoms or more from the front of the list and the others from its back,
  // so that the costly cells are handed out first and the cheap ones fill
  // the end (a slab has many empty or near-empty vapour cells)
  for (int i = k0 + threadIdx.x; i < k1; i += blockDim.x) scatter_atom(i, a.t_cell, a.slot, a.start, a.members);
  for (int cb = gw * 32; cb < a.ntot; cb += nw * 32) {
    const int c = cb + lane;
    const uint32_t n = c < a.ntot ? a.start[c + 1] - a.start[c] : 0u;
    const unsigned mh = __ballot_sync(0xffffffffu, n >= 4u), ml = __ballot_sync(0xffffffffu, n > 0u && n < 4u);
    unsigned bh = 0, bl = 0;
    if (lane == 0 && mh) bh = atomicAdd(&st->ncell_busy, (unsigned)__popc(mh));
    if (lane == 0 && ml) bl = atomicAdd(&st->ncell_light, (unsigned)__popc(ml));
    bh = __shfl_sync(0xffffffffu, bh, 0);
    bl = __shfl_sync(0xffffffffu, bl, 0);
    const unsigned below = (1u << lane) - 1u;
    if (n >= 4u) a.busy[bh + __popc(mh & below)] = (uint32_t)c;
    else if (n > 0u) a.busy[a.ntot - 1 - (int)(bl + __popc(ml & below))] = (uint32_t)c;
  }
  if (!grid_barrier(st)) return;
  // 4. deterministic order inside each cell and the cell's z order (warp
  // per cell)
  for (int c = gw; c < a.ntot; c += nw)
    order_zorder_cell<R>(c, lane, a.start, a.members, a.rcut, a.pos, a.perm, a.zord);
  if (!grid_barrier(st)) return;
  // 5. permute into cell order
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x)
    gather_atom<R>(k, a.perm, a.t_cell, a.cell_of, a.pos, a.vel, a.force, a.image, a.id, a.rcut, a.t_pos, a.t_vel,
                   a.t_force, a.t_image, a.t_id, a.t_rcut, a.lat, a.lat_n[0], a.lat_n[1], a.lat_n[2], st);
  if (!grid_barrier(st)) return;
  // 6. copy back with the per-slot types
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    copyback_atom<R>(k, a.t_pos, a.t_vel, a.t_force, a.t_image, a.t_id, a.t_rcut, a.pos, a.vel, a.force, a.image,
                     a.id, a.rcut);
    if (a.type) a.type[k] = a.type_by_id[a.t_id[k]];
  }
  if (!grid_barrier(st)) return;
  // 7. lists, the non-empty home cells handed out by a counter (cells differ
  // in work by tens of times across a slab; the order of the cells does not
  // change any list); the next cell is fetched while this one is built
  const int nfull = (int)__ldcg(&st->ncell_busy);
  const int nbusy = nfull + (int)__ldcg(&st->ncell_light);
  __shared__ int s_work;
  if (threadIdx.x == 0) s_work = (int)atomicAdd(&st->red_counter[RED_NLWORK], 1u);
  __syncthreads();
  int w = s_work;
  while (w < nbusy) {
    int nxt = 0;
    if (threadIdx.x == 0) nxt = (int)atomicAdd(&st->red_counter[RED_NLWORK], 1u);
    const int c = (int)__ldcg(&a.busy[w < nfull ? w : a.ntot - 1 - (w - nfull)]);
    nl_build_cell<R, MODE>(c, a.pos, a.rcut, a.start, a.zord, a.ng, st, a.rlist, a.skin, a.cap, a.list, a.nnb,
                           a.backup, a.force_mi, st);
    __syncthreads();
    if (threadIdx.x == 0) s_work = nxt;
    __syncthreads();
    w = s_work;
  }
}

template <class R, int MODE>
__global__ void __launch_bounds__(256, rebuild_min_blocks<R>()) k_rebuild(RebuildArgs<R> a) {
  // FLAG_REBUILD does not change while this kernel runs (it is set by the
  // step's first kernel and cleared by its last), so every block takes the
  // same branch
  if (!(a.st->flags & FLAG_REBUILD)) return;
  rebuild_phases<R, MODE>(a);
}

// The Langevin step's first half with the rebuild folded in: the particle
// B A O A and displacement test of k_lv_step1 (the same device function) for
// every atom, a grid barrier, the box of the step committed, and, when an
// atom has moved more than half the skin, the rebuild phases.  This saves the
// step a kernel node against k_lv_step1 followed by k_rebuild.
template <class R, int MODE>
__global__ void __launch_bounds__(256, rebuild_min_blocks<R>())
k_lv_step1_rebuild(typename V4<R>::T* __restrict__ vel, const double4a* __restrict__ force, LvDev p,
                   RebuildArgs<R> a) {
  DevState* st = a.st;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  int k0, k1;
  block_atoms(a.N, k0, k1);
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x)
    lv_particle_step1<R>(k, a.pos, vel, force, a.id, a.backup, st, p);
  // every block is done reading the box of the last step
  if (!grid_barrier(st)) return;
  if (gt == 0) box_commit(st);
  if (!(__ldcg(&st->flags) & FLAG_REBUILD)) return;
  if (!grid_barrier(st)) return;  // the committed box, for the binning
  rebuild_phases<R, MODE>(a);
}

// the kernel of a precision and list mode, its dynamic shared memory, the
// most blocks one cooperative launch can hold (0: not possible on this
// device) and the device's SM count
static const void* rebuild_kernel(int prec, int mode, size_t* smem, int* blocks, bool with_lv = false,
                                  int* sms = nullptr) {
  const void* f;
  if (prec == MD_PREC_FP64) {
    if (with_lv)
      f = mode == MD_NL_MINIMAGE ? (const void*)k_lv_step1_rebuild<double, MD_NL_MINIMAGE>
                                 : (const void*)k_lv_step1_rebuild<double, MD_NL_CELLSHIFT>;
    else
      f = mode == MD_NL_MINIMAGE ? (const void*)k_rebuild<double, MD_NL_MINIMAGE>
                                 : (const void*)k_rebuild<double, MD_NL_CELLSHIFT>;
    *smem = NL_TILE_CAP * sizeof(double4a);
  } else {
    if (with_lv)
      f = mode == MD_NL_MINIMAGE ? (const void*)k_lv_step1_rebuild<float, MD_NL_MINIMAGE>
                                 : (const void*)k_lv_step1_rebuild<float, MD_NL_CELLSHIFT>;
    else
      f = mode == MD_NL_MINIMAGE ? (const void*)k_rebuild<float, MD_NL_MINIMAGE>
                                 : (const void*)k_rebuild<float, MD_NL_CELLSHIFT>;
    *smem = NL_TILE_CAP * sizeof(float4);
  }
  *blocks = 0;
  int dev = 0, coop = 0, nsm = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, 256, *smem) != cudaSuccess) {
    cudaGetLastError();
    return f;
  }
  if (coop) *blocks = per_sm * nsm;
  if (sms) *sms = nsm;
  return f;
}

bool rebuild_fused_ok(const md_system* sys, const md_nlist* nl) {
  if (sys->topo) return false;  // the topology's slot map and exclusions are kernels of bonded.cu
  if (sys->N >= (1 << 26)) return false;
  size_t smem;
  int b1, b2;
  rebuild_kernel(sys->prec, nl->mode, &smem, &b1, false);
  rebuild_kernel(sys->prec, nl->mode, &smem, &b2, true);
  return b1 > 0 && b2 > 0;
}

template <class R>
static int rebuild_fused_t(md_cell_list* cl, md_nlist* nl, md_system* sys, Recorder* rec, bool with_lv) {
  typedef typename V4<R>::T T4;
  RebuildArgs<R> a;
  memset(&a, 0, sizeof(a));
  a.N = sys->N;
  a.ntot = cl->ntot;
  for (int d = 0; d < 3; ++d) { a.cg.nc[d] = cl->ncell[d]; a.ng.nc[d] = cl->ncell[d]; }
  a.cg.ntot = cl->ntot;
  a.pos = (T4*)sys->pos; a.vel = (T4*)sys->vel; a.t_pos = (T4*)sys->t_pos; a.t_vel = (T4*)sys->t_vel;
  a.force = sys->force; a.t_force = sys->t_force;
  a.image = sys->image; a.t_image = sys->t_image;
  a.id = sys->id; a.t_id = sys->t_id;
  a.rcut = sys->rcut; a.t_rcut = sys->t_rcut;
  a.t_cell = cl->t_cell; a.slot = cl->slot; a.count = cl->count; a.start = cl->start;
  a.members = cl->members; a.perm = cl->perm; a.cell_of = cl->cell_of; a.zord = cl->zord; a.busy = cl->busy;
  a.lat = sys->d_lattice;
  for (int d = 0; d < 3; ++d) a.lat_n[d] = sys->lat_n[d];
  if (sys->ntypes > 1) { a.type_by_id = sys->type_by_id; a.type = sys->type; }
  a.st = sys->st;
  a.rlist = nl->rlist; a.skin = nl->skin; a.cap = nl->cap;
  if (int r = nl_force_minimage(nl, sys, cl, &a.force_mi)) return r;
  a.list = nl->list; a.nnb = nl->nnb; a.backup = (T4*)nl->backup;
  size_t smem;
  int blocks, sms = 1;
  const void* f = rebuild_kernel(sys->prec, nl->mode, &smem, &blocks, with_lv, &sms);
  if (blocks <= 0) { md_set_error("fused rebuild: no cooperative launch on this device"); return MD_ERR_CUDA; }
  // a block per 8 cells, at least one per SM: every launch pays the grid
  // barrier and the block launches, and a small system has few cells to
  // share out (4,000-atom fluid, 216 cells: 30,500 steps/s at one block per
  // SM against 26,200 at four; the 65,536-atom slab keeps all four)
  blocks = std::min(blocks, std::max(sms, (cl->ntot + 7) / 8));
  if (!with_lv) {
    void* args[] = {&a};
    return rec_launch_coop(rec, f, dim3(blocks), dim3(256), smem, args);
  }
  LvDev p = make_lv(sys, nl);
  void* args[] = {&sys->vel, &sys->force, &p, &a};
  return rec_launch_coop(rec, f, dim3(blocks), dim3(256), smem, args);
}

int rebuild_fused_impl(md_cell_list* cl, md_nlist* nl, md_system* sys, Recorder* rec, bool with_lv) {
  if (sys->N >= (1 << 26)) { md_set_error("neighbour lists hold at most 2^26 atoms"); return MD_ERR_BADARG; }
  int r = (sys->prec == MD_PREC_FP64) ? rebuild_fused_t<double>(cl, nl, sys, rec, with_lv)
                                      : rebuild_fused_t<float>(cl, nl, sys, rec, with_lv);
  if (r == MD_OK) { cl->built = true; nl->built = true; }
  return r;
}

// ------------------------------------------------------ barrier check
// The fused rebuild's grid barrier on its own, for a test of its bounded
// wait: every block meets one barrier, except block `skip` (when >= 0),
// which returns at once, so the others wait out limit_ns, set FLAG_TIMEOUT
// and return.
__global__ void k_barrier_check(DevState* st, int skip, unsigned long long limit_ns) {
  if ((int)blockIdx.x == skip) return;
  grid_barrier(st, limit_ns);
}

// afterwards: the counter realigned and the timeout flag cleared
__global__ void k_barrier_check_reset(DevState* st) {
  st->gbar = 0ull;
  st->flags &= ~FLAG_TIMEOUT;
}

extern "C" int md_check_grid_barrier(md_system* sys, int skip_block, double limit_s, int* timed_out) {
  if (!sys || !timed_out || !(limit_s > 0.0) || limit_s > 10.0) {
    md_set_error("md_check_grid_barrier: bad arguments (0 < limit_s <= 10)");
    return MD_ERR_BADARG;
  }
  int dev = 0, coop = 0, nsm = 0;
  MD_CUDA(cudaGetDevice(&dev));
  MD_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  MD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (!coop) { md_set_error("md_check_grid_barrier: no cooperative launch on this device"); return MD_ERR_UNSUPPORTED; }
  if (skip_block >= nsm) { md_set_error("md_check_grid_barrier: skip_block beyond the grid (%d blocks)", nsm); return MD_ERR_BADARG; }
  DevState* st = sys->st;
  unsigned long long limit_ns = (unsigned long long)(limit_s * 1e9);
  // one block per SM, from a clean counter
  MD_CUDA(cudaMemsetAsync(&st->gbar, 0, sizeof(unsigned long long), sys->stream));
  void* a[] = {&st, &skip_block, &limit_ns};
  MD_CUDA(cudaLaunchCooperativeKernel((const void*)k_barrier_check, dim3(nsm), dim3(256), a, 0, sys->stream));
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  *timed_out = (hs.flags & FLAG_TIMEOUT) ? 1 : 0;
  k_barrier_check_reset<<<1, 1, 0, sys->stream>>>(st);
  MD_CHECK_LAUNCH("k_barrier_check_reset");
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  return MD_OK;
}

// ------------------------------------------------------------------ C ABI
static int alloc_lists(md_nlist* nl, md_system* sys) {
  if (nl->list) cudaFree(nl->list);
  nl->list = nullptr;
  MD_CUDA(cudaMalloc(&nl->list, sizeof(int) * (size_t)nl->cap * sys->N));
  return MD_OK;
}

extern "C" int md_nlist_create(md_nlist** out, md_system* sys, double rlist, double skin,
                               double expansion, int mode) {
  if (!out || !sys || !(rlist > 0) || skin < 0 || !(expansion > 0) ||
      (mode != MD_NL_MINIMAGE && mode != MD_NL_CELLSHIFT)) {
    md_set_error("md_nlist_create: bad arguments");
    return MD_ERR_BADARG;
  }
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  md_nlist* nl = new md_nlist();
  nl->rlist = rlist;
  nl->skin = skin;
  nl->expansion = expansion;
  nl->mode = mode;
  nl->N = sys->N;
  // mallocDeviceNeighborList: 4/3 pi rlist^3 rho * expansion, at least 30
  double rho = sys->N / (hs.L[0] * hs.L[1] * hs.L[2]);
  double expect = 4.0 / 3.0 * M_PI * rlist * rlist * rlist * rho;
  int cap = (int)(expect * expansion);
  if (cap < 30) cap = 30;
  // rows are a whole number of 32-entry (128-byte) lines: the force kernels
  // read a row in 16-byte vectors, 32 entries per pass, up to the line end
  cap = (cap + 31) & ~31;
  nl->cap = cap;
  size_t r4 = sys->r4_size();
  if (alloc_lists(nl, sys) != MD_OK || cudaMalloc(&nl->nnb, sizeof(int) * sys->N) != cudaSuccess ||
      cudaMalloc(&nl->backup, r4 * sys->N) != cudaSuccess) {
    md_cuda_fail(cudaGetLastError(), "md_nlist_create");
    md_nlist_destroy(nl);
    return MD_ERR_CUDA;
  }
  *out = nl;
  return MD_OK;
}

extern "C" int md_nlist_destroy(md_nlist* nl) {
  if (!nl) return MD_OK;
  if (nl->list) cudaFree(nl->list);
  if (nl->nnb) cudaFree(nl->nnb);
  if (nl->backup) cudaFree(nl->backup);
  delete nl;
  return MD_OK;
}

__global__ void k_clear_nl_flags(DevState* st) {
  st->flags &= ~FLAG_NL_OVERFLOW;
  st->max_nnb = 0;
}

extern "C" int md_nlist_rebuild(md_nlist* nl, md_system* sys, md_cell_list* cl) {
  if (!nl || !sys || !cl) return MD_ERR_BADARG;
  if (!cl->built) { md_set_error("md_nlist_rebuild: cell list not built"); return MD_ERR_BADARG; }
  k_clear_nl_flags<<<1, 1, 0, sys->stream>>>(sys->st);
  Recorder rec;
  rec.stream = sys->stream;
  if (int r = nlist_build_impl(nl, sys, cl, &rec, false)) return r;
  DevState hs;
  if (int r = sys->read_state(hs)) return r;
  if (hs.flags & FLAG_NL_OVERFLOW) {
    md_set_error("neighbour list overflow: %d entries for capacity %d", hs.max_nnb, nl->cap);
    return MD_ERR_NLIST_OVERFLOW;
  }
  return MD_OK;
}

extern "C" int md_nlist_fit(md_nlist* nl, md_system* sys, md_cell_list* cl) {
  for (int attempt = 0; attempt < 4; ++attempt) {
    int r = md_nlist_rebuild(nl, sys, cl);
    if (r != MD_ERR_NLIST_OVERFLOW) return r;
    DevState hs;
    if (int q = sys->read_state(hs)) return q;
    nl->cap = ((int)(hs.max_nnb * 1.2) + 32 + 31) & ~31;
    if (int q = alloc_lists(nl, sys)) return q;
  }
  return MD_ERR_NLIST_OVERFLOW;
}

extern "C" int md_nlist_capacity(md_nlist* nl, int* out) {
  if (!nl || !out) return MD_ERR_BADARG;
  *out = nl->cap;
  return MD_OK;
}

template <class R>
__global__ void k_max_disp(int N, const typename V4<R>::T* pos, const typename V4<R>::T* bk,
                           const DevState* st, double* partials, unsigned* counter, double* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (k < N) {
    typename V4<R>::T a = pos[k], b = bk[k];
    double dx = (double)min_image_exact(sub_rn(a.x, b.x), boxL<R>(st, 0), boxLi<R>(st, 0));
    double dy = (double)min_image_exact(sub_rn(a.y, b.y), boxL<R>(st, 1), boxLi<R>(st, 1));
    double dz = (double)min_image_exact(sub_rn(a.z, b.z), boxL<R>(st, 2), boxLi<R>(st, 2));
    v[0] = dx * dx + dy * dy + dz * dz;
  }
  // max via the sum machinery is wrong; do a block max then atomicMax on the bits
  double m = v[0];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned long long*)out, (unsigned long long)__double_as_longlong(m));
  (void)partials; (void)counter;
}

extern "C" int md_nlist_max_displacement(md_nlist* nl, md_system* sys, double* out) {
  if (!nl || !sys || !out) return MD_ERR_BADARG;
  if (!nl->built) { md_set_error("list not built"); return MD_ERR_BADARG; }
  double* d = nullptr;
  MD_CUDA(cudaMallocAsync((void**)&d, sizeof(double), sys->stream));
  MD_CUDA(cudaMemsetAsync(d, 0, sizeof(double), sys->stream));
  int nb = ceil_div(sys->N, 256);
  if (sys->prec == MD_PREC_FP64)
    k_max_disp<double><<<nb, 256, 0, sys->stream>>>(sys->N, (double4a*)sys->pos, (double4a*)nl->backup, sys->st, nullptr, nullptr, d);
  else
    k_max_disp<float><<<nb, 256, 0, sys->stream>>>(sys->N, (float4*)sys->pos, (float4*)nl->backup, sys->st, nullptr, nullptr, d);
  MD_CHECK_LAUNCH("max disp");
  double h = 0;
  MD_CUDA(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaFreeAsync(d, sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  *out = sqrt(h);
  return MD_OK;
}

extern "C" int md_nlist_sum_neighbor(md_nlist* nl, md_system* sys, int64_t* out) {
  if (!nl || !sys || !out) return MD_ERR_BADARG;
  std::vector<int> h(sys->N);
  MD_CUDA(cudaMemcpyAsync(h.data(), nl->nnb, sizeof(int) * sys->N, cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  int64_t s = 0;
  for (int v : h) s += (v < nl->cap ? v : nl->cap);
  *out = s;
  return MD_OK;
}

extern "C" int md_nlist_get(md_nlist* nl, md_system* sys, int32_t* counts, int32_t* pairs) {
  if (!nl || !sys || !counts) return MD_ERR_BADARG;
  int N = sys->N;
  std::vector<int> nnb(N), id(N);
  std::vector<int> lst((size_t)N * nl->cap);
  MD_CUDA(cudaMemcpyAsync(nnb.data(), nl->nnb, sizeof(int) * N, cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaMemcpyAsync(id.data(), sys->id, sizeof(int) * N, cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaMemcpyAsync(lst.data(), nl->list, sizeof(int) * (size_t)N * nl->cap, cudaMemcpyDeviceToHost, sys->stream));
  MD_CUDA(cudaStreamSynchronize(sys->stream));
  std::vector<int> slot_of(N);
  for (int k = 0; k < N; ++k) slot_of[id[k]] = k;
  size_t off = 0;
  for (int o = 0; o < N; ++o) {
    int k = slot_of[o];
    int c = nnb[k] < nl->cap ? nnb[k] : nl->cap;
    counts[o] = c;
    if (pairs)
      for (int t = 0; t < c; ++t) pairs[off + t] = id[lst[(size_t)k * nl->cap + nl_slot(t)] & 0x03FFFFFF];
    off += c;
  }
  return MD_OK;
}
