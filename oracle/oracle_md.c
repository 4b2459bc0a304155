/*
 * ORACLE -- test infrastructure only.  CPU restatement of the md.error force
 * path used as the parity checker by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference leg of bench.py.  Never linked into, or
 * called by, the product library.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).  Binary32
 * functions evaluate the reference's operation sequence in IEEE binary32,
 * round-to-nearest, no contraction -- the same contract as the CUDA kernels.
 * Paths cited relative to the md.error root; ENG = shortRange.inhomo/template/
 * tools/simulation.hetero.cutoff, UNI = .../simulation.uniform.cutoff.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

/* saturating float -> unsigned, round toward zero (the GPU cvt.rzi.u32.f32
   that `IndexType(x)` compiles to: negative and NaN give 0) */
static unsigned f2u_rz(float v) {
  if (!(v > 0.0f)) return 0u;
  if (v >= 4294967296.0f) return UINT_MAX;
  return (unsigned)v;
}
static unsigned d2u_rz(double v) {
  if (!(v > 0.0)) return 0u;
  if (v >= 4294967296.0) return UINT_MAX;
  return (unsigned)v;
}

/* box.sizei = 1/x in binary32 (ENG/include/BoxGeometry.h:100-111) */
void orc_box_inverse_f32(const float box[3], float inv[3]) {
  for (int d = 0; d < 3; ++d) inv[d] = 1.0f / box[d];
}

/* DecideNumCell (UNI/src/CellList_interface.cu:147-177): floor(L * (1/cellSize)) */
int orc_decide_ncell(const double box[3], double cell_size, int bdir, int divide, int ncell[3]) {
  double csi = 1. / cell_size;
  int mode = 1;
  for (int d = 0; d < 3; ++d) {
    int on = bdir & (1 << d);
    ncell[d] = on ? (int)floor(box[d] * csi) : 1;
    if (on && ncell[d] < 4) mode = 0;
  }
  if (mode)
    for (int d = 0; d < 3; ++d)
      if (bdir & (1 << d)) ncell[d] *= divide;
  return mode;
}

/* moveParticleToBox (ENG/include/BoxGeometry.h:80-96) then the cell index of
   naivelyBuildDeviceCellList2 (ENG/src/NeighborList.cu:101-124):
   IndexType(x * sizei * float(NCell)), wrap when == NCell, D3toD1
   (ENG/include/NeighborList.h:375-384).  pos/image updated in place. */
void orc_bin_f32(int n, float* pos, int* image, const float box[3], const int ncell[3],
                 uint32_t* cell) {
  float inv[3];
  orc_box_inverse_f32(box, inv);
  for (int i = 0; i < n; ++i) {
    unsigned c[3];
    for (int d = 0; d < 3; ++d) {
      float x = pos[3 * i + d];
      float t = floorf(x * inv[d]);
      image[3 * i + d] += (int)t;
      x = x - t * box[d];
      c[d] = f2u_rz((x * inv[d]) * (float)ncell[d]);
      if (c[d] == (unsigned)ncell[d]) {
        c[d] -= ncell[d];
        x = x - box[d];
        image[3 * i + d] += 1;
      }
      if (c[d] >= (unsigned)ncell[d]) c[d] = ncell[d] - 1;
      pos[3 * i + d] = x;
    }
    cell[i] = c[2] + (unsigned)ncell[2] * (c[1] + (unsigned)ncell[1] * c[0]);
  }
}

void orc_bin_f64(int n, double* pos, int* image, const double box[3], const int ncell[3],
                 uint32_t* cell) {
  double inv[3];
  for (int d = 0; d < 3; ++d) inv[d] = 1.0 / box[d];
  for (int i = 0; i < n; ++i) {
    unsigned c[3];
    for (int d = 0; d < 3; ++d) {
      double x = pos[3 * i + d];
      double t = floor(x * inv[d]);
      image[3 * i + d] += (int)t;
      x = x - t * box[d];
      c[d] = d2u_rz((x * inv[d]) * (double)ncell[d]);
      if (c[d] == (unsigned)ncell[d]) {
        c[d] -= ncell[d];
        x = x - box[d];
        image[3 * i + d] += 1;
      }
      if (c[d] >= (unsigned)ncell[d]) c[d] = ncell[d] - 1;
      pos[3 * i + d] = x;
    }
    cell[i] = c[2] + (unsigned)ncell[2] * (c[1] + (unsigned)ncell[1] * c[0]);
  }
}

/* shortestImage (ENG/include/BoxGeometry.h:176-179) */
static float mi_f32(float x, float L, float Li) { return x - floorf(x * Li + 0.5f) * L; }
static double mi_f64(double x, double L, double Li) { return x - floor(x * Li + 0.5) * L; }

/* buildDeviceNeighborList_AllPair (ENG/src/NeighborList.cu:327-420):
   diff = target - ref, shortestImage, keep if d2 < (rcut_i + rlistExten)^2, j != i.
   counts[i] = number kept (may exceed cap); pairs[i*cap + k] the first cap of them,
   ascending j.  O(N^2), OpenMP over i. */
void orc_nlist_allpair_f32(int n, const float* pos, const float* rcut, float skin,
                           const float box[3], int cap, int32_t* counts, int32_t* pairs) {
  float inv[3];
  orc_box_inverse_f32(box, inv);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) {
    const float rx = pos[3 * i], ry = pos[3 * i + 1], rz = pos[3 * i + 2];
    const float rl = rcut[i] + skin;
    const float rl2 = rl * rl;
    int c = 0;
    for (int j = 0; j < n; ++j) {
      float dx = pos[3 * j] - rx, dy = pos[3 * j + 1] - ry, dz = pos[3 * j + 2] - rz;
      dx = mi_f32(dx, box[0], inv[0]);
      dy = mi_f32(dy, box[1], inv[1]);
      dz = mi_f32(dz, box[2], inv[2]);
      float d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < rl2 && j != i) {
        if (c < cap) pairs[(size_t)i * cap + c] = j;
        ++c;
      }
    }
    counts[i] = c;
  }
}

void orc_nlist_allpair_f64(int n, const double* pos, const double* rcut, double skin,
                           const double box[3], int cap, int32_t* counts, int32_t* pairs) {
  double inv[3];
  for (int d = 0; d < 3; ++d) inv[d] = 1.0 / box[d];
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) {
    const double rx = pos[3 * i], ry = pos[3 * i + 1], rz = pos[3 * i + 2];
    const double rl = rcut[i] + skin;
    const double rl2 = rl * rl;
    int c = 0;
    for (int j = 0; j < n; ++j) {
      double dx = pos[3 * j] - rx, dy = pos[3 * j + 1] - ry, dz = pos[3 * j + 2] - rz;
      dx = mi_f64(dx, box[0], inv[0]);
      dy = mi_f64(dy, box[1], inv[1]);
      dz = mi_f64(dz, box[2], inv[2]);
      double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < rl2 && j != i) {
        if (c < cap) pairs[(size_t)i * cap + c] = j;
        ++c;
      }
    }
    counts[i] = c;
  }
}

/* buildCellNeighborhood (ENG/src/NeighborList.cu:170-257, divide 1) +
   buildDeviceNeighborList_DeviceCellList (UNI/src/NeighborList_interface.cu:361-491):
   stencil cells c_i + {-1,0,1}^3 with wrap and shiftNoi = +1 below 0, -1 above;
   shift = shiftNoi * box.size; diff = target - shift - ref; keep d2 < rlist^2.
   cell[] from orc_bin_f32 on the same (already normalised) positions. */
void orc_nlist_cellshift_f32(int n, const float* pos, const uint32_t* cell, float rlist,
                             const float box[3], const int ncell[3], int cap, int32_t* counts,
                             int32_t* pairs) {
  int ntot = ncell[0] * ncell[1] * ncell[2];
  int* cstart = (int*)calloc(ntot + 1, sizeof(int));
  int* members = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) cstart[cell[i] + 1]++;
  for (int c = 0; c < ntot; ++c) cstart[c + 1] += cstart[c];
  int* fill = (int*)calloc(ntot, sizeof(int));
  for (int i = 0; i < n; ++i) members[cstart[cell[i]] + fill[cell[i]]++] = i;
  const float rlist2 = rlist * rlist;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) {
    int cz = cell[i] % ncell[2];
    int cy = (cell[i] / ncell[2]) % ncell[1];
    int cx = cell[i] / (ncell[2] * ncell[1]);
    int c = 0;
    for (int ix = 0; ix < 3; ++ix)
      for (int iy = 0; iy < 3; ++iy)
        for (int iz = 0; iz < 3; ++iz) {
          int my[3] = {ix - 1 + cx, iy - 1 + cy, iz - 1 + cz};
          int sh[3] = {0, 0, 0};
          for (int d = 0; d < 3; ++d) {
            if (my[d] < 0) { my[d] += ncell[d]; sh[d] += 1; }
            else if (my[d] >= ncell[d]) { my[d] -= ncell[d]; sh[d] -= 1; }
          }
          float shift[3] = {sh[0] * box[0], sh[1] * box[1], sh[2] * box[2]};
          int tc = my[2] + ncell[2] * (my[1] + ncell[1] * my[0]);
          for (int m = cstart[tc]; m < cstart[tc + 1]; ++m) {
            int j = members[m];
            float dx = pos[3 * j] - shift[0] - pos[3 * i];
            float dy = pos[3 * j + 1] - shift[1] - pos[3 * i + 1];
            float dz = pos[3 * j + 2] - shift[2] - pos[3 * i + 2];
            if (dx * dx + dy * dy + dz * dz < rlist2 && j != i) {
              if (c < cap) pairs[(size_t)i * cap + c] = j;
              ++c;
            }
          }
        }
    counts[i] = c;
  }
  free(cstart);
  free(members);
  free(fill);
}

/* FP64 all-pairs LJ with the per-atom cutoff of the reference atom
   (calNonBondedInteraction_neighbor, ENG/src/InteractionEngine_interface.cu:1204-1281;
   LennardJones6_12::forcePoten, ENG/include/NonBondedInteraction.h:867-893):
     d = r_j - r_i (min image), keep if |d|^2 < rcut_i^2,
     F_i += 4 eps (6 s^6/r^6 - 12 s^12/r^12)/r^2 d,
     E  += 1/2 (4 eps (s^12/r^12 - s^6/r^6) + shift),  W_aa += 1/2 f_a d_a.
   When pos32 != NULL the pair decision is the binary32 test on pos32/rcut32
   (the interacting set of the single-precision kernels); the arithmetic is FP64.
   stats: [E, Wxx, Wyy, Wzz]. */
void orc_lj_allpair_f64(int n, const double* pos, const double* rcut, double eps, double sigma,
                        double shift, const double box[3], const float* pos32, const float* box32,
                        double* force, double* stats) {
  double inv[3];
  for (int d = 0; d < 3; ++d) inv[d] = 1.0 / box[d];
  float inv32[3] = {0, 0, 0};
  if (pos32) orc_box_inverse_f32(box32, inv32);
  const double e4 = 4.0 * eps, s2 = sigma * sigma;
  double E = 0, Wx = 0, Wy = 0, Wz = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : E, Wx, Wy, Wz)
  for (int i = 0; i < n; ++i) {
    double fx = 0, fy = 0, fz = 0;
    const double rc2 = rcut[i] * rcut[i];
    const float rc32 = (float)rcut[i];
    const float rc232 = rc32 * rc32;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double dx = mi_f64(pos[3 * j] - pos[3 * i], box[0], inv[0]);
      double dy = mi_f64(pos[3 * j + 1] - pos[3 * i + 1], box[1], inv[1]);
      double dz = mi_f64(pos[3 * j + 2] - pos[3 * i + 2], box[2], inv[2]);
      double r2 = dx * dx + dy * dy + dz * dz;
      int in;
      if (pos32) {
        float ex = mi_f32(pos32[3 * j] - pos32[3 * i], box32[0], inv32[0]);
        float ey = mi_f32(pos32[3 * j + 1] - pos32[3 * i + 1], box32[1], inv32[1]);
        float ez = mi_f32(pos32[3 * j + 2] - pos32[3 * i + 2], box32[2], inv32[2]);
        in = (ex * ex + ey * ey + ez * ez) < rc232;
      } else {
        in = r2 < rc2;
      }
      if (!in) continue;
      double ri2 = 1.0 / r2;
      double sr2 = s2 * ri2;
      double sr6 = sr2 * sr2 * sr2;
      double fs = e4 * (6.0 * sr6 - 12.0 * sr6 * sr6) * ri2;
      fx += fs * dx;
      fy += fs * dy;
      fz += fs * dz;
      E += 0.5 * (e4 * (sr6 * sr6 - sr6) + shift);
      Wx += 0.5 * fs * dx * dx;
      Wy += 0.5 * fs * dy * dy;
      Wz += 0.5 * fs * dz * dz;
    }
    force[3 * i] = fx;
    force[3 * i + 1] = fy;
    force[3 * i + 2] = fz;
  }
  if (stats) {
    stats[0] = E;
    stats[1] = Wx;
    stats[2] = Wy;
    stats[3] = Wz;
  }
}

/* The same with atom types (AtomNBForceTable::calForceIndex, ENG/include/
   NonBondedInteraction.h:673-683): the pair (type_i, type_j) takes the pair kind
   kind[type_i][type_j] with parameters tab[type_i][type_j][6] (nb_pair_d), or no force
   and no energy where the kind is 0 (mdForceNULL). */
/* One non-bonded pair of a kind of the nbForcePoten dispatch (ENG/include/
   NonBondedInteraction.h:556-600) for d = r_j - r_i: the force on i and the
   energy, the parameters as the *Parameter classes take them.
     kind 1 LennardJones6_12 (eps, sigma, shift)        :867-886
     kind 5 LennardJones6_12B (eps, sigma, shift, rcut) :1010-1031
     kind 3 CosTail (eps, b, wc)                        :1379-1440
   prec 0 follows the binary32 operations of those functions, prec 1 the same
   formulas in binary64 (the accurate cos and sin for the fast intrinsics). */
/* lj6_12_findCapR / lj6_12B_findCapR with the potential at the cap radius
   (NonBondedInteraction.h:1027-1073, :1204-1250), binary32 and binary64 */
static float capf_force(int bform, float eps, float sig, float rcut, float r) {
  const float dr2 = r * r;
  if (bform ? dr2 > rcut * rcut : dr2 >= rcut * rcut) return 0.f;
  const float ri = 1.f / r, ri2 = ri * ri, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
  return bform ? eps * (12.f * sri6 * sri6 - 12.f * sri6) * ri : 4.f * eps * (12.f * sri6 * sri6 - 6.f * sri6) * ri;
}
static void capf_radius(int bform, float eps, float sig, float sh, float rcut, float cap, float* R, float* P) {
  float point = 0.95f * rcut;
  while (capf_force(bform, eps, sig, rcut, point) < cap) point *= 0.95f;
  float lower = point, upper = rcut;
  while (fabsf(upper - lower) > 1e-4) {
    const float mid = 0.5f * (upper + lower);
    if (capf_force(bform, eps, sig, rcut, mid) > cap) lower = mid; else upper = mid;
  }
  *R = 0.5f * (upper + lower);
  const float dr2 = *R * *R;
  if (bform ? dr2 > rcut * rcut : dr2 >= rcut * rcut) { *P = 0.f; return; }
  const float ri = 1.f / *R, ri2 = ri * ri, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
  *P = bform ? eps * (sri6 * sri6 - 2.f * sri6 + sh) : 4.f * eps * (sri6 * sri6 - sri6) + sh;
}
static double capd_force(int bform, double eps, double sig, double rcut, double r) {
  const double dr2 = r * r;
  if (bform ? dr2 > rcut * rcut : dr2 >= rcut * rcut) return 0.;
  const double ri = 1. / r, ri2 = ri * ri, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
  return bform ? eps * (12. * sri6 * sri6 - 12. * sri6) * ri : 4. * eps * (12. * sri6 * sri6 - 6. * sri6) * ri;
}
static void capd_radius(int bform, double eps, double sig, double sh, double rcut, double cap, double* R, double* P) {
  double point = 0.95 * rcut;
  while (capd_force(bform, eps, sig, rcut, point) < cap) point *= 0.95;
  double lower = point, upper = rcut;
  while (fabs(upper - lower) > 1e-4) {
    const double mid = 0.5 * (upper + lower);
    if (capd_force(bform, eps, sig, rcut, mid) > cap) lower = mid; else upper = mid;
  }
  *R = 0.5 * (upper + lower);
  const double dr2 = *R * *R;
  if (bform ? dr2 > rcut * rcut : dr2 >= rcut * rcut) { *P = 0.; return; }
  const double ri = 1. / *R, ri2 = ri * ri, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
  *P = bform ? eps * (sri6 * sri6 - 2. * sri6 + sh) : 4. * eps * (sri6 * sri6 - sri6) + sh;
}

static float nb_pair_f(int kind, const double* u, float dx, float dy, float dz, float* f) {
  const float dr2 = dx * dx + dy * dy + dz * dz;
  float sc = 0.f, e = 0.f;
  if (kind == 1) {
    const float eps = (float)u[0], sig = (float)u[1], sh = (float)u[2];
    const float ri2 = 1.f / dr2, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
    sc = -4.f * eps * (12.f * sri6 * sri6 - 6.f * sri6) * ri2;
    e = 4.f * (eps * (sri6 * sri6 - sri6) + sh * 0.25f);
  } else if (kind == 5) {
    const float eps = (float)u[0], sig = (float)u[1], sh = (float)u[2], rc = (float)u[3];
    const float b = dr2 > rc * rc ? 0.f : 1.f;
    const float ri2 = 1.f / dr2, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
    sc = -b * eps * (12.f * sri6 * sri6 - 12.f * sri6) * ri2;
    e = b * (eps * (sri6 * sri6 - sri6 * 2.f + sh));
  } else if (kind == 2 || kind == 6) {
    const int bform = kind == 6;
    const float eps = (float)u[0], sig = (float)u[1], sh = (float)u[2], rc = (float)u[3], cap = (float)u[4];
    float R, P;
    capf_radius(bform, eps, sig, sh, rc, cap, &R, &P);
    if (bform ? dr2 > rc * rc : dr2 >= rc * rc) {
    } else if (dr2 < R * R) {
      const float s = 1.f / sqrtf(dx * dx + dy * dy + dz * dz);
      sc = -s * cap;
      e = -cap * (sqrtf(dr2) - R) + P;
    } else {
      const float ri2 = 1.f / dr2, sri2 = sig * sig * ri2, sri6 = sri2 * sri2 * sri2;
      sc = -(bform ? eps * (12.f * sri6 * sri6 - 12.f * sri6) * ri2 : 4.f * eps * (12.f * sri6 * sri6 - 6.f * sri6) * ri2);
      e = bform ? eps * (sri6 * sri6 - 2.f * sri6 + sh) : 4.f * eps * (sri6 * sri6 - sri6) + sh;
    }
  } else if (kind == 3 || kind == 4) {
    const float eps = (float)u[0], bv = (float)u[1], wc = (float)u[2];
    const float wci = wc != 0.f ? 1.f / wc : 0.f;
    const float rc = bv * powf(2.f, 1.f / 6.f), rcut = rc + wc;
    const float ri = 1.f / sqrtf(dr2);
    float R = 0.f, P = 0.f;
    if (kind == 4) capf_radius(0, eps, bv, 0.f, rc, (float)u[3], &R, &P);
    if (kind == 4 && dr2 < R * R) {
      const float s = 1.f / sqrtf(dx * dx + dy * dy + dz * dz);
      sc = -s * (float)u[3];
      e = -(float)u[3] * (sqrtf(dr2) - R) + P;
    } else if (dr2 <= rc * rc) {
      const float sri = bv * ri, sri2 = sri * sri, sri6 = sri2 * sri2 * sri2;
      sc = -24.f * eps * (2.f * sri6 * sri6 - sri6) * ri * ri;
      e = 4.f * eps * (sri6 * sri6 - sri6);
      if (wc == 0.f) e += eps;
    } else if (dr2 < rcut * rcut) {
      const float term = 0.5f * 3.14159265f * (dr2 * ri - rc) * wci;
      const float cost = cosf(term);
      sc = eps * 3.14159265f * wci * cost * sinf(term) * ri;
      e = -eps * cost * cost;
    }
  }
  f[0] = dx * sc; f[1] = dy * sc; f[2] = dz * sc;
  return e;
}

static double nb_pair_d(int kind, const double* u, double dx, double dy, double dz, double* f) {
  const double dr2 = dx * dx + dy * dy + dz * dz;
  double sc = 0., e = 0.;
  if (kind == 1) {
    const double ri2 = 1. / dr2, sri2 = u[1] * u[1] * ri2, sri6 = sri2 * sri2 * sri2;
    sc = -4. * u[0] * (12. * sri6 * sri6 - 6. * sri6) * ri2;
    e = 4. * (u[0] * (sri6 * sri6 - sri6) + u[2] * 0.25);
  } else if (kind == 5) {
    const double b = dr2 > u[3] * u[3] ? 0. : 1.;
    const double ri2 = 1. / dr2, sri2 = u[1] * u[1] * ri2, sri6 = sri2 * sri2 * sri2;
    sc = -b * u[0] * (12. * sri6 * sri6 - 12. * sri6) * ri2;
    e = b * (u[0] * (sri6 * sri6 - sri6 * 2. + u[2]));
  } else if (kind == 2 || kind == 6) {
    const int bform = kind == 6;
    double R, P;
    capd_radius(bform, u[0], u[1], u[2], u[3], u[4], &R, &P);
    if (bform ? dr2 > u[3] * u[3] : dr2 >= u[3] * u[3]) {
    } else if (dr2 < R * R) {
      const double s = 1. / sqrt(dr2);
      sc = -s * u[4];
      e = -u[4] * (sqrt(dr2) - R) + P;
    } else {
      const double ri2 = 1. / dr2, sri2 = u[1] * u[1] * ri2, sri6 = sri2 * sri2 * sri2;
      sc = -(bform ? u[0] * (12. * sri6 * sri6 - 12. * sri6) * ri2 : 4. * u[0] * (12. * sri6 * sri6 - 6. * sri6) * ri2);
      e = bform ? u[0] * (sri6 * sri6 - 2. * sri6 + u[2]) : 4. * u[0] * (sri6 * sri6 - sri6) + u[2];
    }
  } else if (kind == 3 || kind == 4) {
    const double eps = u[0], bv = u[1], wc = u[2];
    const double wci = wc != 0. ? 1. / wc : 0.;
    const double rc = bv * pow(2., 1. / 6.), rcut = rc + wc;
    const double ri = 1. / sqrt(dr2);
    double R = 0., P = 0.;
    if (kind == 4) capd_radius(0, eps, bv, 0., rc, u[3], &R, &P);
    if (kind == 4 && dr2 < R * R) {
      sc = -ri * u[3];
      e = -u[3] * (sqrt(dr2) - R) + P;
    } else if (dr2 <= rc * rc) {
      const double sri = bv * ri, sri2 = sri * sri, sri6 = sri2 * sri2 * sri2;
      sc = -24. * eps * (2. * sri6 * sri6 - sri6) * ri * ri;
      e = 4. * eps * (sri6 * sri6 - sri6);
      if (wc == 0.) e += eps;
    } else if (dr2 < rcut * rcut) {
      const double term = 0.5 * M_PI * (dr2 * ri - rc) * wci;
      const double cost = cos(term);
      sc = eps * M_PI * wci * cost * sin(term) * ri;
      e = -eps * cost * cost;
    }
  }
  f[0] = dx * sc; f[1] = dy * sc; f[2] = dz * sc;
  return e;
}

void orc_nb_pair(int kind, const double* u, int prec, const double* d, double* f, double* e) {
  if (prec == 0) {
    float ff[3];
    *e = nb_pair_f(kind, u, (float)d[0], (float)d[1], (float)d[2], ff);
    for (int k = 0; k < 3; ++k) f[k] = ff[k];
  } else {
    *e = nb_pair_d(kind, u, d[0], d[1], d[2], f);
  }
}

void orc_lj_allpair_typed(int n, const double* pos, const double* rcut, const int* type, int nt,
                          const double* tab, const int* kind, const double box[3], const float* pos32,
                          const float* box32, double* force, double* stats) {
  double inv[3];
  for (int d = 0; d < 3; ++d) inv[d] = 1.0 / box[d];
  float inv32[3] = {0, 0, 0};
  if (pos32) orc_box_inverse_f32(box32, inv32);
  double E = 0, Wx = 0, Wy = 0, Wz = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : E, Wx, Wy, Wz)
  for (int i = 0; i < n; ++i) {
    double fx = 0, fy = 0, fz = 0;
    const double rc2 = rcut[i] * rcut[i];
    const float rc32 = (float)rcut[i];
    const float rc232 = rc32 * rc32;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const int pr = type[i] * nt + type[j];
      if (!kind[pr]) continue;
      double dx = mi_f64(pos[3 * j] - pos[3 * i], box[0], inv[0]);
      double dy = mi_f64(pos[3 * j + 1] - pos[3 * i + 1], box[1], inv[1]);
      double dz = mi_f64(pos[3 * j + 2] - pos[3 * i + 2], box[2], inv[2]);
      double r2 = dx * dx + dy * dy + dz * dz;
      int in;
      if (pos32) {
        float ex = mi_f32(pos32[3 * j] - pos32[3 * i], box32[0], inv32[0]);
        float ey = mi_f32(pos32[3 * j + 1] - pos32[3 * i + 1], box32[1], inv32[1]);
        float ez = mi_f32(pos32[3 * j + 2] - pos32[3 * i + 2], box32[2], inv32[2]);
        in = (ex * ex + ey * ey + ez * ez) < rc232;
      } else {
        in = r2 < rc2;
      }
      if (!in) continue;
      double f[3];
      const double e = nb_pair_d(kind[pr], tab + 6 * pr, dx, dy, dz, f);
      fx += f[0];
      fy += f[1];
      fz += f[2];
      E += 0.5 * e;
      Wx += 0.5 * f[0] * dx;
      Wy += 0.5 * f[1] * dy;
      Wz += 0.5 * f[2] * dz;
    }
    force[3 * i] = fx;
    force[3 * i + 1] = fy;
    force[3 * i + 2] = fz;
  }
  stats[0] = E;
  stats[1] = Wx;
  stats[2] = Wy;
  stats[3] = Wz;
}

/* AssignRCut::assign index (ENG/src/AssignRCut.cu:93-112) in binary32 */
float orc_lattice_rcut_f32(float x, float y, float z, const float box[3], const float* lat,
                           int nx, int ny, int nz) {
  if (x < 0) x += box[0]; else if (x >= box[0]) x -= box[0];
  if (y < 0) y += box[1]; else if (y >= box[1]) y -= box[1];
  if (z < 0) z += box[2]; else if (z >= box[2]) z -= box[2];
  int ix = (int)((x * (float)nx) / box[0]);
  int iy = (int)((y * (float)ny) / box[1]);
  int iz = (int)((z * (float)nz) / box[2]);
  if (ix < 0) ix = 0; if (ix >= nx) ix = nx - 1;
  if (iy < 0) iy = 0; if (iy >= ny) iy = ny - 1;
  if (iz < 0) iz = 0; if (iz >= nz) iz = nz - 1;
  return lat[iz + nz * (iy + ny * ix)];
}

void orc_assign_rcut_f32(int n, const float* pos, const float box[3], const float* lat, int nx,
                         int ny, int nz, float* rcut) {
  for (int i = 0; i < n; ++i)
    rcut[i] = orc_lattice_rcut_f32(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], box, lat, nx, ny, nz);
}
