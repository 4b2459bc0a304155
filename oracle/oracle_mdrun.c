/*
 * ORACLE -- test infrastructure only.  CPU FP64 restatement of the Langevin
 * MD step (cell list + Verlet list with skin, per-atom adaptive LJ cutoff,
 * BAOAB Langevin NVT/NPT) used (a) as the trajectory checker of the GPU
 * driver and (b) as the timed CPU arm of bench.py (`--impl reference`,
 * cpu_baseline).  OpenMP over atoms.
 *
 * Semantics followed:
 *  - LJ force / cutoff: ENG/src/InteractionEngine_interface.cu:1204-1281,
 *    ENG/include/NonBondedInteraction.h:867-893 (cutoff of atom i only).
 *  - list radius rcut_i + skin, rebuild when max |dr| > skin/2:
 *    ENG/src/NeighborList.cu:327-420, ENG/app/lj.nhc-xtc.cu:169-181.
 *  - moveParticleToBox before a rebuild: ENG/include/BoxGeometry.h:80-96.
 *  - per-atom rcut from the lattice at each rebuild: ENG/src/AssignRCut.cu:78-117.
 *  - Langevin NVT/NPT equations: langevin.npt/writedown/paper.tex:355-369,
 *    382-440, 586-600, integrated with the same BAOAB splitting, Philox-4x32-10
 *    normal stream and box-length piston as the CUDA driver.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

float orc_lattice_rcut_f32(float x, float y, float z, const float box[3], const float* lat,
                           int nx, int ny, int nz);

/* ---- Philox-4x32-10 (Salmon et al., SC'11), same counter layout as the device */
static void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t y0 = hi1 ^ c[1] ^ k0, y1 = lo1, y2 = hi0 ^ c[3] ^ k1, y3 = lo0;
    c[0] = y0; c[1] = y1; c[2] = y2; c[3] = y3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

/* raw generator, for the published known-answer vectors */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  philox(c, key[0], key[1]);
  memcpy(out, c, sizeof(c));
}

void orc_normals4(uint64_t seed, uint64_t step, uint32_t id, double out[4]) {
  uint32_t c[4] = {id, (uint32_t)step, (uint32_t)(step >> 32), 0x6d646672u};
  philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double inv = 2.3283064365386963e-10;
  double u1 = ((double)c[0] + 0.5) * inv, u2 = ((double)c[1] + 0.5) * inv;
  double u3 = ((double)c[2] + 0.5) * inv, u4 = ((double)c[3] + 0.5) * inv;
  double m1 = sqrt(-2.0 * log(u1)), m2 = sqrt(-2.0 * log(u3));
  out[0] = m1 * cos(2.0 * M_PI * u2);
  out[1] = m1 * sin(2.0 * M_PI * u2);
  out[2] = m2 * cos(2.0 * M_PI * u4);
  out[3] = m2 * sin(2.0 * M_PI * u4);
}

typedef struct {
  double dt, temperature, gamma_t, tau_p, kappa_t, p_ref[3];
  int npt_dirs;
  uint64_t seed;
  double skin, eps, sigma, shift;
} orc_lv_params;

typedef struct {
  int n, cap;
  double* pos;
  double* vel;
  double* invm;
  double* force;
  double* backup;
  float* rcut;
  int* image;
  int* nnb;
  int* list;
  double L[3];
  double ph[3], Mh[3], Pcur[3];
  double stats[8]; /* E, Wxx, Wyy, Wzz, Kxx, Kyy, Kzz */
  uint64_t step;
  int64_t rebuilds;
  const float* lat;
  int lat_n[3];
} orc_state;

static double mi(double x, double L, double Li) { return x - floor(x * Li + 0.5) * L; }

static void wrap_and_rcut(orc_state* s) {
  for (int i = 0; i < s->n; ++i) {
    for (int d = 0; d < 3; ++d) {
      double x = s->pos[3 * i + d];
      double t = floor(x * (1.0 / s->L[d]));
      s->image[3 * i + d] += (int)t;
      s->pos[3 * i + d] = x - t * s->L[d];
    }
    if (s->lat) {
      float bf[3] = {(float)s->L[0], (float)s->L[1], (float)s->L[2]};
      s->rcut[i] = orc_lattice_rcut_f32((float)s->pos[3 * i], (float)s->pos[3 * i + 1],
                                        (float)s->pos[3 * i + 2], bf, s->lat, s->lat_n[0],
                                        s->lat_n[1], s->lat_n[2]);
    }
  }
}

/* cell-list Verlet build, radius rcut_i + skin, minimum image; returns max count */
static int build_list(orc_state* s, double skin) {
  double rmax = 0;
  for (int i = 0; i < s->n; ++i) rmax = s->rcut[i] > rmax ? s->rcut[i] : rmax;
  double rl = rmax + skin;
  int nc[3];
  for (int d = 0; d < 3; ++d) {
    nc[d] = (int)floor(s->L[d] / rl);
    if (nc[d] < 3) nc[d] = 1;
  }
  int ntot = nc[0] * nc[1] * nc[2];
  int* cst = (int*)calloc(ntot + 1, sizeof(int));
  int* cof = (int*)malloc(sizeof(int) * s->n);
  int* mem = (int*)malloc(sizeof(int) * s->n);
  int* fill = (int*)calloc(ntot, sizeof(int));
  for (int i = 0; i < s->n; ++i) {
    int c[3];
    for (int d = 0; d < 3; ++d) {
      c[d] = (int)(s->pos[3 * i + d] / s->L[d] * nc[d]);
      if (c[d] < 0) c[d] = 0;
      if (c[d] >= nc[d]) c[d] = nc[d] - 1;
    }
    cof[i] = c[2] + nc[2] * (c[1] + nc[1] * c[0]);
    cst[cof[i] + 1]++;
  }
  for (int c = 0; c < ntot; ++c) cst[c + 1] += cst[c];
  for (int i = 0; i < s->n; ++i) mem[cst[cof[i]] + fill[cof[i]]++] = i;
  double Li[3] = {1.0 / s->L[0], 1.0 / s->L[1], 1.0 / s->L[2]};
  int maxc = 0;
#pragma omp parallel for schedule(dynamic, 32) reduction(max : maxc)
  for (int i = 0; i < s->n; ++i) {
    int cz = cof[i] % nc[2], cy = (cof[i] / nc[2]) % nc[1], cx = cof[i] / (nc[2] * nc[1]);
    double r = s->rcut[i] + skin, r2 = r * r;
    int cnt = 0;
    int lo[3], hi[3];
    int cc[3] = {cx, cy, cz};
    for (int d = 0; d < 3; ++d) {
      if (nc[d] == 1) { lo[d] = 0; hi[d] = 0; }
      else { lo[d] = cc[d] - 1; hi[d] = cc[d] + 1; }
    }
    for (int ax = lo[0]; ax <= hi[0]; ++ax)
      for (int ay = lo[1]; ay <= hi[1]; ++ay)
        for (int az = lo[2]; az <= hi[2]; ++az) {
          int tx = (ax + nc[0]) % nc[0], ty = (ay + nc[1]) % nc[1], tz = (az + nc[2]) % nc[2];
          int tc = tz + nc[2] * (ty + nc[1] * tx);
          for (int m = cst[tc]; m < cst[tc + 1]; ++m) {
            int j = mem[m];
            if (j == i) continue;
            double dx = mi(s->pos[3 * j] - s->pos[3 * i], s->L[0], Li[0]);
            double dy = mi(s->pos[3 * j + 1] - s->pos[3 * i + 1], s->L[1], Li[1]);
            double dz = mi(s->pos[3 * j + 2] - s->pos[3 * i + 2], s->L[2], Li[2]);
            if (dx * dx + dy * dy + dz * dz < r2) {
              if (cnt < s->cap) s->list[(size_t)i * s->cap + cnt] = j;
              ++cnt;
            }
          }
        }
    s->nnb[i] = cnt;
    if (cnt > maxc) maxc = cnt;
  }
  memcpy(s->backup, s->pos, sizeof(double) * 3 * s->n);
  free(cst); free(cof); free(mem); free(fill);
  return maxc;
}

static void forces(orc_state* s, const orc_lv_params* p) {
  const double e4 = 4.0 * p->eps, s2 = p->sigma * p->sigma;
  double Li[3] = {1.0 / s->L[0], 1.0 / s->L[1], 1.0 / s->L[2]};
  double E = 0, Wx = 0, Wy = 0, Wz = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : E, Wx, Wy, Wz)
  for (int i = 0; i < s->n; ++i) {
    double fx = 0, fy = 0, fz = 0;
    double rc2 = (double)s->rcut[i] * (double)s->rcut[i];
    int c = s->nnb[i] < s->cap ? s->nnb[i] : s->cap;
    for (int k = 0; k < c; ++k) {
      int j = s->list[(size_t)i * s->cap + k];
      double dx = mi(s->pos[3 * j] - s->pos[3 * i], s->L[0], Li[0]);
      double dy = mi(s->pos[3 * j + 1] - s->pos[3 * i + 1], s->L[1], Li[1]);
      double dz = mi(s->pos[3 * j + 2] - s->pos[3 * i + 2], s->L[2], Li[2]);
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rc2) {
        double ri2 = 1.0 / r2, sr2 = s2 * ri2, sr6 = sr2 * sr2 * sr2;
        double fs = e4 * (6.0 * sr6 - 12.0 * sr6 * sr6) * ri2;
        fx += fs * dx; fy += fs * dy; fz += fs * dz;
        E += 0.5 * (e4 * (sr6 * sr6 - sr6) + p->shift);
        Wx += 0.5 * fs * dx * dx; Wy += 0.5 * fs * dy * dy; Wz += 0.5 * fs * dz * dz;
      }
    }
    s->force[3 * i] = fx; s->force[3 * i + 1] = fy; s->force[3 * i + 2] = fz;
  }
  s->stats[0] = E; s->stats[1] = Wx; s->stats[2] = Wy; s->stats[3] = Wz;
}

static void kick_kinetic(orc_state* s, const orc_lv_params* p, double dt, const double* pcorr) {
  double K[3] = {0, 0, 0};
  for (int i = 0; i < s->n; ++i) {
    for (int d = 0; d < 3; ++d) {
      s->vel[3 * i + d] += 0.5 * dt * s->force[3 * i + d] * s->invm[i];
      K[d] += 0.5 / s->invm[i] * s->vel[3 * i + d] * s->vel[3 * i + d];
    }
  }
  double V = s->L[0] * s->L[1] * s->L[2];
  for (int d = 0; d < 3; ++d) {
    s->stats[4 + d] = K[d];
    s->Pcur[d] = 2.0 / V * (K[d] - 0.5 * s->stats[1 + d]) + (pcorr ? pcorr[d] : 0.0);
    if (p->npt_dirs & (1 << d)) s->ph[d] += 0.5 * dt * V / s->L[d] * (s->Pcur[d] - p->p_ref[d]);
  }
}

/* Run nsteps of Langevin dynamics.  pos/vel/box are in/out (pos returned
   wrapped as of the last rebuild plus drift, like the device arrays); rcut is
   used when lat == NULL; stats_out (7): E, Wxx, Wyy, Wzz, Kxx, Kyy, Kzz after
   the last step; counters_out (2): rebuilds, max list length.
   Returns 0, or 2 when a list outgrew cap (mdErrorShortNeighborList). */
int orc_md_langevin_run(int n, double* pos, double* vel, const double* mass, const float* rcut,
                        const float* lat, int nx, int ny, int nz, double box[3],
                        const orc_lv_params* p, const double* pcorr, int nsteps, int cap,
                        double* stats_out, int64_t* counters_out) {
  orc_state s;
  memset(&s, 0, sizeof(s));
  s.n = n;
  s.cap = cap;
  s.pos = pos;
  s.vel = vel;
  s.invm = (double*)malloc(sizeof(double) * n);
  s.force = (double*)calloc(3 * (size_t)n, sizeof(double));
  s.backup = (double*)malloc(sizeof(double) * 3 * n);
  s.rcut = (float*)malloc(sizeof(float) * n);
  s.image = (int*)calloc(3 * (size_t)n, sizeof(int));
  s.nnb = (int*)calloc(n, sizeof(int));
  s.list = (int*)malloc(sizeof(int) * (size_t)n * cap);
  s.lat = lat;
  s.lat_n[0] = nx; s.lat_n[1] = ny; s.lat_n[2] = nz;
  for (int i = 0; i < n; ++i) {
    s.invm[i] = mass ? 1.0 / mass[i] : 1.0;
    s.rcut[i] = rcut ? rcut[i] : 0.f;
  }
  for (int d = 0; d < 3; ++d) s.L[d] = box[d];
  double V = s.L[0] * s.L[1] * s.L[2];
  for (int d = 0; d < 3; ++d) {
    double A = V / s.L[d], w = 2.0 * M_PI / (p->tau_p > 0 ? p->tau_p : 1.0);
    s.Mh[d] = A * A / (p->kappa_t > 0 ? p->kappa_t * V : 1.0) / (w * w);
  }
  const double c1 = exp(-p->gamma_t * p->dt), c2 = sqrt(1.0 - c1 * c1);
  const double gp = p->tau_p > 0 ? 1.0 / p->tau_p : 0.0;
  const double c1p = exp(-gp * p->dt), c2p = sqrt(1.0 - c1p * c1p);
  const double h = 0.5 * p->dt, sh2 = 0.25 * p->skin * p->skin;
  int status = 0, maxc;
  wrap_and_rcut(&s);
  maxc = build_list(&s, p->skin);
  if (maxc > cap) status = 2;
  forces(&s, p);
  kick_kinetic(&s, p, 0.0, pcorr);
  for (int it = 0; it < nsteps; ++it) {
    s.step += 1;
    double lam1[3] = {1, 1, 1}, lam2[3] = {1, 1, 1};
    double xi[4];
    orc_normals4(p->seed ^ 0x5bd1e995ull, s.step, 0xffffffffu, xi);
    if (p->npt_dirs) {
      double Vb = s.L[0] * s.L[1] * s.L[2];
      for (int d = 0; d < 3; ++d) {
        if (!(p->npt_dirs & (1 << d))) continue;
        double A = Vb / s.L[d], ph = s.ph[d], M = s.Mh[d];
        ph += h * A * (s.Pcur[d] - p->p_ref[d]);
        double L0 = s.L[d], L1 = L0 + h * ph / M;
        ph = c1p * ph + c2p * sqrt(M * p->temperature) * xi[d];
        double L2 = L1 + h * ph / M;
        lam1[d] = L1 / L0; lam2[d] = L2 / L1;
        s.ph[d] = ph; s.L[d] = L2;
      }
    }
    int far = 0;
    double Li[3] = {1.0 / s.L[0], 1.0 / s.L[1], 1.0 / s.L[2]};
#pragma omp parallel for schedule(static) reduction(| : far)
    for (int i = 0; i < n; ++i) {
      double v[3], r[3], z[4];
      for (int d = 0; d < 3; ++d) {
        v[d] = s.vel[3 * i + d] + h * s.force[3 * i + d] * s.invm[i];
        r[d] = s.pos[3 * i + d];
      }
      for (int d = 0; d < 3; ++d) { r[d] = lam1[d] * r[d] + h * v[d]; v[d] /= lam1[d]; }
      orc_normals4(p->seed, s.step, (uint32_t)i, z);
      double sd = c2 * sqrt(p->temperature * s.invm[i]);
      for (int d = 0; d < 3; ++d) v[d] = c1 * v[d] + sd * z[d];
      for (int d = 0; d < 3; ++d) { r[d] = lam2[d] * r[d] + h * v[d]; v[d] /= lam2[d]; }
      double d2 = 0;
      for (int d = 0; d < 3; ++d) {
        s.pos[3 * i + d] = r[d];
        s.vel[3 * i + d] = v[d];
        double dd = mi(r[d] - s.backup[3 * i + d], s.L[d], Li[d]);
        d2 += dd * dd;
      }
      if (d2 > sh2) far = 1;
    }
    if (far) {
      s.rebuilds++;
      wrap_and_rcut(&s);
      maxc = build_list(&s, p->skin);
      if (maxc > cap) status = 2;
    }
    forces(&s, p);
    kick_kinetic(&s, p, p->dt, pcorr);
  }
  for (int d = 0; d < 3; ++d) box[d] = s.L[d];
  if (stats_out) memcpy(stats_out, s.stats, sizeof(double) * 7);
  if (counters_out) { counters_out[0] = s.rebuilds; counters_out[1] = maxc; }
  free(s.invm); free(s.force); free(s.backup); free(s.rcut); free(s.image); free(s.nnb); free(s.list);
  return status;
}

/* ---------------------------------------------------------------- NHC NVT
 * The step of ENG/app/lj.nhc-xtc.cu:159-200 restated literally in FP64:
 * COM velocity removal (TranslationalFreedomRemover), NoseHoover_Chains2::
 * operator_L(dt/2) (ENG/src/Thermostat.cu:255-275: the kinetic energy summed
 * again after the velocity scaling), velocity Verlet step1, displacement test
 * and rebuild, forces, step2, operator_L(dt/2). */
typedef struct {
  double xi1, xi2, vxi1, vxi2, Q1, Q2, LL, T;
} orc_nhc;

static double kinetic_sum(const orc_state* s, double K3[3]) {
  double K[3] = {0, 0, 0};
  for (int i = 0; i < s->n; ++i)
    for (int d = 0; d < 3; ++d) K[d] += 0.5 / s->invm[i] * s->vel[3 * i + d] * s->vel[3 * i + d];
  if (K3) for (int d = 0; d < 3; ++d) K3[d] = K[d];
  return K[0] + K[1] + K[2];
}

static void nhc_L(orc_state* s, orc_nhc* c, double dt, double K3out[3]) {
  c->vxi2 += (c->Q1 * c->vxi1 * c->vxi1 - c->T) / c->Q2 * (0.5 * dt);        /* G2 */
  c->vxi1 *= exp(-c->vxi2 * 0.25 * dt);                                      /* vxi1 */
  c->vxi1 += (2.0 * kinetic_sum(s, NULL) - c->LL * c->T) / c->Q1 * (0.5 * dt); /* G1 */
  c->vxi1 *= exp(-c->vxi2 * 0.25 * dt);
  const double a = exp(-c->vxi1 * dt);                                       /* Cv */
  for (int k = 0; k < 3 * s->n; ++k) s->vel[k] *= a;
  c->xi1 += c->vxi1 * dt;                                                    /* xi */
  c->xi2 += c->vxi2 * dt;
  c->vxi1 *= exp(-c->vxi2 * 0.25 * dt);
  c->vxi1 += (2.0 * kinetic_sum(s, K3out) - c->LL * c->T) / c->Q1 * (0.5 * dt);
  c->vxi1 *= exp(-c->vxi2 * 0.25 * dt);
  c->vxi2 += (c->Q1 * c->vxi1 * c->vxi1 - c->T) / c->Q2 * (0.5 * dt);
}

static void remove_com(orc_state* s) {
  double P[3] = {0, 0, 0}, M = 0;
  for (int i = 0; i < s->n; ++i) {
    const double m = 1.0 / s->invm[i];
    M += m;
    for (int d = 0; d < 3; ++d) P[d] += m * s->vel[3 * i + d];
  }
  for (int i = 0; i < s->n; ++i)
    for (int d = 0; d < 3; ++d) s->vel[3 * i + d] -= P[d] / M;
}

/* p: dt, temperature (target T), gamma_t (unused), tau_p = tau_T of the chain,
   skin, eps, sigma, shift.  stats_out (7): E, Wxx..Wzz, Kxx..Kzz after the last
   step; nhc_out (5): xi1, xi2, vxi1, vxi2, HamiltonianContribution. */
int orc_md_nhc_run(int n, double* pos, double* vel, const double* mass, const float* rcut, double box[3],
                   const orc_lv_params* p, int remove_com_flag, int nsteps, int cap, double* stats_out,
                   double* nhc_out, int64_t* counters_out) {
  orc_state s;
  memset(&s, 0, sizeof(s));
  s.n = n;
  s.cap = cap;
  s.pos = pos;
  s.vel = vel;
  s.invm = (double*)malloc(sizeof(double) * n);
  s.force = (double*)calloc(3 * (size_t)n, sizeof(double));
  s.backup = (double*)malloc(sizeof(double) * 3 * n);
  s.rcut = (float*)malloc(sizeof(float) * n);
  s.image = (int*)calloc(3 * (size_t)n, sizeof(int));
  s.nnb = (int*)calloc(n, sizeof(int));
  s.list = (int*)malloc(sizeof(int) * (size_t)n * cap);
  for (int i = 0; i < n; ++i) {
    s.invm[i] = mass ? 1.0 / mass[i] : 1.0;
    s.rcut[i] = rcut[i];
  }
  for (int d = 0; d < 3; ++d) s.L[d] = box[d];
  orc_nhc c;
  c.LL = 3.0 * n;
  c.T = p->temperature;
  c.Q1 = p->tau_p * p->tau_p * c.T / (4 * M_PI * M_PI) * c.LL;
  c.Q2 = c.Q1 / c.LL;
  c.xi1 = c.xi2 = 1.0;
  c.vxi1 = c.vxi2 = 0.0;
  const double h = 0.5 * p->dt, sh2 = 0.25 * p->skin * p->skin;
  int status = 0, maxc;
  wrap_and_rcut(&s);
  maxc = build_list(&s, p->skin);
  if (maxc > cap) status = 2;
  forces(&s, p);
  double K3[3] = {0, 0, 0};
  for (int it = 0; it < nsteps; ++it) {
    if (remove_com_flag) remove_com(&s);
    nhc_L(&s, &c, h, NULL);
    int far = 0;
    double Li[3] = {1.0 / s.L[0], 1.0 / s.L[1], 1.0 / s.L[2]};
    for (int i = 0; i < n; ++i) {
      double d2 = 0;
      for (int d = 0; d < 3; ++d) {
        s.vel[3 * i + d] += h * s.force[3 * i + d] * s.invm[i];
        s.pos[3 * i + d] += p->dt * s.vel[3 * i + d];
        double dd = mi(s.pos[3 * i + d] - s.backup[3 * i + d], s.L[d], Li[d]);
        d2 += dd * dd;
      }
      if (d2 > sh2) far = 1;
    }
    if (far) {
      s.rebuilds++;
      wrap_and_rcut(&s);
      maxc = build_list(&s, p->skin);
      if (maxc > cap) status = 2;
    }
    forces(&s, p);
    for (int k = 0; k < 3 * n; ++k) s.vel[k] += h * s.force[k] * s.invm[k / 3];
    nhc_L(&s, &c, h, K3);
  }
  for (int d = 0; d < 3; ++d) s.stats[4 + d] = K3[d];
  if (stats_out) memcpy(stats_out, s.stats, sizeof(double) * 7);
  if (nhc_out) {
    nhc_out[0] = c.xi1; nhc_out[1] = c.xi2; nhc_out[2] = c.vxi1; nhc_out[3] = c.vxi2;
    nhc_out[4] = 0.5 * c.Q1 * c.vxi1 * c.vxi1 + 0.5 * c.Q2 * c.vxi2 * c.vxi2 + c.LL * c.T * c.xi1 + c.T * c.xi2;
  }
  if (counters_out) { counters_out[0] = s.rebuilds; counters_out[1] = maxc; }
  free(s.invm); free(s.force); free(s.backup); free(s.rcut); free(s.image); free(s.nnb); free(s.list);
  return status;
}

/* ---------------------------------------------------------------- NHC NPT
 * NoseHoover_Chains2_Isobaric operators (ENG/src/Barostat.cu:6-460) restated
 * literally in FP64 (velocities scaled in place, K summed again), composed
 * into the MTK step L_CP(dt/2) L_v(dt/2) L_r(dt) L_box(dt) | list + forces |
 * L_v(dt/2) L_CP(dt/2); the list is rebuilt every step. */
typedef struct {
  double ep, vep, xi1, vxi1, Nf, Q1, W, T, Pref, pcorr;
} orc_nhcp;

static double nhcp_P(const orc_state* s, const orc_nhcp* c, const double K[3]) {
  const double V = s->L[0] * s->L[1] * s->L[2];
  double P = 0;
  for (int d = 0; d < 3; ++d) P += 2.0 / V * (K[d] - 0.5 * s->stats[1 + d]);
  return P / 3.0 + c->pcorr;
}

static void nhcp_L_CP(orc_state* s, orc_nhcp* c, double t) {
  const double V = s->L[0] * s->L[1] * s->L[2];
  double K3[3];
  double K = kinetic_sum(s, K3);
  c->vxi1 += (2.0 * K + c->W * c->vep * c->vep - (c->Nf + 1.0) * c->T) / c->Q1 * (0.5 * t); /* G1 */
  c->vep *= exp(-c->vxi1 * 0.25 * t);                                                        /* vep */
  c->vep += (6.0 / c->Nf * K + 3.0 * V * (nhcp_P(s, c, K3) - c->Pref)) / c->W * (0.5 * t);   /* Gep */
  c->vep *= exp(-c->vxi1 * 0.25 * t);
  const double a = exp(-(c->vxi1 + (1.0 + 3.0 / c->Nf) * c->vep) * t);                       /* Cv */
  for (int k = 0; k < 3 * s->n; ++k) s->vel[k] *= a;
  K = kinetic_sum(s, K3);
  c->xi1 += c->vxi1 * t;                                                                     /* xi */
  c->vep *= exp(-c->vxi1 * 0.25 * t);
  c->vep += (6.0 / c->Nf * K + 3.0 * V * (nhcp_P(s, c, K3) - c->Pref)) / c->W * (0.5 * t);
  c->vep *= exp(-c->vxi1 * 0.25 * t);
  c->vxi1 += (2.0 * K + c->W * c->vep * c->vep - (c->Nf + 1.0) * c->T) / c->Q1 * (0.5 * t);
  for (int d = 0; d < 3; ++d) s->stats[4 + d] = K3[d];
}

/* p: dt, temperature, gamma_t = tau_T, tau_p = tau_P, p_ref[0] = P_ref, skin, LJ;
   pcorr: constant pressure correction.  state_out (5): ep, vep, xi1, vxi1, H. */
int orc_md_nhc_npt_run(int n, double* pos, double* vel, const double* mass, const float* rcut, double box[3],
                       const orc_lv_params* p, double pcorr, int nsteps, int cap, double* stats_out,
                       double* state_out) {
  orc_state s;
  memset(&s, 0, sizeof(s));
  s.n = n;
  s.cap = cap;
  s.pos = pos;
  s.vel = vel;
  s.invm = (double*)malloc(sizeof(double) * n);
  s.force = (double*)calloc(3 * (size_t)n, sizeof(double));
  s.backup = (double*)malloc(sizeof(double) * 3 * n);
  s.rcut = (float*)malloc(sizeof(float) * n);
  s.image = (int*)calloc(3 * (size_t)n, sizeof(int));
  s.nnb = (int*)calloc(n, sizeof(int));
  s.list = (int*)malloc(sizeof(int) * (size_t)n * cap);
  for (int i = 0; i < n; ++i) {
    s.invm[i] = mass ? 1.0 / mass[i] : 1.0;
    s.rcut[i] = rcut[i];
  }
  for (int d = 0; d < 3; ++d) s.L[d] = box[d];
  orc_nhcp c;
  c.Nf = 3.0 * n - 3.0;
  c.T = p->temperature;
  c.Q1 = p->gamma_t * p->gamma_t * c.T * c.Nf;
  c.W = p->tau_p * p->tau_p * c.T * c.Nf;
  c.Pref = p->p_ref[0];
  c.pcorr = pcorr;
  c.ep = log(s.L[0] * s.L[1] * s.L[2]) / 3.0;
  c.vep = 0.0;
  c.xi1 = 1.0;
  c.vxi1 = 0.0;
  const double h = 0.5 * p->dt;
  int status = 0;
  wrap_and_rcut(&s);
  if (build_list(&s, p->skin) > cap) status = 2;
  forces(&s, p);
  for (int it = 0; it < nsteps; ++it) {
    nhcp_L_CP(&s, &c, h);
    for (int k = 0; k < 3 * n; ++k) s.vel[k] += h * s.force[k] * s.invm[k / 3];      /* L_v */
    {                                                                                 /* L_r */
      const double xx = c.vep * p->dt * 0.5, s1 = exp(c.vep * p->dt);
      const double x2 = xx * xx, x4 = x2 * x2, x6 = x4 * x2, x8 = x6 * x2, x10 = x8 * x2;
      const double s2 = p->dt * exp(xx) *
                        (1. + 1. / 6. * x2 + 1. / 120. * x4 + 1. / 5040. * x6 + 1. / 362880. * x8 +
                         1. / 39916800. * x10);
      for (int k = 0; k < 3 * n; ++k) s.pos[k] = s1 * s.pos[k] + s2 * s.vel[k];
    }
    {                                                                                 /* L_box */
      const double sc = exp(c.vep * p->dt);
      for (int d = 0; d < 3; ++d) s.L[d] *= sc;
      c.ep += p->dt * c.vep;
    }
    wrap_and_rcut(&s);
    if (build_list(&s, p->skin) > cap) status = 2;
    forces(&s, p);
    for (int k = 0; k < 3 * n; ++k) s.vel[k] += h * s.force[k] * s.invm[k / 3];
    nhcp_L_CP(&s, &c, h);
  }
  for (int d = 0; d < 3; ++d) box[d] = s.L[d];
  if (stats_out) memcpy(stats_out, s.stats, sizeof(double) * 7);
  if (state_out) {
    const double V = s.L[0] * s.L[1] * s.L[2];
    state_out[0] = c.ep; state_out[1] = c.vep; state_out[2] = c.xi1; state_out[3] = c.vxi1;
    state_out[4] = 0.5 * c.W * c.vep * c.vep + 0.5 * c.Q1 * c.vxi1 * c.vxi1 + (c.Nf + 1.0) * c.T * c.xi1 +
                   c.Pref * V;
  }
  free(s.invm); free(s.force); free(s.backup); free(s.rcut); free(s.image); free(s.nnb); free(s.list);
  return status;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
