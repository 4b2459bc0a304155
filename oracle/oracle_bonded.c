/* ORACLE -- test infrastructure only.  CPU restatement of the reference
 * engine's bonded terms (shortRange.inhomo/template/tools/simulation.hetero.cutoff):
 *   bonds   HarmonicSpring / FENE / FENE2        include/BondInteraction.h:217-372
 *   angles  AngleHarmonic / CosAngle0 (forcePoten01)  include/AngleInteraction.h:365-1216
 *   per-atom gather kernels calBondInteraction / calAngleInteraction
 *           (src/InteractionEngine_interface.cu:1399-1775): each atom sums the
 *           forces of its own bonds and angles; energies are shared 1/2 (bond)
 *           and 1/3 (angle); bond virial 1/2 f.d, angle virial on the centre
 *           atom only: -(f0 d0 - f1 d1)
 *   angle neighbour order (src/SystemBondedInteraction.cu:204-219): edge0 sees
 *           (centre, edge1), the centre (edge0, edge1), edge1 (centre, edge0)
 * Each formula keeps the reference's operation order.  prec 0 evaluates in
 * binary32 (the reference's ScalorType), prec 1 in binary64.  The energies use
 * the accurate logarithm. */
#include <math.h>
#include <string.h>

enum { T_HARM = 10000, T_FENE = 10001, T_FENE2 = 10002, T_ANG = 20000, T_COS0 = 20001 };

/* ---------------------------------------------------------- binary32 */
static void param_f(int type, const double* u, float* p) {
  p[0] = p[1] = p[2] = 0.f;
  if (type == T_HARM) { p[0] = (float)u[0]; p[1] = (float)u[1]; }
  else if (type == T_FENE) { float r = (float)u[1]; p[0] = (float)u[0]; p[1] = r * r; }
  else if (type == T_FENE2) { float rs = (float)u[1]; p[0] = (float)u[0]; p[1] = rs * rs; p[2] = (float)u[2]; }
  else if (type == T_ANG) { p[0] = (float)u[0]; p[1] = 3.14159265f - (float)u[1]; }
  else if (type == T_COS0) { p[0] = (float)u[0]; }
}

static float bond_f(int type, const float* p, float dx, float dy, float dz, float* f) {
  if (type == T_HARM) {
    float dr = dx * dx + dy * dy + dz * dz;
    float dri = (float)(1. / (double)sqrtf(dr));
    dr *= dri;
    float s = p[0] * (1.f - p[1] * dri);
    f[0] = dx * s; f[1] = dy * s; f[2] = dz * s;
    return 0.5f * p[0] * (dr - p[1]) * (dr - p[1]);
  }
  if (type == T_FENE) {
    float dr2 = dx * dx + dy * dy + dz * dz;
    float core = p[1] / (p[1] - dr2);
    float s = core * p[0];
    f[0] = dx * s; f[1] = dy * s; f[2] = dz * s;
    float t = 1.f / core;
    return t <= 0.f ? 1e10f : -0.5f * p[0] * p[1] * logf(t);
  }
  /* FENE2 */
  float dr = sqrtf(dx * dx + dy * dy + dz * dz);
  float rr = dr - p[2];
  float core = p[1] - rr * rr;
  float s = p[0] * p[1] * rr / (core * dr);
  f[0] = dx * s; f[1] = dy * s; f[2] = dz * s;
  float t = core / p[1];
  return t <= 0.f ? 1e10f : -0.5f * p[0] * p[1] * logf(t);
}

static float angle_f(int type, const float* p, const float* a, const float* b, float* f0, float* f1) {
  float c00 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  float c01 = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  float c11 = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
  float i0 = 1.f / sqrtf(c00), i1 = 1.f / sqrtf(c11);
  if (type == T_COS0) {
    float t = i0 * i1, cs = c01 * t, s = p[0] * t;
    for (int d = 0; d < 3; ++d) {
      f0[d] = s * (b[d] - c01 * i0 * i0 * a[d]);
      f1[d] = s * (-a[d] + c01 * i1 * i1 * b[d]);
    }
    return p[0] * (1.f - cs);
  }
  float e[3], g[3];
  for (int d = 0; d < 3; ++d) {
    e[d] = b[d] - c01 * i0 * i0 * a[d];
    g[d] = a[d] - c01 * i1 * i1 * b[d];
  }
  float ct = c01 * i1 * i0;
  if (ct > 1.f) ct = 1.f;
  float th = acosf(ct);
  float s = 2 * p[0] * (th - p[1]);
  for (int d = 0; d < 3; ++d) { e[d] *= 1e6f; g[d] *= 1e6f; }
  float t0 = sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
  float t1 = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  float s0 = i0 * s, s1 = i1 * s;
  f0[0] = f0[1] = f0[2] = 0.f;
  f1[0] = f1[1] = f1[2] = 0.f;
  if (t0 != 0) { s0 *= (1.f / t0); for (int d = 0; d < 3; ++d) f0[d] += s0 * e[d]; }
  else f0[0] += s0;
  if (t1 != 0) { s1 *= (1.f / t1); for (int d = 0; d < 3; ++d) f1[d] -= s1 * g[d]; }
  else f1[0] -= s1;
  return p[0] * (th - p[1]) * (th - p[1]);
}

/* ---------------------------------------------------------- binary64 */
static void param_d(int type, const double* u, double* p) {
  p[0] = p[1] = p[2] = 0.;
  if (type == T_HARM) { p[0] = u[0]; p[1] = u[1]; }
  else if (type == T_FENE) { p[0] = u[0]; p[1] = u[1] * u[1]; }
  else if (type == T_FENE2) { p[0] = u[0]; p[1] = u[1] * u[1]; p[2] = u[2]; }
  else if (type == T_ANG) { p[0] = u[0]; p[1] = M_PI - u[1]; }
  else if (type == T_COS0) { p[0] = u[0]; }
}

static double bond_d(int type, const double* p, double dx, double dy, double dz, double* f) {
  if (type == T_HARM) {
    double dr = dx * dx + dy * dy + dz * dz;
    double dri = 1. / sqrt(dr);
    dr *= dri;
    double s = p[0] * (1. - p[1] * dri);
    f[0] = dx * s; f[1] = dy * s; f[2] = dz * s;
    return 0.5 * p[0] * (dr - p[1]) * (dr - p[1]);
  }
  if (type == T_FENE) {
    double dr2 = dx * dx + dy * dy + dz * dz;
    double core = p[1] / (p[1] - dr2);
    double s = core * p[0];
    f[0] = dx * s; f[1] = dy * s; f[2] = dz * s;
    double t = 1. / core;
    return t <= 0. ? 1e10 : -0.5 * p[0] * p[1] * log(t);
  }
  double dr = sqrt(dx * dx + dy * dy + dz * dz);
  double rr = dr - p[2];
  double core = p[1] - rr * rr;
  double s = p[0] * p[1] * rr / (core * dr);
  f[0] = dx * s; f[1] = dy * s; f[2] = dz * s;
  double t = core / p[1];
  return t <= 0. ? 1e10 : -0.5 * p[0] * p[1] * log(t);
}

static double angle_d(int type, const double* p, const double* a, const double* b, double* f0, double* f1) {
  double c00 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  double c01 = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  double c11 = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
  double i0 = 1. / sqrt(c00), i1 = 1. / sqrt(c11);
  if (type == T_COS0) {
    double t = i0 * i1, cs = c01 * t, s = p[0] * t;
    for (int d = 0; d < 3; ++d) {
      f0[d] = s * (b[d] - c01 * i0 * i0 * a[d]);
      f1[d] = s * (-a[d] + c01 * i1 * i1 * b[d]);
    }
    return p[0] * (1. - cs);
  }
  double e[3], g[3];
  for (int d = 0; d < 3; ++d) {
    e[d] = b[d] - c01 * i0 * i0 * a[d];
    g[d] = a[d] - c01 * i1 * i1 * b[d];
  }
  double ct = c01 * i1 * i0;
  if (ct > 1.) ct = 1.;
  double th = acos(ct);
  double s = 2 * p[0] * (th - p[1]);
  for (int d = 0; d < 3; ++d) { e[d] *= 1e6; g[d] *= 1e6; }
  double t0 = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
  double t1 = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  double s0 = i0 * s, s1 = i1 * s;
  f0[0] = f0[1] = f0[2] = 0.;
  f1[0] = f1[1] = f1[2] = 0.;
  if (t0 != 0) { s0 *= (1. / t0); for (int d = 0; d < 3; ++d) f0[d] += s0 * e[d]; }
  else f0[0] += s0;
  if (t1 != 0) { s1 *= (1. / t1); for (int d = 0; d < 3; ++d) f1[d] -= s1 * g[d]; }
  else f1[0] -= s1;
  return p[0] * (th - p[1]) * (th - p[1]);
}

/* one bond term on the reference atom, d = r_partner - r_ref: force and energy */
void orc_bond_term(int type, const double* uparam, int prec, const double* d, double* f, double* e) {
  if (prec == 0) {
    float p[3], ff[3];
    param_f(type, uparam, p);
    *e = bond_f(type, p, (float)d[0], (float)d[1], (float)d[2], ff);
    for (int k = 0; k < 3; ++k) f[k] = ff[k];
  } else {
    double p[3];
    param_d(type, uparam, p);
    *e = bond_d(type, p, d[0], d[1], d[2], f);
  }
}

/* forcePoten01 of an angle term for the difference vectors d0, d1 */
void orc_angle_term(int type, const double* uparam, int prec, const double* d0, const double* d1, double* f0,
                    double* f1, double* e) {
  if (prec == 0) {
    float p[3], a[3], b[3], g0[3], g1[3];
    param_f(type, uparam, p);
    for (int k = 0; k < 3; ++k) { a[k] = (float)d0[k]; b[k] = (float)d1[k]; }
    *e = angle_f(type, p, a, b, g0, g1);
    for (int k = 0; k < 3; ++k) { f0[k] = g0[k]; f1[k] = g1[k]; }
  } else {
    double p[3];
    param_d(type, uparam, p);
    *e = angle_d(type, p, d0, d1, f0, f1);
  }
}

static double img_d(double x, double L) { return x - floor(x * (1. / L) + 0.5) * L; }
static float img_f(float x, float L, float Li) { return x - floorf(x * Li + 0.5f) * L; }

/* The per-atom gather over a whole configuration.  bonds [nb][2] with type,
 * user parameters [nb][3]; angles [na][3] (edge0, centre, edge1) with type,
 * parameters [na][3].  force [n][3] receives the bonded force (original
 * order); stats = {energy, virial xx, yy, zz}.  Each atom visits its bonds in
 * the order given, then its angles in the order given. */
void orc_bonded_apply(int n, const double* pos, const double* box, int prec, int nb, const int* bonds,
                      const int* btype, const double* bparam, int na, const int* angles, const int* atype,
                      const double* aparam, double* force, double* stats) {
  memset(force, 0, sizeof(double) * 3 * n);
  memset(stats, 0, sizeof(double) * 4);
  const float Lf[3] = {(float)box[0], (float)box[1], (float)box[2]};
  const float Lif[3] = {1.f / Lf[0], 1.f / Lf[1], 1.f / Lf[2]};
  for (int i = 0; i < n; ++i) {
    double F[3] = {0, 0, 0}, E = 0, V[3] = {0, 0, 0};
    float Ff[3] = {0, 0, 0};
    for (int b = 0; b < nb; ++b) {
      int j;
      if (bonds[2 * b] == i) j = bonds[2 * b + 1];
      else if (bonds[2 * b + 1] == i) j = bonds[2 * b];
      else continue;
      double d[3], f[3], e;
      for (int k = 0; k < 3; ++k) {
        if (prec == 0) d[k] = img_f((float)pos[3 * j + k] - (float)pos[3 * i + k], Lf[k], Lif[k]);
        else d[k] = img_d(pos[3 * j + k] - pos[3 * i + k], box[k]);
      }
      orc_bond_term(btype[b], bparam + 3 * b, prec, d, f, &e);
      for (int k = 0; k < 3; ++k) {
        if (prec == 0) Ff[k] += (float)f[k]; else F[k] += f[k];
        V[k] += 0.5 * f[k] * d[k];
      }
      E += 0.5 * e;
    }
    for (int a = 0; a < na; ++a) {
      const int e0 = angles[3 * a], c = angles[3 * a + 1], e1 = angles[3 * a + 2];
      int posi, t0, t1;
      if (i == e0) { posi = 0; t0 = c; t1 = e1; }
      else if (i == c) { posi = 1; t0 = e0; t1 = e1; }
      else if (i == e1) { posi = 2; t0 = c; t1 = e0; }
      else continue;
      double d0[3], d1[3], f0[3], f1[3], e;
      for (int k = 0; k < 3; ++k) {
        double x0, x1;
        if (prec == 0) {
          float r = (float)pos[3 * i + k], p0 = (float)pos[3 * t0 + k], p1 = (float)pos[3 * t1 + k];
          x0 = posi == 1 ? img_f(r - p0, Lf[k], Lif[k]) : img_f(p0 - r, Lf[k], Lif[k]);
          x1 = posi == 1 ? img_f(p1 - r, Lf[k], Lif[k]) : img_f(p1 - p0, Lf[k], Lif[k]);
        } else {
          const double r = pos[3 * i + k], p0 = pos[3 * t0 + k], p1 = pos[3 * t1 + k];
          x0 = posi == 1 ? img_d(r - p0, box[k]) : img_d(p0 - r, box[k]);
          x1 = posi == 1 ? img_d(p1 - r, box[k]) : img_d(p1 - p0, box[k]);
        }
        d0[k] = x0; d1[k] = x1;
      }
      orc_angle_term(atype[a], aparam + 3 * a, prec, d0, d1, f0, f1, &e);
      for (int k = 0; k < 3; ++k) {
        const double fk = posi == 1 ? f0[k] + f1[k] : -f0[k];
        if (prec == 0) Ff[k] += (float)fk; else F[k] += fk;
        if (posi == 1) V[k] -= f0[k] * d0[k] - f1[k] * d1[k];
      }
      E += e / 3.;
    }
    for (int k = 0; k < 3; ++k) force[3 * i + k] = prec == 0 ? (double)Ff[k] : F[k];
    stats[0] += E;
    for (int k = 0; k < 3; ++k) stats[1 + k] += V[k];
  }
}
