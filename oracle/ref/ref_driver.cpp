// ORACLE build (test infrastructure only): extern "C" entry points that drive
// the md.error reference sources compiled where they lie under the reference
// tree (see oracle/ref/Makefile), so tests can compare our restatement with
// the reference's own code on the same inputs.
//   ref_spme_*: longRange.hetero/profile.test/template/tools/real.error
//               ElectrostaticInteraction (EleRecBSpline / EleRecFBSpline / EleRecES / EleDir)
//   ref_arc_*:  shortRange.inhomo/template/tools/simulation.hetero.cutoff
//               AdaptRCut + PressureCorrection (host code)
#include <cstring>
#include <iostream>
#include <sstream>
#include <vector>

#ifdef REF_SPME
#include "ElectrostaticInteraction.h"
#include "BoxGeometry.h"
#include "Particle.h"

extern "C" int ref_spme_forces(int n, const double* pos, const double* q, const double* box,
                               double beta, const int* K, double rcut, int method, int order,
                               double* dir_force, double* rec_force, double* energy,
                               double* err_dir, double* err_rec, double* err_interp) {
  TimeConstRectangularBoxGeometry bx(box[0], box[1], box[2]);
  std::vector<StandardParticle> parts(n);
  for (int i = 0; i < n; ++i) {
    StandardParticle& p = parts[i];
    for (int d = 0; d < 3; ++d) { p.r()[d] = pos[3 * i + d]; p.v()[d] = 0.; }
    p.mass() = 1.;
    p.id() = i;
    p.type() = 0;
    p.charge() = q[i];
    bx.moveParticleToBox(p);
  }
  std::vector<unsigned> KK(3);
  for (int d = 0; d < 3; ++d) KK[d] = (unsigned)K[d];
  InterpolationInfo::Method m = method == 0 ? InterpolationInfo::BSpline
                                : (method == 1 ? InterpolationInfo::FBSpline : InterpolationInfo::ES);
  ElectrostaticInteraction ele;
  ele.init(beta, KK, rcut, bx, m, (InterpolationInfo::Order)order);
  for (int i = 0; i < n; ++i) ele.registerParticle(parts[i]);
  ele.build();
  std::vector<double> zero3(3, 0.);
  std::vector<std::vector<double> > df(n, zero3), rf(n, zero3);
  // the exact Ewald sum prints a progress line per k-vector: silence std::cout
  std::ostringstream sink;
  std::streambuf* keep = std::cout.rdbuf(sink.rdbuf());
  double e = ele.applyInteractionCalPotential(df, rf);
  std::cout.rdbuf(keep);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) { dir_force[3 * i + d] = df[i][d]; rec_force[3 * i + d] = rf[i][d]; }
  *energy = e;
  if (err_dir && err_rec) ele.errorEstimatePME(*err_dir, *err_rec);
  if (err_interp && method == 0) ele.errorEstimateInterpolRec(*err_interp);
  return 0;
}

// SelfCorr::reinit + correction (app/spme.cpp:266-270): adds the self-force
// correction of analytic differentiation to force [n][3]
#include "SelfCorr.h"
extern "C" int ref_selfcorr(int n, const double* pos, const double* q, const double* box, double beta,
                            const int* K, int order, double* force) {
  std::vector<std::vector<double> > p(n, std::vector<double>(3)), f(n, std::vector<double>(3));
  std::vector<double> qq(q, q + n);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) { p[i][d] = pos[3 * i + d]; f[i][d] = force[3 * i + d]; }
  std::ostringstream sink;  // reinit prints progress on stdout
  std::streambuf* keep = std::cout.rdbuf(sink.rdbuf());
  SelfCorr sc;
  sc.reinit(beta, order, K[0], K[1], K[2], box[0], box[1], box[2]);
  std::cout.rdbuf(keep);
  sc.correction(p, qq, f);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) force[3 * i + d] = f[i][d];
  return 0;
}
#endif

#ifdef REF_ERRMAP
// ErrorEstimate_SPME_Ik::reinit + calError (analyze/app/error.spme.ik.cpp:82-85)
// on a density profile given on the grid K (profile1: charge-sign density,
// profile2: number density); error1 / error2 as [n][2] (real, imaginary).
// the profile class keeps its data private and fills it only from trajectory
// files: read its header with default-public members (same layout) so that
// the driver can set the profile directly
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>
#define class struct
#include "DensityProfile.h"
#undef class
#include "ErrorEstimate_SPME_Ik.h"
extern "C" int ref_spme_ik_errmap(const int* K, const double* box, double beta, int order, const double* rho1,
                                  const double* rho2, double charge, double* e1, double* e2) {
  DensityProfile_PiecewiseConst dp;
  dp.boxsize.assign(box, box + 3);
  dp.nx = K[0]; dp.ny = K[1]; dp.nz = K[2];
  dp.nele = K[0] * K[1] * K[2];
  dp.hx = box[0] / K[0]; dp.hy = box[1] / K[1]; dp.hz = box[2] / K[2];
  dp.profile1.assign(rho1, rho1 + dp.nele);
  dp.profile2.assign(rho2, rho2 + dp.nele);
  dp.profileP.assign(dp.nele, 0.);
  dp.profileN.assign(dp.nele, 0.);
  ErrorEstimate_SPME_Ik est;
  est.reinit(beta, order, dp);
  est.calError(dp, charge);
  for (unsigned i = 0; i < dp.nele; ++i) {
    e1[2 * i] = est.error1[i][0]; e1[2 * i + 1] = est.error1[i][1];
    e2[2 * i] = est.error2[i][0]; e2[2 * i + 1] = est.error2[i][1];
  }
  return 0;
}
#endif

#ifdef REF_ARC
#include "AdaptRCut.h"
#include "PressureCorrection.h"

// AdaptRCut on a given density profile: error[nrc*nele], rcut[nele], rcidx[nele]
extern "C" int ref_arc_run(const double* box, const int* nbin, double rcmin, double rcmax,
                           double rcstep, const double* profile, double prec, int nrefine,
                           double* error_out, double* rcut_out, int* rcidx_out,
                           double* rerr_out, double* pcorr_out) {
  DensityProfile_PiecewiseConst dp;
  dp.set(box, nbin, profile);
  AdaptRCut arc;
  arc.reinit(rcmin, rcmax, rcstep, dp);
  arc.calError(dp);
  arc.calRCut(prec);
  for (int i = 0; i < nrefine; ++i) arc.refineRCut();
  const int nele = nbin[0] * nbin[1] * nbin[2];
  int nrc = (int)arc.getRcList().size();
  // error / result_error are private members; this translation unit is built
  // with -Dprivate=public so the harness can read them
  if (error_out)
    for (int c = 0; c < nrc; ++c)
      for (int i = 0; i < nele; ++i) error_out[(size_t)c * nele + i] = arc.error[c][i][0];
  for (int i = 0; i < nele; ++i) {
    rcut_out[i] = arc.getRCut()[i];
    rcidx_out[i] = arc.getProfileIndex()[i];
  }
  if (rerr_out)
    for (int i = 0; i < nele; ++i) rerr_out[i] = arc.result_error[i];
  if (pcorr_out) {
    PressureCorrection pc(arc, dp);
    pc.correction(arc, dp);
    pcorr_out[0] = pc.pxx;
    pcorr_out[1] = pc.pyy;
    pcorr_out[2] = pc.pzz;
  }
  (void)nrc;
  return 0;
}
#endif

#ifdef REF_FCORR
#include "ForceCorr.h"

// ForceCorr::reinit(rc, dp) + calError(dp) on a given profile: the complex
// field error2r{x,y,z}, real parts re[3][nele], imaginary parts im[3][nele]
extern "C" int ref_fcorr_run(const double* box, const int* nbin, double rc, const double* profile, double* re,
                             double* im) {
  DensityProfile_PiecewiseConst dp;
  dp.set(box, nbin, profile);
  ForceCorr fc;
  fc.reinit(rc, dp);
  fc.calError(dp);
  const int nele = nbin[0] * nbin[1] * nbin[2];
  const fftw_complex* f[3] = {fc.getForceCorrX(), fc.getForceCorrY(), fc.getForceCorrZ()};
  for (int d = 0; d < 3; ++d)
    for (int i = 0; i < nele; ++i) {
      re[(size_t)d * nele + i] = f[d][i][0];
      im[(size_t)d * nele + i] = f[d][i][1];
    }
  return 0;
}
#endif

#ifdef REF_ERRDIR
// ErrorEstimate_dir::reinit + calError (analyze/app/error.dir.cpp) on a density
// profile given on the grid K; error1 / error2 as [n][2] (real, imaginary).
// The profile header is read with default-public members, as for the ik map.
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>
#define class struct
#include "DensityProfile.h"
#undef class
#include "ErrorEstimate_dir.h"
extern "C" int ref_dir_errmap(const int* K, const double* box, double beta, double rcut, const double* rho1,
                              const double* rho2, double charge, double* e1, double* e2) {
  DensityProfile_PiecewiseConst dp;
  dp.boxsize.assign(box, box + 3);
  dp.nx = K[0]; dp.ny = K[1]; dp.nz = K[2];
  dp.nele = K[0] * K[1] * K[2];
  dp.hx = box[0] / K[0]; dp.hy = box[1] / K[1]; dp.hz = box[2] / K[2];
  dp.profile1.assign(rho1, rho1 + dp.nele);
  dp.profile2.assign(rho2, rho2 + dp.nele);
  dp.profileP.assign(dp.nele, 0.);
  dp.profileN.assign(dp.nele, 0.);
  ErrorEstimate_dir est;
  est.reinit(beta, rcut, dp);
  est.calError(dp, charge);
  for (unsigned i = 0; i < dp.nele; ++i) {
    e1[2 * i] = est.error1[i][0]; e1[2 * i + 1] = est.error1[i][1];
    e2[2 * i] = est.error2[i][0]; e2[2 * i + 1] = est.error2[i][1];
  }
  return 0;
}
#endif

#ifdef REF_ERRANA
// ErrorEstimate_SPME_Ana::reinit + calError (analyze/app/error.spme.ana.cpp) on a
// density profile given on the grid K; error1 / error2 as [n][2] (real, imaginary),
// the uncharged self error, and (when fconv is not null) FConvRho1 of the four
// alias indices k = -2, -1, 1, 2 as [4][3][n][2].  The profile header is read with
// default-public members, as for the ik map.
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>
#define class struct
#include "DensityProfile.h"
#undef class
#include "ErrorEstimate_SPME_Ana.h"
extern "C" int ref_spme_ana_errmap(const int* K, const double* box, double beta, int order, const double* rho1,
                                   const double* rho2, double charge, double* e1, double* e2, double* self_out,
                                   double* fconv) {
  DensityProfile_PiecewiseConst dp;
  dp.boxsize.assign(box, box + 3);
  dp.nx = K[0]; dp.ny = K[1]; dp.nz = K[2];
  dp.nele = K[0] * K[1] * K[2];
  dp.hx = box[0] / K[0]; dp.hy = box[1] / K[1]; dp.hz = box[2] / K[2];
  dp.profile1.assign(rho1, rho1 + dp.nele);
  dp.profile2.assign(rho2, rho2 + dp.nele);
  dp.profileP.assign(dp.nele, 0.);
  dp.profileN.assign(dp.nele, 0.);
  ErrorEstimate_SPME_Ana est;
  est.reinit(beta, order, dp);
  est.calError(dp, charge);
  const unsigned n = dp.nele;
  for (unsigned i = 0; i < n; ++i) {
    e1[2 * i] = est.error1[i][0]; e1[2 * i + 1] = est.error1[i][1];
    e2[2 * i] = est.error2[i][0]; e2[2 * i + 1] = est.error2[i][1];
  }
  *self_out = est.self_error;
  if (fconv) {
    // kcut (a default-private member) is global_half_N_k_sum = 2 of the source file
    const int kc = 2;
    int slot = 0;
    for (int k = -kc; k <= kc; ++k) {
      if (k == 0) continue;
      fftw_complex* src[3] = {est.FConvRho1x[k + kc], est.FConvRho1y[k + kc], est.FConvRho1z[k + kc]};
      for (int d = 0; d < 3; ++d)
        for (unsigned i = 0; i < n; ++i) {
          fconv[2 * (n * (3 * slot + d) + i)] = src[d][i][0];
          fconv[2 * (n * (3 * slot + d) + i) + 1] = src[d][i][1];
        }
      ++slot;
    }
  }
  return 0;
}
#endif

#ifdef REF_GRO
// GromacsFileManager::readGroFile / writeGroFile (ENG/src/GromacsFileManager.cpp)
// with the engine's ScalorType (float) arrays; names in StringSize (8) slots.
// Reading returns 0, or 1 when the reader threw (cannot open / wrong format).
#include "GromacsFileManager.h"
extern "C" int ref_gro_read(const char* path, int n, int* resd_index, char* resd_name, char* atom_name,
                            int* atom_index, float* pos, float* vel, float* box) {
  std::vector<IndexType> ri(n), ai(n);
  std::vector<ScalorType> x(n), y(n), z(n), u(n), v(n), w(n);
  try {
    GromacsFileManager::readGroFile(path, ri.data(), resd_name, atom_name, ai.data(), x.data(), y.data(), z.data(),
                                    u.data(), v.data(), w.data(), &box[0], &box[1], &box[2]);
  } catch (...) {
    return 1;
  }
  for (int i = 0; i < n; ++i) {
    resd_index[i] = (int)ri[i]; atom_index[i] = (int)ai[i];
    pos[3 * i] = x[i]; pos[3 * i + 1] = y[i]; pos[3 * i + 2] = z[i];
    vel[3 * i] = u[i]; vel[3 * i + 1] = v[i]; vel[3 * i + 2] = w[i];
  }
  return 0;
}
extern "C" int ref_gro_write(const char* path, const char* title, int n, const int* resd_index,
                             const char* resd_name, const char* atom_name, const int* atom_index, const float* pos,
                             const float* vel, const float* box) {
  FILE* fp = fopen(path, "w");
  if (!fp) return 1;
  fputs(title, fp);
  std::vector<IndexType> ri(resd_index, resd_index + n), ai(atom_index, atom_index + n);
  std::vector<ScalorType> x(n), y(n), z(n), u(n), v(n), w(n);
  for (int i = 0; i < n; ++i) {
    x[i] = pos[3 * i]; y[i] = pos[3 * i + 1]; z[i] = pos[3 * i + 2];
    u[i] = vel[3 * i]; v[i] = vel[3 * i + 1]; w[i] = vel[3 * i + 2];
  }
  GromacsFileManager::writeGroFile(fp, n, ri.data(), resd_name, atom_name, ai.data(), x.data(), y.data(), z.data(),
                                   u.data(), v.data(), w.data(), box[0], box[1], box[2]);
  fclose(fp);
  return 0;
}
#endif

#ifdef REF_BONDED
// The engine's bond and angle force functions (include/BondInteraction.h,
// include/AngleInteraction.h) evaluated on the host in binary32: one term for
// the given parameters (as the *Parameter classes take them) and difference
// vectors.  Bonds give the force on the reference atom; angles forcePoten01.
#include "BondInteraction.h"
#include "AngleInteraction.h"
extern "C" int ref_bonded_term(int ftype, const double* u, const double* d0, const double* d1, double* f0,
                               double* f1, double* e) {
  ScalorType p[3] = {0, 0, 0};
  ScalorType a0 = (ScalorType)d0[0], a1 = (ScalorType)d0[1], a2 = (ScalorType)d0[2];
  ScalorType b0 = (ScalorType)d1[0], b1 = (ScalorType)d1[1], b2 = (ScalorType)d1[2];
  ScalorType g0[3] = {0, 0, 0}, g1[3] = {0, 0, 0}, dp = 0;
  switch (ftype) {
    case mdForceHarmonicSpring: HarmonicSpring::initParameter(p, (ScalorType)u[0], (ScalorType)u[1]); break;
    case mdForceFENE: FENE::initParameter(p, (ScalorType)u[0], (ScalorType)u[1]); break;
    case mdForceFENE2: FENE2::initParameter(p, (ScalorType)u[0], (ScalorType)u[1], (ScalorType)u[2]); break;
    case mdForceAngleHarmonic: AngleHarmonic::initParameter(p, (ScalorType)u[0], (ScalorType)u[1]); break;
    case mdForceCosAngle0: CosAngle0::initParameter(p, (ScalorType)u[0]); break;
    default: return 1;
  }
  if (ftype < mdForceAngleHarmonic) {
    bondForcePoten((InteractionType)ftype, p, a0, a1, a2, &g0[0], &g0[1], &g0[2], &dp);
  } else {
    angleForcePoten(false, (InteractionType)ftype, p, a0, a1, a2, b0, b1, b2, &g0[0], &g0[1], &g0[2], &g1[0],
                    &g1[1], &g1[2], &dp);
  }
  for (int k = 0; k < 3; ++k) { f0[k] = g0[k]; f1[k] = g1[k]; }
  *e = dp;
  return 0;
}
#endif

#ifdef REF_NB
// The engine's non-bonded pair functions (include/NonBondedInteraction.h,
// nbForcePoten dispatch) evaluated on the host in binary32 for one pair:
// kind 1 LennardJones6_12 (eps, sigma, shift, rcut), 5 LennardJones6_12B
// (eps, sigma, shift, rcut), 3 CosTail (eps, b, wc), 2 / 6 the capped LJ forms
// (eps, sigma, shift, rcut, cap), 4 CosTail_cap (eps, b, wc, cap).
#include "NonBondedInteraction.h"
extern "C" int ref_nb_pair(int kind, const double* u, const double* d, double* f, double* e) {
  ScalorType p[16] = {0};
  switch (kind) {
    case mdForceLennardJones6_12:
      LennardJones6_12::initParameter(p, (ScalorType)u[0], (ScalorType)u[1], (ScalorType)u[2], (ScalorType)u[3]);
      break;
    case mdForceLennardJones6_12B:
      LennardJones6_12B::initParameter(p, (ScalorType)u[0], (ScalorType)u[1], (ScalorType)u[2], (ScalorType)u[3]);
      break;
    case mdForceCosTail:
      CosTail::initParameter(p, (ScalorType)u[0], (ScalorType)u[1], (ScalorType)u[2]);
      break;
    case mdForceLennardJones6_12_cap:
      LennardJones6_12_cap::initParameter(p, (ScalorType)u[0], (ScalorType)u[1], (ScalorType)u[2],
                                          (ScalorType)u[3], (ScalorType)u[4]);
      break;
    case mdForceLennardJones6_12B_cap:
      LennardJones6_12B_cap::initParameter(p, (ScalorType)u[0], (ScalorType)u[1], (ScalorType)u[2],
                                           (ScalorType)u[3], (ScalorType)u[4]);
      break;
    case mdForceCosTail_cap:
      CosTail_cap::initParameter(p, (ScalorType)u[0], (ScalorType)u[1], (ScalorType)u[2], (ScalorType)u[3]);
      break;
    default: return 1;
  }
  ScalorType fx = 0, fy = 0, fz = 0, dp = 0;
  nbForcePoten((InteractionType)kind, p, (ScalorType)d[0], (ScalorType)d[1], (ScalorType)d[2], &fx, &fy, &fz, &dp);
  f[0] = fx; f[1] = fy; f[2] = fz;
  *e = dp;
  return 0;
}
#endif
