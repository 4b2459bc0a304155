/* ORACLE build shim (test infrastructure only), force-included (-include) when
 * compiling the reference's host-side AdaptRCut / PressureCorrection /
 * Integral1D sources.  It pre-defines the include guard of the engine's
 * DensityProfile.h (which pulls in CUDA and xdrfile headers) and supplies a
 * minimal profile holder with the accessors those sources call. */
#ifndef ORACLE_ENG_PRELUDE_H
#define ORACLE_ENG_PRELUDE_H
#define __DensityProfile_h_wanghan__
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>
class DensityProfile_PiecewiseConst {
  std::vector<double> boxsize;
  unsigned nx, ny, nz;
  std::vector<double> profile;
 public:
  DensityProfile_PiecewiseConst() : nx(0), ny(0), nz(0) {}
  void set(const double* box, const int* n, const double* prof) {
    boxsize.assign(box, box + 3);
    nx = n[0]; ny = n[1]; nz = n[2];
    profile.assign(prof, prof + (size_t)nx * ny * nz);
  }
  const double& getProfile(const unsigned& ix, const unsigned& iy, const unsigned& iz) const {
    return profile[iz + nz * (iy + ny * ix)];
  }
  const double& getProfile(const unsigned& i) const { return profile[i]; }
  const unsigned& getNx() const { return nx; }
  const unsigned& getNy() const { return ny; }
  const unsigned& getNz() const { return nz; }
  const std::vector<double>& getBox() const { return boxsize; }
};
#endif
