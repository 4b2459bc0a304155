// Seeded synthetic configurations for the benchmark and test systems
// (host code; no GPU needed).  The reference builds its inputs with small
// generators (shortRange.inhomo/template/tools/gen.conf.tube/app/gen.liquid.cpp);
// these produce the lattice, random-sequential-addition liquid/vapour slab,
// Maxwell velocities and +-1 charges of the benchmark systems.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>
#include "../../include/mdforce.h"

void md_set_error(const char* fmt, ...);

extern "C" int md_synth_fcc(int nx, int ny, int nz, const double box[3], double jitter,
                            uint64_t seed, double* pos) {
  if (nx < 1 || ny < 1 || nz < 1 || !box || !pos || jitter < 0) return MD_ERR_BADARG;
  const double b[4][3] = {{0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5}};
  const double a[3] = {box[0] / nx, box[1] / ny, box[2] / nz};
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> u(-jitter, jitter);
  long long k = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int l = 0; l < nz; ++l)
        for (int s = 0; s < 4; ++s) {
          double c[3] = {(i + b[s][0]) * a[0], (j + b[s][1]) * a[1], (l + b[s][2]) * a[2]};
          for (int d = 0; d < 3; ++d) {
            double x = c[d] + u(rng);
            x -= std::floor(x / box[d]) * box[d];
            pos[3 * k + d] = x;
          }
          ++k;
        }
  return MD_OK;
}

namespace {
struct Grid {
  double h[3];
  int n[3];
  std::vector<std::vector<int>> cells;
  Grid(const double box[3], double cell) {
    for (int d = 0; d < 3; ++d) {
      n[d] = std::max(1, (int)std::floor(box[d] / cell));
      h[d] = box[d] / n[d];
    }
    cells.resize((size_t)n[0] * n[1] * n[2]);
  }
  int index(const double x[3], int c[3]) const {
    for (int d = 0; d < 3; ++d) {
      c[d] = (int)(x[d] / h[d]);
      if (c[d] >= n[d]) c[d] = n[d] - 1;
      if (c[d] < 0) c[d] = 0;
    }
    return c[2] + n[2] * (c[1] + n[1] * c[0]);
  }
};
}  // namespace

// Random sequential addition: atoms are drawn uniformly inside the slab
// |x_axis - center| < half_width (n_in of them) and then in the rest of the box
// (n - n_in), each accepted only if it is >= min_sep from every atom placed.
extern "C" int md_synth_slab(int n, int n_in, const double box[3], int axis, double center,
                             double half_width, double min_sep, uint64_t seed, double* pos) {
  if (n < 1 || n_in < 0 || n_in > n || !box || !pos || axis < 0 || axis > 2 || min_sep < 0) {
    md_set_error("md_synth_slab: bad arguments");
    return MD_ERR_BADARG;
  }
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> u01(0.0, 1.0);
  Grid g(box, std::max(min_sep, 1e-3));
  const double ms2 = min_sep * min_sep;
  const long long max_tries = 2000LL * n + 1000000LL;
  long long tries = 0;
  const double lo = center - half_width, width = 2 * half_width;
  for (int k = 0; k < n; ++k) {
    const bool inside = k < n_in;
    for (;;) {
      if (++tries > max_tries) {
        md_set_error("md_synth_slab: could not place atom %d (density too high for min_sep)", k);
        return MD_ERR_BADARG;
      }
      double x[3];
      for (int d = 0; d < 3; ++d) x[d] = u01(rng) * box[d];
      if (inside) {
        double z = lo + u01(rng) * width;
        z -= std::floor(z / box[axis]) * box[axis];
        x[axis] = z;
      } else {
        double z = x[axis];
        double dz = z - center;
        dz -= std::round(dz / box[axis]) * box[axis];
        if (std::fabs(dz) < half_width) continue;
      }
      int c[3];
      int ci = g.index(x, c);
      (void)ci;
      bool ok = true;
      for (int a = -1; a <= 1 && ok; ++a)
        for (int b = -1; b <= 1 && ok; ++b)
          for (int e = -1; e <= 1 && ok; ++e) {
            int cc[3] = {(c[0] + a + g.n[0]) % g.n[0], (c[1] + b + g.n[1]) % g.n[1], (c[2] + e + g.n[2]) % g.n[2]};
            const auto& cell = g.cells[cc[2] + g.n[2] * (cc[1] + (size_t)g.n[1] * cc[0])];
            for (int j : cell) {
              double r2 = 0;
              for (int d = 0; d < 3; ++d) {
                double dd = pos[3 * j + d] - x[d];
                dd -= std::round(dd / box[d]) * box[d];
                r2 += dd * dd;
              }
              if (r2 < ms2) { ok = false; break; }
            }
          }
      if (!ok) continue;
      for (int d = 0; d < 3; ++d) pos[3 * k + d] = x[d];
      g.cells[g.index(x, c)].push_back(k);
      break;
    }
  }
  return MD_OK;
}

extern "C" int md_synth_maxwell(int n, const double* mass, double temperature, uint64_t seed,
                                double* vel) {
  if (n < 1 || !vel || temperature < 0) return MD_ERR_BADARG;
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> g(0.0, 1.0);
  double p[3] = {0, 0, 0}, mt = 0;
  for (int i = 0; i < n; ++i) {
    double m = mass ? mass[i] : 1.0;
    double s = std::sqrt(temperature / m);
    for (int d = 0; d < 3; ++d) {
      vel[3 * i + d] = s * g(rng);
      p[d] += m * vel[3 * i + d];
    }
    mt += m;
  }
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) vel[3 * i + d] -= p[d] / mt;  // remove centre-of-mass motion
  return MD_OK;
}

extern "C" int md_synth_charges(int n, uint64_t seed, double* q) {
  if (n < 2 || !q) return MD_ERR_BADARG;
  for (int i = 0; i < n; ++i) q[i] = (i < n / 2) ? 1.0 : -1.0;
  std::mt19937_64 rng(seed);
  std::shuffle(q, q + n, rng);
  return MD_OK;
}
