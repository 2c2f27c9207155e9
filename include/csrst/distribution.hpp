// Distribution (src/Distribution.cpp:55-163): the bunch the reference builds
// from its command line (Np, mean_Rx, mean_Ry, sigma_x, Ekin, sigma_p,
// Qtotal; defaults in src/main.cpp:126-133), as host arrays for
// csrst::Simulation::loadBunch.  Point k = 1 .. n of the 2D Halton sequence
// (bases 2 and 3, the published construction; GSL's gsl_qrng_halton is not
// used) becomes a round Gaussian sample by Box-Muller, sigma sqrt(-2 ln v0)
// (cos, sin)(2 pi v1).  Positions and momentum offsets come from two
// generators of the same sequence, so they are proportional point by point;
// momenta are (sqrt(gamma^2 - 1), 0) + offset with gamma = Ekin / m_e + 1;
// charges -Qtotal 1e-9 / n each.  Then the positions alone are sorted by
// truncated mesh row and x (Utils::XFirst, src/utils.hh:116-142), which, as
// in the reference, unpairs them from the momenta.  Same arithmetic as
// csrst_b200.workloads.halton_bunch.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

namespace csrst {

struct HostBunch {
  std::vector<double> x, y, px, py, q;
};

// Van der Corput radical inverse of n in `base`: digits mirrored about the
// point, accumulated most significant first.
inline double radical_inverse(unsigned long long n, unsigned base) {
  double r = 0.0, v = 1.0;
  while (n > 0) {
    v /= base;
    r += v * (double)(n % base);
    n /= base;
  }
  return r;
}

struct DistributionParams {
  size_t n = 50000;            // Np
  double mean_rx = 0.05;       // mean_Rx [m]
  double mean_ry = 0.0;        // mean_Ry [m]
  double sigma_x = 0.01;       // sigma_x [m]
  double ekin_mev = 250.0;     // Ekin [MeV]
  double sigma_p = 1.0;        // sigma_p [beta gamma]
  double qtotal_nc = -1.0;     // Qtotal [nC]
  double origin[2] = {0.0, 0.0}, spacing[2] = {1.0, 1.0};  // static mesh (for the row sort)
};

inline HostBunch halton_bunch(const DistributionParams &p) {
  constexpr double kMassMeV = 0.51099906e-03 * 1e3;  // Distribution.cpp:26 (Physics::m_e * 1e3)
  constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
  const size_t n = p.n;
  std::vector<double> x(n), y(n), c(n), s(n), r(n);
  HostBunch b;
  b.px.resize(n); b.py.resize(n);
  const double gamma = p.ekin_mev / kMassMeV + 1.0, mean_p = std::sqrt(gamma * gamma - 1.0);
  for (size_t i = 0; i < n; ++i) {
    const unsigned long long k = i + 1;
    const double v0 = radical_inverse(k, 2), v1 = radical_inverse(k, 3);
    r[i] = std::sqrt(-2.0 * std::log(v0));
    const double a = kTwoPi * v1;
    c[i] = std::cos(a);
    s[i] = std::sin(a);
    x[i] = p.mean_rx + p.sigma_x * r[i] * c[i];
    y[i] = p.mean_ry + p.sigma_x * r[i] * s[i];
    b.px[i] = mean_p + p.sigma_p * r[i] * c[i];
    b.py[i] = p.sigma_p * r[i] * s[i];
  }
  std::vector<long long> row(n);
  for (size_t i = 0; i < n; ++i) row[i] = (long long)std::trunc((y[i] - p.origin[1]) / p.spacing[1]);
  std::vector<size_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b2) {
    return row[a] != row[b2] ? row[a] < row[b2] : x[a] < x[b2];
  });
  b.x.resize(n); b.y.resize(n);
  for (size_t i = 0; i < n; ++i) { b.x[i] = x[order[i]]; b.y[i] = y[order[i]]; }
  b.q.assign(n, -p.qtotal_nc * 1e-9 / (double)n);
  return b;
}

}  // namespace csrst
