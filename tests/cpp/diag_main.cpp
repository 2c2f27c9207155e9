// Writes the statistics, line-field and VTK files of include/csrst/diagnostics.hpp
// from fixed host arrays (no GPU) into the directory argv[1], for comparison
// with the Python writers on the same values.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "csrst/diagnostics.hpp"

static double val(int k, int salt) { return (double)((k * 37 + salt * 11) % 101 - 50) * 1.25e-3; }

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  // statistics: two rows from fixed moments and field-energy sums
  std::FILE *f = std::fopen((dir + "/stats.stat").c_str(), "w");
  csrst::format::sdds_header(f, 1, "csrst_b200");
  csrst::format::EnergyAverage avg{3.5};
  const double ee[2] = {4.25, 5.0}, hh[2] = {0.5, 0.75}, t[2] = {1e-12, 2e-12};
  for (int r = 0; r < 2; ++r) {
    double m[18];
    for (int k = 0; k < 18; ++k) m[k] = val(k, r);
    csrst::format::sdds_row(f, csrst::format::stat_row(t[r], m, avg(ee[r], hh[r])));
  }
  std::fclose(f);
  // one line-field file of 5 samples
  std::vector<double> rows(35);
  for (int k = 0; k < 35; ++k) rows[k] = val(k, 3) * (k % 3 == 0 ? 1e6 : 1.0);
  csrst::format::field_on_line(dir + "/FieldOnLine_0000.dat", rows.data(), 5);
  // VTK: a 12 x 8 static mesh with a 4 x 3 window at (3, 2), two steps, then the window series
  const int Nx = 12, Ny = 8, L0 = 4, L1 = 3;
  std::vector<double> st[4];
  for (int k = 0; k < 4; ++k) st[k].resize(Nx * Ny);
  for (int n = 0; n < Nx * Ny; ++n) {
    st[0][n] = n; st[1][n] = n + 1000.0; st[2][n] = 2.0 * n; st[3][n] = 3.0 * n;
  }
  std::vector<double> wp[6];
  for (int k = 0; k < 6; ++k) {
    wp[k].assign(L0 * L1, 10000.0 * (k + 1));
    wp[k][1 * L0 + 1] += 1.0;
  }
  const double *stat[4] = {st[0].data(), st[1].data(), st[2].data(), st[3].data()};
  const double *win[6] = {wp[0].data(), wp[1].data(), wp[2].data(), wp[3].data(), wp[4].data(), wp[5].data()};
  csrst::format::PlotFields p;
  p.nx = Nx; p.ny = Ny; p.hx = 0.5; p.hy = 0.25; p.ox = -1.0; p.oy = 2.0;
  csrst::format::overlay(p, stat, win, 3, 2, L0, L1, true);
  std::vector<double> times;
  for (double tt : {1e-12, 2e-12}) {
    csrst::format::vtk_step(dir, "c", (int)times.size(), p);
    times.push_back(tt);
    csrst::format::vtk_collection(dir, "c", times);
  }
  csrst::format::PlotFields w;
  w.nx = L0; w.ny = L1; w.hx = 0.5; w.hy = 0.25; w.ox = 0.5; w.oy = 2.5;
  w.ex = wp[0]; w.ey = wp[1]; w.jx = wp[4]; w.jy = wp[5];
  w.hz.resize(L0 * L1);
  for (int n = 0; n < L0 * L1; ++n) w.hz[n] = wp[2][n] + wp[3][n];
  csrst::format::vtk_step(dir, "mm", 0, w);
  csrst::format::vtk_collection(dir, "mm", {0.0});
  // energy change: Kahan sums of three sample sets (NaN where off the window)
  std::vector<long double> sum(8, 0.0L), corr(8, 0.0L);
  for (int k = 0; k < 3; ++k) {
    double e[8];
    for (int i = 0; i < 8; ++i) e[i] = (double)((k * 7 + i * 13) % 17 - 8) * 1.5e4;
    e[0] = std::nan("");
    if (k % 2) e[7] = std::nan("");
    csrst::format::kahan_add(sum, corr, e);
  }
  csrst::format::energy_change_file(dir + "/energyChange.dat", 0.5e-3, 0.25e-3, 0.75e-3, 5e-12, sum);
  const std::vector<double> back = csrst::format::read_vtk_collection(dir, "c");
  std::printf("collection %zu %g %g\n", back.size(), back.size() > 1 ? back[1] : -1.0, back.empty() ? -1.0 : back[0]);
  return 0;
}
