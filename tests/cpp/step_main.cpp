// C++ caller of the reference-shaped facade: loads a bunch, solves its
// initial fields, runs the reference's main-loop body through TETMSolver / moveMesh, and prints the
// beam centroid.  Built by tests/test_cpp_facade.py.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "csrst/csrst.hpp"

int main(int argc, char **argv) {
  const int steps = argc > 1 ? std::atoi(argv[1]) : 4;
  // 512 x 104 mesh at 20 um, 2 mm pipe, R = 0.25 m, gamma = 1000, TSC
  csrst_config cfg{};
  cfg.Nx = 512; cfg.Ny = 104; cfg.shape_order = 1;
  cfg.length_before = 0.0055976313069747725; cfg.length_after = 0.001; cfg.width = 0.002;
  cfg.phi_deg = 0.8223645856699741; cfg.ekin_mev = 510.489; cfg.bz = 6.8180466968243225;
  cfg.dt = 0.5 * 20e-6 / 299792458.0; cfg.charge_mass = -1e-9 / 0.51099906e-03;
  try {
    csrst::Simulation sim(cfg);
    const size_t n = 4000;
    std::mt19937_64 g(3);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<double> x(n), y(n), px(n), py(n, 0.0), q(n, -1e-9 / n);
    for (size_t i = 0; i < n; ++i) {
      x[i] = 40 * 20e-6 + 6 * 60e-6 + 60e-6 * nd(g);
      y[i] = 1e-3 + 40e-6 * nd(g);
      const double gam = 1000.0 * (1 + 1e-4 * nd(g));
      px[i] = std::sqrt(gam * gam - 1);
    }
    sim.loadBunch(x, y, px, py, q);
    csrst::PoissonSolver poisson(sim);  // initial fields, as main.cpp:232-248
    poisson.computeField();
    std::printf("poisson gamma %.6f iterations %g %g %g\n", poisson.report()[0], poisson.report()[1],
                poisson.report()[3], poisson.report()[5]);
    csrst::TETMSolver solver(sim);
    csrst::PartBunch bunch(sim);
    for (int s = 0; s < steps; ++s) {
      solver.updateField_firstStep();
      solver.updateField_secondStep();
      csrst::moveMesh(sim);
    }
    csrst::PartBunchState st;
    bunch.calcBeamParameters(st);
    std::printf("rmean %.12e %.12e Ekin %.9f\n", st.rmean[0], st.rmean[1], st.Ekin);
  } catch (const csrst::Error &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
