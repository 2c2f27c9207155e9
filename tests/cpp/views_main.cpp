// A caller written against the reference's argument lists (main.cpp:232-506):
// PoissonSolver(bunch, bend, bc, mesh, layout).computeField(EFD, HFD, JFD, dt),
// TETMSolver(AlphaE, AlphaH, bunch, msg, EFD, dt), updateField_firstStep /
// updateField_secondStep(EFD, HFD, JFD, mmE, mmH, mmJ, ddim, bc, geo) and
// moveMesh(mmE, mmH, mmJ, EFD, HFD, ddim, bunch.getGlobalBounds()), with host
// views bound to its own arrays.  Prints the window domain, checksums of the
// mirrored static and window fields and the beam centroid.  Built by
// tests/test_cpp_facade.py.
#include <cmath>
#include <cstdio>
#include <vector>

#include "csrst/csrst.hpp"

namespace {

struct Inform {};
struct Tag {};

csrst::FieldView view(std::vector<double> &buf, int nx, int ny, int guard) {
  const int pitch = nx + 2 * guard;
  buf.assign((size_t)pitch * (ny + 2 * guard), 0.0);
  csrst::FieldView v;
  v.ptr = buf.data(); v.nx = nx; v.ny = ny; v.pitch = pitch; v.guard = guard;
  return v;
}

double abs_sum(const csrst::FieldView &v) {
  double s = 0.0;
  for (int j = 0; j < v.ny; ++j)
    for (int i = 0; i < v.nx; ++i) s += std::fabs(v(i, j));
  return s;
}

}  // namespace

int main(int argc, char **argv) {
  const int steps = argc > 1 ? std::atoi(argv[1]) : 4;
  // 512 x 104 mesh at 20 um, 2 mm pipe, R = 0.25 m, gamma = 1000, TSC
  csrst_config cfg{};
  cfg.Nx = 512; cfg.Ny = 104; cfg.shape_order = 1;
  cfg.length_before = 0.0055976313069747725; cfg.length_after = 0.001; cfg.width = 0.002;
  cfg.phi_deg = 0.8223645856699741; cfg.ekin_mev = 510.489; cfg.bz = 6.8180466968243225;
  cfg.dt = 0.5 * 20e-6 / 299792458.0; cfg.charge_mass = -1e-9 / 0.51099906e-03;
  const double dt = cfg.dt;
  try {
    csrst::Simulation sim(cfg);
    // the bunch: argv[2] holds x, y, px, py, q of n particles as five arrays of doubles
    if (argc < 3) {
      std::fprintf(stderr, "usage: views_main steps bunch.bin\n");
      return 1;
    }
    FILE *f = std::fopen(argv[2], "rb");
    if (!f) return 1;
    std::fseek(f, 0, SEEK_END);
    const size_t n = (size_t)std::ftell(f) / (5 * sizeof(double));
    std::fseek(f, 0, SEEK_SET);
    std::vector<double> x(n), y(n), px(n), py(n), q(n);
    size_t got = 0;
    for (std::vector<double> *v : {&x, &y, &px, &py, &q}) got += std::fread(v->data(), sizeof(double), n, f);
    std::fclose(f);
    if (got != 5 * n) return 1;
    sim.loadBunch(x, y, px, py, q);
    csrst::PartBunch bunch(sim);
    bunch.makeReady(dt);
    std::vector<double> b[12];
    csrst::EdgeFieldView EFD{view(b[0], cfg.Nx, cfg.Ny, 1), view(b[1], cfg.Nx, cfg.Ny, 1)}, JFD;
    csrst::CellFieldView HFD{view(b[2], cfg.Nx, cfg.Ny, 1), view(b[3], cfg.Nx, cfg.Ny, 1)};
    Tag bend, bcells, mesh, layout, bc, geo;
    int alphaE = 0, alphaH = 0;
    Inform msg;
    csrst::PoissonSolver poisson(bunch, bend, bcells, mesh, layout);
    poisson.computeField(EFD, HFD, JFD, dt, 1e-12, 500);
    std::printf("poisson %.17g %.17g\n", abs_sum(EFD.x), abs_sum(HFD.x));
    csrst::TETMSolver solver(alphaE, alphaH, bunch, msg, EFD, dt);
    csrst::NDIndex2 ddim, gb;
    csrst::Vector2 org;
    sim.window(ddim, gb, org);
    const int L0 = ddim.length(0), L1 = ddim.length(1);
    csrst::EdgeFieldView mmE{view(b[4], L0, L1, 1), view(b[5], L0, L1, 1)};
    csrst::CellFieldView mmH{view(b[6], L0, L1, 1), view(b[7], L0, L1, 1)};
    csrst::EdgeFieldView mmJ{view(b[8], L0, L1, 1), view(b[9], L0, L1, 1)};
    for (int s = 0; s < steps; ++s) {
      solver.updateField_firstStep(EFD, HFD, JFD, mmE, mmH, mmJ, ddim, bc, geo);
      solver.updateField_secondStep(EFD, HFD, JFD, mmE, mmH, mmJ, ddim, bc, geo);
      csrst::moveMesh(sim, mmE, mmH, mmJ, EFD, HFD, ddim, bunch.getGlobalBounds());
    }
    std::printf("ddim %d %d %d %d\n", ddim.i0, ddim.i1, ddim.j0, ddim.j1);
    std::printf("static %.17g %.17g %.17g %.17g\n", abs_sum(EFD.x), abs_sum(EFD.y), abs_sum(HFD.x), abs_sum(HFD.y));
    std::printf("window %.17g %.17g %.17g\n", abs_sum(mmE.x), abs_sum(mmE.y), abs_sum(mmJ.y));
    csrst::PartBunchState st;
    bunch.calcBeamParameters(st);
    std::printf("rmean %.17g %.17g\n", st.rmean[0], st.rmean[1]);
  } catch (const csrst::Error &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
