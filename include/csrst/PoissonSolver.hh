// PoissonSolver of the reference (src/PoissonSolver.hh:47-66) over the GPU
// Simulation: the initial fields of the loaded bunch in its rest frame,
// boosted to the lab frame (PoissonSolver::computeField,
// src/PoissonSolver.cpp:85-201), followed by resetOutsideDomain as
// src/main.cpp:232-248 does.  The three solves run as multigrid-preconditioned
// CG on the device; the bend, its boundary cells, the mesh and the layout are
// the Simulation's (the reference's constructor arguments are accepted for
// the call shape).
#pragma once

#include <cmath>

#include "PartBunch.hh"
#include "core.hpp"

namespace csrst {

class PoissonSolver {
 public:
  // PoissonSolver(bunch, bend, bc, mesh, fl, periodicX, periodicY)
  // (PoissonSolver.hh:50-56); only PEC ends, as the reference's loop uses.
  template <class BendT, class BC, class Mesh, class Layout>
  PoissonSolver(PartBunch &bunch, const BendT &, const BC &, const Mesh &, const Layout &) : s_(bunch.simulation()) {}
  explicit PoissonSolver(Simulation &s) : s_(s) {}

  // computeField(EFD, HFD, JFD, dt, tol, maxIterations) (PoissonSolver.hh:60-65):
  // tol is the first solve's relative residual; the other two use 1e-6 as
  // the reference does (PoissonSolver.cpp:172).  dt must be the
  // Simulation's.  Bound views receive the static fields afterwards (E, the
  // split Hz, and J = 0).
  void computeField(EdgeFieldView &EFD, CellFieldView &HFD, EdgeFieldView &JFD, const double &dt,
                    const double &tol = 1e-8, const int &maxIterations = 100) {
    const double own = s_.info()[4];
    if (!(std::abs(dt - own) <= 1e-12 * own)) throw Error(CSRST_E_ARG, "computeField: dt differs from the Simulation's");
    computeField(tol, maxIterations);
    detail::mirror_static(s_, EFD, HFD, JFD);
  }
  void computeField(double tol = 1e-12, int maxIterations = 500) {
    check(csrst_initial_fields(s_.handle(), tol, 1e-6, maxIterations, report_.data()), s_.handle());
  }
  // gamma, (iterations, relative residual) of each solve, multigrid levels
  const std::array<double, 8> &report() const { return report_; }

 private:
  Simulation &s_;
  std::array<double, 8> report_{};
};

}  // namespace csrst
