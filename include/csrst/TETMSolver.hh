// TETMSolver of the reference (src/TETMSolver.hh:36-110) and moveMesh
// (src/main.cpp:562-652) over the GPU Simulation: the same method names,
// argument order and meaning, with the host views of core.hpp in place of
// IPPL fields.  The fields live on the device; every bound view receives its
// field after the call, and ddim the window's domain.  The template
// arguments bc (the cut-cell boundary, SCBoundaryCondition) and geo (the
// bend, Bend) are accepted for the call shape: the Simulation's
// configuration fixes both.
#pragma once

#include <cmath>

#include "PartBunch.hh"
#include "core.hpp"

namespace csrst {

class TETMSolver {
 public:
  // TETMSolver(AlphaE, AlphaH, bunch, msg, EFD, dt) (TETMSolver.hh:40-45): the
  // cut-cell coefficient fields AlphaE / AlphaH are built on the device from
  // the bend; dt must be the Simulation's.
  template <class AlphaField, class Msg>
  TETMSolver(AlphaField &, AlphaField &, PartBunch &bunch, Msg &, const EdgeFieldView &, const double &dt)
      : TETMSolver(bunch.simulation()) {
    if (!(std::abs(dt - dt_) <= 1e-12 * dt_)) throw Error(CSRST_E_ARG, "TETMSolver: dt differs from the Simulation's");
  }
  explicit TETMSolver(Simulation &s) : s_(s) { dt_ = s.info()[4]; }

  double getDT() const { return dt_; }

  // updateField_firstStep(EFD, Hz, JFD, mmE, mmH, mmJ, ddim, bc, geo)
  // (TETMSolver.hh:50-59): push with Jcomp 0, half H, Ex, half H (static
  // mesh, cut cells and window, with the strip exchanges), drift back.
  template <class G, class BC>
  void updateField_firstStep(EdgeFieldView &EFD, CellFieldView &Hz, EdgeFieldView &JFD, EdgeFieldView &mmE,
                             CellFieldView &mmH, EdgeFieldView &mmJ, NDIndex2 &ddim, const BC &, G &) {
    updateField_firstStep();
    mirror(EFD, Hz, JFD, mmE, mmH, mmJ, ddim);
  }
  // updateField_secondStep (TETMSolver.hh:61-70): push with Jcomp 1, Ey,
  // drift back.
  template <class G, class BC>
  void updateField_secondStep(EdgeFieldView &EFD, CellFieldView &Hz, EdgeFieldView &JFD, EdgeFieldView &mmE,
                              CellFieldView &mmH, EdgeFieldView &mmJ, NDIndex2 &ddim, const BC &, G &) {
    updateField_secondStep();
    mirror(EFD, Hz, JFD, mmE, mmH, mmJ, ddim);
  }
  void updateField_firstStep() { check(csrst_step_first(s_.handle()), s_.handle()); }
  void updateField_secondStep() { check(csrst_step_second(s_.handle()), s_.handle()); }

 private:
  void mirror(EdgeFieldView &EFD, CellFieldView &Hz, EdgeFieldView &JFD, EdgeFieldView &mmE, CellFieldView &mmH,
              EdgeFieldView &mmJ, NDIndex2 &ddim) {
    NDIndex2 gb;
    Vector2 org;
    s_.window(ddim, gb, org);
    detail::mirror_static(s_, EFD, Hz, JFD);
    const FieldView *v[6] = {&mmE.x, &mmE.y, &mmH.x, &mmH.y, &mmJ.x, &mmJ.y};
    detail::mirror_window(s_, v, ddim, org);
  }
  Simulation &s_;
  double dt_ = 0;
};

// moveMesh(miniMeshE, miniMeshH, miniMeshJ, EFD, HFD, ddim, newGlobalPos)
// (main.cpp:562-652): the window follows the bunch by whole cells and
// refreshes its strips.  newGlobalPos is the bunch's bounds of the last push
// (bunch.getGlobalBounds(), which the device already holds); another value
// is an error.  Bound views receive the fields after the move, ddim the new
// window domain.
inline void moveMesh(Simulation &s, EdgeFieldView &miniMeshE, CellFieldView &miniMeshH, EdgeFieldView &miniMeshJ,
                     EdgeFieldView &EFD, CellFieldView &HFD, NDIndex2 &ddim, const NDIndex2 &newGlobalPos) {
  NDIndex2 now, gb;
  Vector2 org;
  s.window(now, gb, org);
  if (gb != newGlobalPos) throw Error(CSRST_E_ARG, "moveMesh: newGlobalPos is not the bunch's bounds of the last push");
  check(csrst_move_window(s.handle()), s.handle());
  s.window(ddim, gb, org);
  EdgeFieldView nojx;
  detail::mirror_static(s, EFD, HFD, nojx);
  const FieldView *v[6] = {&miniMeshE.x, &miniMeshE.y, &miniMeshH.x, &miniMeshH.y, &miniMeshJ.x, &miniMeshJ.y};
  detail::mirror_window(s, v, ddim, org);
}
inline void moveMesh(Simulation &s) { check(csrst_move_window(s.handle()), s.handle()); }

}  // namespace csrst
