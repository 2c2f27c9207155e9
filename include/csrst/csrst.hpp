// C++ facade over the C ABI (include/csrst.h) that keeps the call shapes of
// the reference's PIC-loop classes:
//   TETMSolver::updateField_firstStep / updateField_secondStep  (src/TETMSolver.hh:50-70)
//   PartBunch::push_particles / drift_particles / calcBeamParameters /
//             getGlobalBounds                                   (src/PartBunch.hh:46-112)
//   ScatterGatherImpl<IntOp, double>::gather                    (src/ScatterGatherImpl.hh:27-64)
//   moveMesh                                                    (src/main.cpp:562-652)
//   PoissonSolver::computeField                                 (src/PoissonSolver.hh:60-65)
// IPPL field and attribute types are replaced by host views (core.hpp:
// FieldView, EdgeFieldView, CellFieldView, ParticleView, NDIndex2); the
// fields and the bunch themselves live on the GPU inside a Simulation.
// Failures throw csrst::Error (the reference aborts through PAssert).
#pragma once

#include "core.hpp"
#include "PartBunch.hh"
#include "PoissonSolver.hh"
#include "ScatterGatherImpl.hh"
#include "TETMSolver.hh"
