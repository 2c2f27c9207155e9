// ScatterGatherImpl<IntOp, double> of the reference (src/ScatterGatherImpl.hh:27-64,
// specialisations for IntCIC, IntS1, IntS2 below it) and its FieldPatch
// (src/FieldPatch.hh:33-132) on host data, computed on the GPU
// (csrst_gather).  The particle attributes are the views of core.hpp.
#pragma once

#include <algorithm>

#include "core.hpp"

namespace csrst {

// A dense field patch on the host: element (i, j) relative to the patch's
// first cell at data[j * nx + i] (FieldPatch::getRelative(i, j)), with the
// patch's origin and spacing (getOrigin, getSpacing).
struct FieldPatch {
  const double *data;
  int nx, ny;
  std::array<double, 2> origin, spacing;
  const double &getRelative(size_t i, size_t j) const { return data[j * (size_t)nx + i]; }
  const std::array<double, 2> &getOrigin() const { return origin; }
  const std::array<double, 2> &getSpacing() const { return spacing; }
};

template <class IntOp, class T = double>
struct ScatterGatherImpl {
  // gather(fp, fld, R, comp, from, to) (ScatterGatherImpl.hh:29-36): the edge
  // component comp % 2 of fp at R[from, to) into fld's component comp % 2.
  static void gather(const FieldPatch &fp, VectorAttribView &fld, const ParticleView &R, const size_t &comp,
                     size_t from, size_t to) {
    to = std::min({to, fld.n, R.n});
    from = std::min(from, to);
    gather(fp, fld.c[comp % 2], R.x, R.y, comp, from, to);
  }
  // gather(fp, fld, R, from, to) (ScatterGatherImpl.hh:38-44): a cell-centred
  // field into a scalar attribute.
  static void gather(const FieldPatch &fp, double *fld, size_t nfld, const ParticleView &R, size_t from, size_t to) {
    to = std::min({to, nfld, R.n});
    from = std::min(from, to);
    gather(fp, fld, R.x, R.y, from, to);
  }
  // The same on plain arrays: x, y, fld indexed from 0 like R.
  static void gather(const FieldPatch &fp, double *fld, const double *x, const double *y, size_t comp, size_t from,
                     size_t to) {
    if (to <= from) return;
    check(csrst_gather(IntOp::order, (int)(comp % 2), fp.data, fp.nx, fp.ny, fp.origin.data(), fp.spacing.data(),
                       x + from, y + from, to - from, fld + from));
  }
  static void gather(const FieldPatch &fp, double *fld, const double *x, const double *y, size_t from, size_t to) {
    if (to <= from) return;
    check(csrst_gather(IntOp::order, 2, fp.data, fp.nx, fp.ny, fp.origin.data(), fp.spacing.data(), x + from,
                       y + from, to - from, fld + from));
  }
};

}  // namespace csrst
