// C entry points into the reference's own sources, compiled here from where
// they lie (oracle/Makefile, target `ref`, output oracle/_ref/) against the
// one-process IPPL stand-in of oracle/refshim: the cell and dual-cell
// crossing splits and Q_rsqrt of src/utils.hh, the current deposits of
// src/{Zeroth,First,Second}OrderShapeFunction.cpp (getCurrentDensityBaseImplX/Y)
// and the field gathers of src/FieldPatch.hh / src/ScatterGatherImpl.hh.
// Test infrastructure: the oracle is checked against these; nothing else
// loads them.
#include "PartBunch.hh"
#include "Communicator.hh"
#include "FieldPatch.hh"
#include "ShapeFunction.hh"
#include "utils.hh"

namespace {

template <class SF>
int deposit(int comp, const double *ox, const double *oy, const double *x, const double *y, const double *q,
            long n, double org0, double org1, double h0, double h1, double dt, int i0, int j0, int ni, int nj,
            double *J, int *dom4) {
  PartBunch b;
  b.R.create(n); b.oldR.create(n); b.Q.create(n);
  for (long k = 0; k < n; ++k) {
    b.R[k] = Vector_t(x[k], y[k]);
    b.oldR[k] = Vector_t(ox[k], oy[k]);
    b.Q[k] = q[k];
  }
  VField_Edge_t JFD;
  const double hh[2] = {h0, h1};
  JFD.get_mesh().set_meshSpacing(hh);
  JFD.get_mesh().set_origin(Vector_t(org0, org1));
  const Timings::TimerRef t = 0;
  try {
    FieldPatch<double> fp = comp == 0 ? SF::getCurrentDensityBaseImplX(JFD, b, dt, t, 0, (size_t)n)
                                      : SF::getCurrentDensityBaseImplY(JFD, b, dt, t, 0, (size_t)n);
    const NDIndex<DIM> &d = fp.getDomain();
    if (dom4) { dom4[0] = d[0].first(); dom4[1] = d[0].last(); dom4[2] = d[1].first(); dom4[3] = d[1].last(); }
    for (int j = d[1].first(); j <= d[1].last(); ++j)
      for (int i = d[0].first(); i <= d[0].last(); ++i) {
        const int a = i - i0, c = j - j0;
        if (a >= 0 && c >= 0 && a < ni && c < nj) J[(size_t)c * ni + a] += fp(i, j);
      }
  } catch (const PAssertFailed &) {
    return 1;  // the reference's patch index check failed
  }
  return 0;
}

}  // namespace

extern "C" {

float ref_q_rsqrt(float x) { return Utils::Q_rsqrt(x); }

// The crossing split of the move old -> new (cells borders or, dual != 0,
// dual-cell borders): fractions and points, n of them (the return value).
long ref_crossings(int dual, double o0, double o1, double n0, double n1, double h0, double h1, double org0,
                   double org1, double *frac, double *s0, double *s1) {
  Utils::CompanionSorterItem xs[32];
  const Vector_t dx(h0, h1);
  Utils::samePos uni(sqrt(dot(dx, dx)));
  const size_t n = dual ? Utils::calcDualCellBorderCrossings(xs, Vector_t(o0, o1), Vector_t(n0, n1), dx,
                                                             Vector_t(org0, org1), uni)
                        : Utils::calcCellBorderCrossings(xs, Vector_t(o0, o1), Vector_t(n0, n1), dx,
                                                         Vector_t(org0, org1), uni);
  for (size_t k = 0; k < n; ++k) { frac[k] = xs[k].fraction; s0[k] = xs[k].subStep(0); s1[k] = xs[k].subStep(1); }
  return (long)n;
}

// getCurrentDensityBaseImplX (comp 0) / Y (comp 1) of shape order `order`
// for n particles moving old -> new, added into the dense (ni x nj) patch J
// whose element (0, 0) is mesh index (i0, j0); dom4 receives the reference's
// own patch domain.  Returns 1 if the reference's patch index check failed.
int ref_deposit(int order, int comp, const double *ox, const double *oy, const double *x, const double *y,
                const double *q, long n, double org0, double org1, double h0, double h1, double dt, int i0, int j0,
                int ni, int nj, double *J, int *dom4) {
  if (order == 0)
    return deposit<ZerothOrderShapeFunction>(comp, ox, oy, x, y, q, n, org0, org1, h0, h1, dt, i0, j0, ni, nj, J, dom4);
  if (order == 1)
    return deposit<FirstOrderShapeFunction>(comp, ox, oy, x, y, q, n, org0, org1, h0, h1, dt, i0, j0, ni, nj, J, dom4);
  return deposit<SecondOrderShapeFunction>(comp, ox, oy, x, y, q, n, org0, org1, h0, h1, dt, i0, j0, ni, nj, J, dom4);
}

// FieldPatch<double>::gather of a dense (nx x ny) patch (x fastest) with
// origin o and spacing h at n positions: comp 0 / 1 edge components, 2 the
// cell-centred scalar.  Returns 1 if a patch index check failed.
int ref_gather(int order, int comp, const double *patch, int nx, int ny, double o0, double o1, double h0,
               double h1, const double *x, const double *y, long n, double *out) {
  FieldPatch<double> fp(NDIndex<DIM>(Index(0, nx - 1), Index(0, ny - 1)));
  fp.setOrigin(Vector_t(o0, o1));
  fp.setSpacing(Vector_t(h0, h1));
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) fp(i, j) = patch[(size_t)j * nx + i];
  ParticleAttrib<Vector_t> pp;
  pp.create(n);
  for (long k = 0; k < n; ++k) pp[k] = Vector_t(x[k], y[k]);
  try {
    if (comp == 2) {
      ParticleAttrib<double> f;
      f.create(n);
      if (order == 0) fp.gather(f, pp, IntCIC(), 0, (size_t)n);
      else if (order == 1) fp.gather(f, pp, IntS1(), 0, (size_t)n);
      else fp.gather(f, pp, IntS2(), 0, (size_t)n);
      for (long k = 0; k < n; ++k) out[k] = f[k];
    } else {
      ParticleAttrib<Vector_t> f;
      f.create(n);
      if (order == 0) fp.gather(f, pp, (size_t)comp, IntCIC(), 0, (size_t)n);
      else if (order == 1) fp.gather(f, pp, (size_t)comp, IntS1(), 0, (size_t)n);
      else fp.gather(f, pp, (size_t)comp, IntS2(), 0, (size_t)n);
      for (long k = 0; k < n; ++k) out[k] = f[k](comp);
    }
  } catch (const PAssertFailed &) {
    return 1;
  }
  return 0;
}

}  // extern "C"
