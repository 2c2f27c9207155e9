// CPU ORACLE -- test infrastructure, not part of the product.
//
// A plain C++ restatement of the reference CSRST per-time-step PIC loop
// (kreischtauf/CSRST, src/), written to be the parity checker for the CUDA
// path.  Only tests/, __graft_entry__.smoke() and the cpu_baseline / reference
// arm of bench.py load this library.  The product (csrst_b200) never links,
// imports or calls it.
//
// Every function names the reference file:line it restates.  Floating point
// follows the reference's operation order exactly; it is compiled with
// -ffp-contract=off so that no FMA contraction changes a rounding.
//
// Restated IPPL semantics (the reference's third-party field library, not
// vendored): an edge-centred field on N vertices has index domain [0, N-1];
// a cell-centred field on the (N+1)-vertex mesh also has [0, N-1]; guard
// layers are one cell wide, start at zero and are written only by the
// explicit exchanges; where(mask, a, b) leaves masked-out elements unchanged.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// Physical constants, src/Physics.cpp:41-51.
const double PI = 3.14159265358979323846;
const double C = 299792458.0;
const double MU0 = 1.256637061e-06;
const double EPS0 = 8.854187817e-12;
// src/defs.hh:30-31
const double SPACE_EPS = 1e-10;
const double MINAREA = 1e-20;

// src/utils.hh:491-504 (float fast inverse square root used for 1/gamma).
float q_rsqrt(float x) {
  float xhalf = 0.5f * x;
  float xqhalf = 0.5010936f * x;
  uint32_t i;
  std::memcpy(&i, &x, sizeof(i));
  i = 0x5f3759df - (i >> 1);
  std::memcpy(&x, &i, sizeof(i));
  x = x * (1.5f - xhalf * x * x);
  x = x * (1.5010936f - xqhalf * x * x);
  return x;
}

// A 2D field component with a guard layer of width g on every side.
struct Grid {
  int nx = 0, ny = 0, g = 1;
  std::vector<double> v;
  void init(int nx_, int ny_, int g_ = 1) {
    nx = nx_; ny = ny_; g = g_;
    v.assign((size_t)(nx + 2 * g) * (ny + 2 * g), 0.0);
  }
  double &at(int i, int j) { return v[(size_t)(j + g) * (nx + 2 * g) + (i + g)]; }
  double at(int i, int j) const { return v[(size_t)(j + g) * (nx + 2 * g) + (i + g)]; }
};

// Crossing list entry, src/utils.hh:64-67.
struct Xing {
  double fraction;
  double s0, s1;
};

// libstdc++ std::sort on <= 16 elements is an insertion sort, which keeps the
// order of equal keys; this restates it (src/utils.hh:418, 481).
void sort_fractions(Xing *b, Xing *e) {
  for (Xing *i = b + 1; i < e; ++i) {
    Xing v = *i;
    Xing *j = i;
    while (j > b && v.fraction < (j - 1)->fraction) { *j = *(j - 1); --j; }
    *j = v;
  }
}

// std::unique with samePos (|a-b| < 1e-6 on the fraction), src/utils.hh:87-90.
size_t unique_fractions(Xing *b, size_t n) {
  if (n == 0) return 0;
  size_t dest = 0;
  for (size_t k = 1; k < n; ++k) {
    if (!(std::abs(b[dest].fraction - b[k].fraction) < 1e-6)) b[++dest] = b[k];
  }
  return dest + 1;
}

// src/utils.hh:427-489 (cell borders) and :364-425 (dual cell borders, shift=0.5).
size_t border_crossings(Xing *xs, double o0, double o1, double n0, double n1,
                        double h0, double h1, double org0, double org1, bool dual) {
  o0 -= org0; o1 -= org1; n0 -= org0; n1 -= org1;
  int Ii, Ji, If, Jf;
  if (dual) {
    Ii = (int)std::floor(o0 / h0 - 0.5); Ji = (int)std::floor(o1 / h1 - 0.5);
    If = (int)std::floor(n0 / h0 - 0.5); Jf = (int)std::floor(n1 / h1 - 0.5);
  } else {
    Ii = (int)std::floor(o0 / h0); Ji = (int)std::floor(o1 / h1);
    If = (int)std::floor(n0 / h0); Jf = (int)std::floor(n1 / h1);
  }
  int I = Ii, J = Ji;
  const double D0 = n0 - o0, D1 = n1 - o1;
  size_t next = 0;
  xs[next++].fraction = 0.0;
  while (I < If) {
    double x = dual ? h0 * (I + 1.5) : h0 * (I + 1);
    xs[next].fraction = (x - o0) / D0;
    xs[next].s0 = x; xs[next].s1 = o1 + xs[next].fraction * D1;
    ++I; ++next;
  }
  while (I > If) {
    double x = dual ? h0 * (I + 0.5) : h0 * I;
    xs[next].fraction = (x - o0) / D0;
    xs[next].s0 = x; xs[next].s1 = o1 + xs[next].fraction * D1;
    --I; ++next;
  }
  while (J < Jf) {
    double y = dual ? h1 * (J + 1.5) : h1 * (J + 1);
    xs[next].fraction = (y - o1) / D1;
    xs[next].s0 = o0 + xs[next].fraction * D0; xs[next].s1 = y;
    ++J; ++next;
  }
  while (J > Jf) {
    double y = dual ? h1 * (J + 0.5) : h1 * J;
    xs[next].fraction = (y - o1) / D1;
    xs[next].s0 = o0 + xs[next].fraction * D0; xs[next].s1 = y;
    --J; ++next;
  }
  xs[next++].fraction = 1.0;
  sort_fractions(xs + 1, xs + next - 1);
  size_t num = unique_fractions(xs, next);
  xs[0].s0 = o0; xs[0].s1 = o1;
  xs[num - 1].s0 = n0; xs[num - 1].s1 = n1;
  return num;
}

// ---------------------------------------------------------------------------
// Field gather, src/ScatterGatherImpl.hh.  f(I, J) reads a patch whose
// relative index (0, 0) sits at the patch origin.
struct Patch {
  const double *p; int nx, ny; double o0, o1, h0, h1;
  double operator()(long i, long j) const { return p[(size_t)j * nx + i]; }
};

// IntCIC edge gather, ScatterGatherImpl.hh:69-104
double gather_cic_edge(const Patch &fp, double r0, double r1, int comp) {
  const double ood0 = 1.0 / fp.h0, ood1 = 1.0 / fp.h1;
  double add0 = comp == 0 ? 0.5 : 0.0, add1 = comp == 1 ? 0.5 : 0.0;
  double pp0 = (r0 - fp.o0) * ood0, pp1 = (r1 - fp.o1) * ood1;
  long l0 = (long)std::floor(pp0 + add0), l1 = (long)std::floor(pp1 + add1);
  if (comp == 0) l0 -= 1; else l1 -= 1;
  double g0 = (double)l0, g1 = (double)l1;
  if (comp == 0) g0 += 0.5; else g1 += 0.5;
  double d0 = pp0 - g0, d1 = pp1 - g1;
  return ((1 - d1) * ((1 - d0) * fp(l0, l1) + d0 * fp(l0 + 1, l1)) +
          d1 * ((1 - d0) * fp(l0, l1 + 1) + d0 * fp(l0 + 1, l1 + 1)));
}

// IntCIC cell gather, ScatterGatherImpl.hh:106-134
double gather_cic_cell(const Patch &fp, double r0, double r1) {
  const double ood0 = 1.0 / fp.h0, ood1 = 1.0 / fp.h1;
  double pp0 = (r0 - fp.o0) * ood0, pp1 = (r1 - fp.o1) * ood1;
  long l0 = (long)std::floor(pp0 - 0.5), l1 = (long)std::floor(pp1 - 0.5);
  double d0 = pp0 - (l0 + 0.5), d1 = pp1 - (l1 + 0.5);
  return ((1 - d1) * ((1 - d0) * fp(l0, l1) + d0 * fp(l0 + 1, l1)) +
          d1 * ((1 - d0) * fp(l0, l1 + 1) + d0 * fp(l0 + 1, l1 + 1)));
}

inline void s1_w(double d, double &a, double &b, double &c) {
  b = 0.75 - d * d;
  c = 0.5 * (0.5 + d) * (0.5 + d);
  a = 1.0 - (b + c);
}

double s1_sum(const Patch &fp, long I, long J, double d0, double d1) {
  double ax, bx, cx, ay, by, cy;
  s1_w(d0, ax, bx, cx);
  s1_w(d1, ay, by, cy);
  return (ay * (ax * fp(I - 1, J - 1) + bx * fp(I, J - 1) + cx * fp(I + 1, J - 1)) +
          by * (ax * fp(I - 1, J) + bx * fp(I, J) + cx * fp(I + 1, J)) +
          cy * (ax * fp(I - 1, J + 1) + bx * fp(I, J + 1) + cx * fp(I + 1, J + 1)));
}

// IntS1 edge gather, ScatterGatherImpl.hh:201-253
double gather_s1_edge(const Patch &fp, double r0, double r1, int comp) {
  const double ood0 = 1.0 / fp.h0, ood1 = 1.0 / fp.h1;
  double add0 = comp == 0 ? 0.0 : 0.5, add1 = comp == 1 ? 0.0 : 0.5;
  double pp0 = (r0 - fp.o0) * ood0, pp1 = (r1 - fp.o1) * ood1;
  long l0 = (long)std::floor(pp0 + add0), l1 = (long)std::floor(pp1 + add1);
  double g0 = (double)l0, g1 = (double)l1;
  if (comp == 0) g0 += 0.5; else g1 += 0.5;
  return s1_sum(fp, l0, l1, pp0 - g0, pp1 - g1);
}

// IntS1 cell gather, ScatterGatherImpl.hh:255-301
double gather_s1_cell(const Patch &fp, double r0, double r1) {
  const double ood0 = 1.0 / fp.h0, ood1 = 1.0 / fp.h1;
  double pp0 = (r0 - fp.o0) * ood0, pp1 = (r1 - fp.o1) * ood1;
  long l0 = (long)std::floor(pp0), l1 = (long)std::floor(pp1);
  return s1_sum(fp, l0, l1, pp0 - (l0 + 0.5), pp1 - (l1 + 0.5));
}

const double TWOTHIRDS = 2.0 / 3.0;
const double ONESIXTH = 1.0 / 6.0;

inline void s2_w(double d, double &a, double &b, double &c, double &e) {
  double dsq = d * d;
  b = TWOTHIRDS - dsq * (1 - 0.5 * d);
  c = TWOTHIRDS - 0.5 * (1 - d) * (1 - dsq);
  e = ONESIXTH * dsq * d;
  a = 1.0 - (b + c + e);
}

// The last term reads (I+1, J+2) as the reference does (ScatterGatherImpl.hh:467, :525).
double s2_sum(const Patch &fp, long I, long J, double d0, double d1) {
  double ax, bx, cx, ex, ay, by, cy, ey;
  s2_w(d0, ax, bx, cx, ex);
  s2_w(d1, ay, by, cy, ey);
  return (ay * (ax * fp(I - 1, J - 1) + bx * fp(I, J - 1) + cx * fp(I + 1, J - 1) + ex * fp(I + 2, J - 1)) +
          by * (ax * fp(I - 1, J) + bx * fp(I, J) + cx * fp(I + 1, J) + ex * fp(I + 2, J)) +
          cy * (ax * fp(I - 1, J + 1) + bx * fp(I, J + 1) + cx * fp(I + 1, J + 1) + ex * fp(I + 2, J + 1)) +
          ey * (ax * fp(I - 1, J + 2) + bx * fp(I, J + 2) + cx * fp(I + 1, J + 2) + ex * fp(I + 1, J + 2)));
}

// IntS2 edge gather, ScatterGatherImpl.hh:406-468
double gather_s2_edge(const Patch &fp, double r0, double r1, int comp) {
  const double ood0 = 1.0 / fp.h0, ood1 = 1.0 / fp.h1;
  double add0 = comp == 0 ? 0.5 : 0.0, add1 = comp == 1 ? 0.5 : 0.0;
  double pp0 = (r0 - fp.o0) * ood0, pp1 = (r1 - fp.o1) * ood1;
  long l0 = (long)std::floor(pp0 + add0), l1 = (long)std::floor(pp1 + add1);
  if (comp == 0) l0 -= 1; else l1 -= 1;
  double g0 = (double)l0, g1 = (double)l1;
  if (comp == 0) g0 += 0.5; else g1 += 0.5;
  return s2_sum(fp, l0, l1, pp0 - g0, pp1 - g1);
}

// IntS2 cell gather, ScatterGatherImpl.hh:470-527
double gather_s2_cell(const Patch &fp, double r0, double r1) {
  const double ood0 = 1.0 / fp.h0, ood1 = 1.0 / fp.h1;
  double pp0 = (r0 - fp.o0) * ood0, pp1 = (r1 - fp.o1) * ood1;
  long l0 = (long)std::floor(pp0 - 0.5), l1 = (long)std::floor(pp1 - 0.5);
  return s2_sum(fp, l0, l1, pp0 - (l0 + 0.5), pp1 - (l1 + 0.5));
}

double gather_edge(int order, const Patch &fp, double r0, double r1, int comp) {
  if (order == 0) return gather_cic_edge(fp, r0, r1, comp);
  if (order == 1) return gather_s1_edge(fp, r0, r1, comp);
  return gather_s2_edge(fp, r0, r1, comp);
}
double gather_cell(int order, const Patch &fp, double r0, double r1) {
  if (order == 0) return gather_cic_cell(fp, r0, r1);
  if (order == 1) return gather_s1_cell(fp, r0, r1);
  return gather_s2_cell(fp, r0, r1);
}

// Scatter (used by the reference's own known-answer test), ScatterGatherImpl.hh:136-194,
// :303-392, :529-642.  Adds w * value into a writable patch.
struct WPatch {
  double *p; int nx, ny; double o0, o1, h0, h1;
  double &operator()(long i, long j) { return p[(size_t)j * nx + i]; }
};

void scatter_one(int order, bool edge, int comp, WPatch &fp, double r0, double r1, double val) {
  const double ood0 = 1.0 / fp.h0, ood1 = 1.0 / fp.h1;
  double pp0 = (r0 - fp.o0) * ood0, pp1 = (r1 - fp.o1) * ood1;
  if (order == 0) {
    long l0, l1; double g0, g1;
    if (edge) {
      l0 = (long)std::floor(pp0 + (comp == 0 ? 0.5 : 0.0));
      l1 = (long)std::floor(pp1 + (comp == 1 ? 0.5 : 0.0));
      if (comp == 0) l0 -= 1; else l1 -= 1;
      g0 = (double)l0; g1 = (double)l1;
      if (comp == 0) g0 += 0.5; else g1 += 0.5;
    } else {
      l0 = (long)std::floor(pp0 - 0.5); l1 = (long)std::floor(pp1 - 0.5);
      g0 = l0 + 0.5; g1 = l1 + 0.5;
    }
    double d0 = pp0 - g0, d1 = pp1 - g1;
    fp(l0, l1) += (1 - d0) * (1 - d1) * val;
    fp(l0 + 1, l1) += d0 * (1 - d1) * val;
    fp(l0, l1 + 1) += (1 - d0) * d1 * val;
    fp(l0 + 1, l1 + 1) += d0 * d1 * val;
  } else if (order == 1) {
    long l0, l1; double g0, g1;
    if (edge) {
      l0 = (long)std::floor(pp0 + (comp == 0 ? 0.0 : 0.5));
      l1 = (long)std::floor(pp1 + (comp == 1 ? 0.0 : 0.5));
      g0 = (double)l0; g1 = (double)l1;
      if (comp == 0) g0 += 0.5; else g1 += 0.5;
    } else {
      l0 = (long)std::floor(pp0); l1 = (long)std::floor(pp1);
      g0 = l0 + 0.5; g1 = l1 + 0.5;
    }
    double d0 = pp0 - g0, d1 = pp1 - g1;
    double ax, bx, cx, ay, by, cy;
    if (edge) { s1_w(d0, ax, bx, cx); s1_w(d1, ay, by, cy); }
    else {  // the cell scatter uses the explicit a = 1/2 (1/2 - d)^2 (ScatterGatherImpl.hh:372-377)
      ax = 0.5 * (0.5 - d0) * (0.5 - d0); bx = 0.75 - d0 * d0; cx = 0.5 * (0.5 + d0) * (0.5 + d0);
      ay = 0.5 * (0.5 - d1) * (0.5 - d1); by = 0.75 - d1 * d1; cy = 0.5 * (0.5 + d1) * (0.5 + d1);
    }
    double wx[3] = {ax, bx, cx}, wy[3] = {ay, by, cy};
    for (int b = 0; b < 3; ++b)
      for (int a = 0; a < 3; ++a) fp(l0 - 1 + a, l1 - 1 + b) += wx[a] * wy[b] * val;
  } else {
    long l0, l1; double g0, g1;
    if (edge) {
      l0 = (long)std::floor(pp0 + (comp == 0 ? 0.5 : 0.0));
      l1 = (long)std::floor(pp1 + (comp == 1 ? 0.5 : 0.0));
      if (comp == 0) l0 -= 1; else l1 -= 1;
      g0 = (double)l0; g1 = (double)l1;
      if (comp == 0) g0 += 0.5; else g1 += 0.5;
    } else {
      l0 = (long)std::floor(pp0 - 0.5); l1 = (long)std::floor(pp1 - 0.5);
      g0 = l0 + 0.5; g1 = l1 + 0.5;
    }
    double ax, bx, cx, ex, ay, by, cy, ey;
    s2_w(pp0 - g0, ax, bx, cx, ex);
    s2_w(pp1 - g1, ay, by, cy, ey);
    double wx[4] = {ax, bx, cx, ex}, wy[4] = {ay, by, cy, ey};
    for (int b = 0; b < 4; ++b)
      for (int a = 0; a < 4; ++a) fp(l0 - 1 + a, l1 - 1 + b) += wx[a] * wy[b] * val;
  }
}

// ---------------------------------------------------------------------------
// Charge-conserving current deposit.  J(I, J) is an absolute index into a
// grid whose index (0, 0) sits at the mesh origin (the reference's
// FieldPatch::operator() uses absolute indices).
struct JSink {
  Grid *g;        // target (mini-mesh J component); contributions outside are dropped
  bool fixed;     // accumulate in 64-bit fixed point like the CUDA path
  double scale;
  std::vector<long long> acc;
  int i0 = 0, j0 = 0;  // absolute index of the target's element (0, 0)
  void add(int i, int j, double v) {
    i -= i0; j -= j0;
    if (i < -g->g || j < -g->g || i >= g->nx + g->g || j >= g->ny + g->g) return;
    if (fixed) acc[(size_t)(j + g->g) * (g->nx + 2 * g->g) + (i + g->g)] += std::llrint(v * scale);
    else g->at(i, j) += v;
  }
};

// ZerothOrderShapeFunction.cpp:171-294
void deposit0(JSink &J, int comp, double q, double o0, double o1, double n0, double n1,
              double h0, double h1, double org0, double org1, double dt) {
  Xing xs[16];
  const double ood0 = 1.0 / h0, ood1 = 1.0 / h1;
  const double oodt0 = 1.0 / (h1 * dt), oodt1 = 1.0 / (h0 * dt);
  size_t n = border_crossings(xs, o0, o1, n0, n1, h0, h1, org0, org1, false);
  for (size_t k = 0; k + 1 < n; ++k) {
    double xi0 = xs[k].s0 * ood0, xi1 = xs[k].s1 * ood1;
    double xf0 = xs[k + 1].s0 * ood0, xf1 = xs[k + 1].s1 * ood1;
    double D0 = q * (xf0 - xi0) * oodt0, D1 = q * (xf1 - xi1) * oodt1;
    double c0 = (xi0 + xf0) * 0.5, c1 = (xi1 + xf1) * 0.5;
    int I = (int)std::floor(c0), Jj = (int)std::floor(c1);
    if (comp == 0) {
      J.add(I, Jj, D0 * (Jj + 1 - c1));
      J.add(I, Jj + 1, D0 * (c1 - Jj));
    } else {
      J.add(I, Jj, D1 * (I + 1 - c0));
      J.add(I + 1, Jj, D1 * (c0 - I));
    }
  }
}

// FirstOrderShapeFunction.cpp:540-683 (getCurrentX / getCurrentY)
void current1(double *Jc, int comp, double tau, double a0, double a1, double b0, double b1,
              double qd0, double qd1, double dl0, double dl1) {
  const double cd0 = qd1 * dl0, cd1 = qd0 * dl1;
  const double half = 0.5, onethird = 1.0 / 3.0, onefourth = half * half;
  const double tp2 = tau * tau * half;
  const double tp3 = tp2 * tau * 2 * onethird;
  if (comp == 0) {
    const double Am = a0, Bm = -dl0 * tau, A0 = 1.0 - a0, B0 = dl0 * tau;
    const double Aym = half * (half + b1) * (half + b1) * tau;
    const double Bym = -(half + b1) * dl1 * tp2;
    const double Cym = half * dl1 * dl1 * tp3;
    const double Ay0 = (0.75 - b1 * b1) * tau;
    const double By0 = 2 * b1 * dl1 * tp2;
    const double Cy0 = -dl1 * dl1 * tp3;
    const double Ayp = half * (half - b1) * (half - b1) * tau;
    const double Byp = (half - b1) * dl1 * tp2;
    const double Cyp = half * dl1 * dl1 * tp3;
    Jc[0] = cd0 * ((Am + Bm) * (Aym + Bym + Cym) - Bm * (half * Aym + onethird * Bym + onefourth * Cym));
    Jc[1] = cd0 * ((A0 + B0) * (Aym + Bym + Cym) - B0 * (half * Aym + onethird * Bym + onefourth * Cym));
    Jc[2] = cd0 * ((Am + Bm) * (Ay0 + By0 + Cy0) - Bm * (half * Ay0 + onethird * By0 + onefourth * Cy0));
    Jc[3] = cd0 * ((A0 + B0) * (Ay0 + By0 + Cy0) - B0 * (half * Ay0 + onethird * By0 + onefourth * Cy0));
    Jc[4] = cd0 * ((Am + Bm) * (Ayp + Byp + Cyp) - Bm * (half * Ayp + onethird * Byp + onefourth * Cyp));
    Jc[5] = cd0 * ((A0 + B0) * (Ayp + Byp + Cyp) - B0 * (half * Ayp + onethird * Byp + onefourth * Cyp));
  } else {
    const double Axm = half * (half + b0) * (half + b0) * tau;
    const double Bxm = -(half + b0) * dl0 * tp2;
    const double Cxm = half * dl0 * dl0 * tp3;
    const double Ax0 = (0.75 - b0 * b0) * tau;
    const double Bx0 = 2 * b0 * dl0 * tp2;
    const double Cx0 = -dl0 * dl0 * tp3;
    const double Axp = half * (half - b0) * (half - b0) * tau;
    const double Bxp = (half - b0) * dl0 * tp2;
    const double Cxp = half * dl0 * dl0 * tp3;
    const double Am = a1, Bm = -dl1 * tau, A0 = 1.0 - a1, B0 = dl1 * tau;
    Jc[0] = cd1 * ((Am + Bm) * (Axm + Bxm + Cxm) - Bm * (half * Axm + onethird * Bxm + onefourth * Cxm));
    Jc[1] = cd1 * ((Am + Bm) * (Ax0 + Bx0 + Cx0) - Bm * (half * Ax0 + onethird * Bx0 + onefourth * Cx0));
    Jc[2] = cd1 * ((Am + Bm) * (Axp + Bxp + Cxp) - Bm * (half * Axp + onethird * Bxp + onefourth * Cxp));
    Jc[3] = cd1 * ((A0 + B0) * (Axm + Bxm + Cxm) - B0 * (half * Axm + onethird * Bxm + onefourth * Cxm));
    Jc[4] = cd1 * ((A0 + B0) * (Ax0 + Bx0 + Cx0) - B0 * (half * Ax0 + onethird * Bx0 + onefourth * Cx0));
    Jc[5] = cd1 * ((A0 + B0) * (Axp + Bxp + Cxp) - B0 * (half * Axp + onethird * Bxp + onefourth * Cxp));
  }
}

// FirstOrderShapeFunction.cpp:179-329
void deposit1(JSink &J, int comp, double q, double o0, double o1, double n0, double n1,
              double h0, double h1, double org0, double org1, double dt) {
  Xing xs[16];
  const double ood0 = 1.0 / h0, ood1 = 1.0 / h1;
  const double oodt0 = ood0 / dt, oodt1 = ood1 / dt;
  const double Dx0 = n0 - o0, Dx1 = n1 - o1;
  const double dl0 = Dx0 * ood0, dl1 = Dx1 * ood1;
  const double cov = std::sqrt(Dx0 * Dx0 + Dx1 * Dx1);
  // A particle that does not move deposits nothing (the reference evaluates 0/0 here).
  if (cov == 0.0) return;
  size_t n = border_crossings(xs, o0, o1, n0, n1, h0, h1, org0, org1, true);
  double Jc[6];
  for (size_t k = 0; k + 1 < n; ++k) {
    double xi0 = xs[k].s0 * ood0, xi1 = xs[k].s1 * ood1;
    double xf0 = xs[k + 1].s0 * ood0, xf1 = xs[k + 1].s1 * ood1;
    double sg0 = xs[k + 1].s0 - xs[k].s0, sg1 = xs[k + 1].s1 - xs[k].s1;
    double tau = std::sqrt(sg0 * sg0 + sg1 * sg1) / cov;
    double c0 = (xi0 + xf0) * 0.5, c1 = (xi1 + xf1) * 0.5;
    int I = (int)std::floor(c0 + 0.5), Jj = (int)std::floor(c1 + 0.5);
    double a0 = I + 0.5 - xi0, a1 = Jj + 0.5 - xi1;
    double b0 = I - xi0, b1 = Jj - xi1;
    current1(Jc, comp, tau, a0, a1, b0, b1, q * oodt0, q * oodt1, dl0, dl1);
    if (comp == 0) {
      J.add(I - 1, Jj - 1, Jc[0]); J.add(I, Jj - 1, Jc[1]);
      J.add(I - 1, Jj, Jc[2]);     J.add(I, Jj, Jc[3]);
      J.add(I - 1, Jj + 1, Jc[4]); J.add(I, Jj + 1, Jc[5]);
    } else {
      J.add(I - 1, Jj - 1, Jc[0]); J.add(I, Jj - 1, Jc[1]); J.add(I + 1, Jj - 1, Jc[2]);
      J.add(I - 1, Jj, Jc[3]);     J.add(I, Jj, Jc[4]);     J.add(I + 1, Jj, Jc[5]);
    }
  }
}

// SecondOrderShapeFunction.cpp:583-826.  x3 = S3 factors along the first axis
// of the cross direction, s2 = S2 factors along the current direction.
struct S2f { double A, B, C; };
struct S3f { double A, B, C, D; };

double cur2_term(double cd, const S2f &s, const S3f &t) {
  const double half = 0.5, onethird = 1.0 / 3.0, onefourth = 0.25, onefifth = 0.2;
  return cd * ((s.A + s.B + s.C) * (t.D + t.C + t.B + t.A)
               + (s.C * (t.D - t.A) - s.B * t.B) * onethird
               + (s.C * t.C - s.B * t.D) * onefifth
               - s.B * t.C * onefourth - s.B * t.A * half);
}

void s2_factors(S2f *f, double a, double dl, double dl2, double tau, double tp2) {
  const double half = 0.5;
  f[0] = {half * (half + a) * (half + a), -(half + a) * dl * tau, half * dl2 * tp2};
  f[1] = {0.75 - a * a, 2 * a * dl * tau, -dl2 * tp2};
  f[2] = {half * (0.5 - a) * (0.5 - a), (half - a) * dl * tau, half * dl2 * tp2};
}
// Jy variant of the S2 factors uses a different association (SecondOrderShapeFunction.cpp:776-784).
void s2_factors_y(S2f *f, double a, double dl, double dl2, double tau, double tp2) {
  const double half = 0.5;
  f[0] = {(half + a) * (half + a) * half, -(half + a) * dl * tau, dl2 * half * tp2};
  f[1] = {0.75 - a * a, 2 * a * dl * tau, -dl2 * tp2};
  f[2] = {(half - a) * (half - a) * half, (half - a) * dl * tau, dl2 * half * tp2};
}
void s3_factors(S3f *f, double b, double dl, double dl2, double dl3, double tau, double tp2,
                double tp3, double tp4) {
  const double half = 0.5, onesixth = half * (1.0 / 3.0);
  f[0] = {(1 + b) * (1 + b) * (1 + b) * onesixth * tau, -(1 + b) * (1 + b) * dl * half * tp2,
          (1 + b) * dl2 * half * tp3, -dl3 * onesixth * tp4};
  f[1] = {(4 - 3 * b * b * (2 + b)) * onesixth * tau, b * dl * (3 * b + 4) * half * tp2,
          -dl2 * (2 + 3 * b) * half * tp3, dl3 * half * tp4};
  f[2] = {(4 - 3 * (b + 1) * (b + 1) * (1 - b)) * onesixth * tau, (1 - 2 * b - 3 * b * b) * dl * half * tp2,
          (1 + 3 * b) * dl2 * half * tp3, -dl3 * half * tp4};
  f[3] = {-b * b * b * onesixth * tau, b * b * dl * half * tp2, -b * dl2 * half * tp3,
          dl3 * onesixth * tp4};
}

// SecondOrderShapeFunction.cpp:179-346
void deposit2(JSink &J, int comp, double q, double o0, double o1, double n0, double n1,
              double h0, double h1, double org0, double org1, double dt) {
  Xing xs[16];
  const double ood0 = 1.0 / h0, ood1 = 1.0 / h1;
  const double oodt0 = ood0 / dt, oodt1 = ood1 / dt;
  const double Dx0 = n0 - o0, Dx1 = n1 - o1;
  const double dl0 = Dx0 * ood0, dl1 = Dx1 * ood1;
  const double cov = std::sqrt(Dx0 * Dx0 + Dx1 * Dx1);
  if (cov == 0.0) return;
  size_t n = border_crossings(xs, o0, o1, n0, n1, h0, h1, org0, org1, false);
  const double cd0 = (q * oodt1) * dl0, cd1 = (q * oodt0) * dl1;
  const double p20 = dl0 * dl0, p21 = dl1 * dl1, p30 = p20 * dl0, p31 = p21 * dl1;
  for (size_t k = 0; k + 1 < n; ++k) {
    double xi0 = xs[k].s0 * ood0, xi1 = xs[k].s1 * ood1;
    double xf0 = xs[k + 1].s0 * ood0, xf1 = xs[k + 1].s1 * ood1;
    double c0 = 0.5 * (xi0 + xf0), c1 = 0.5 * (xi1 + xf1);
    int I = (int)(long)std::floor(c0), Jj = (int)(long)std::floor(c1);
    double sg0 = xs[k + 1].s0 - xs[k].s0, sg1 = xs[k + 1].s1 - xs[k].s1;
    double tau = std::sqrt(sg0 * sg0 + sg1 * sg1) / cov;
    double a0 = I + 0.5 - xi0, a1 = Jj + 0.5 - xi1;
    double b0 = I - xi0, b1 = Jj - xi1;
    const double tp2 = tau * tau / 2;
    const double tp3 = tp2 * tau * 2 / 3;
    const double tp4 = tp2 * tp2;
    S2f s[3]; S3f t[4];
    if (comp == 0) {
      s2_factors(s, a0, dl0, p20, tau, tp2);
      s3_factors(t, b1, dl1, p21, p31, tau, tp2, tp3, tp4);
      for (int jy = 0; jy < 4; ++jy)
        for (int ix = 0; ix < 3; ++ix) J.add(I - 1 + ix, Jj - 1 + jy, cur2_term(cd0, s[ix], t[jy]));
    } else {
      s2_factors_y(s, a1, dl1, p21, tau, tp2);
      s3_factors(t, b0, dl0, p20, p30, tau, tp2, tp3, tp4);
      for (int jy = 0; jy < 3; ++jy)
        for (int ix = 0; ix < 4; ++ix) J.add(I - 1 + ix, Jj - 1 + jy, cur2_term(cd1, s[jy], t[ix]));
    }
  }
}

void deposit(int order, JSink &J, int comp, double q, double o0, double o1, double n0, double n1,
             double h0, double h1, double org0, double org1, double dt) {
  if (order == 0) deposit0(J, comp, q, o0, o1, n0, n1, h0, h1, org0, org1, dt);
  else if (order == 1) deposit1(J, comp, q, o0, o1, n0, n1, h0, h1, org0, org1, dt);
  else deposit2(J, comp, q, o0, o1, n0, n1, h0, h1, org0, org1, dt);
}

// ---------------------------------------------------------------------------
// Bend geometry, src/Bend.cpp:60-124, :126-235, :427-545, :664-799;
// cut-cell area limit src/SCBoundaryCondition.hh:131-137.
struct Bend {
  double Lb, La, w, phi, ekin, bz, R;
  double hr0, hr1, org0, org1, cen0, cen1, dlen, dwid;
  double cphi, sphi;  // cos(phi), sin(phi)
  int Nx, Ny;
};

void bend_setup(Bend &b, int Nx, int Ny, double Lb, double La, double w, double phi_deg,
                double ekin_mev, double bz) {
  const double mass = 0.511e6;
  b.Nx = Nx; b.Ny = Ny; b.Lb = Lb; b.La = La; b.w = w; b.ekin = ekin_mev * 1e6; b.bz = bz;
  if (std::abs(bz) > 1e-8) {
    b.R = std::sqrt(b.ekin * b.ekin + 2. * b.ekin * mass) / (C * std::abs(bz));
    b.phi = -bz / std::abs(bz) * std::abs(phi_deg) * PI / 180.;
  } else {
    b.R = 9999999.9;
    b.phi = 0.0;
  }
  const double cosphi = std::cos(b.phi);
  const double sinphi = std::abs(std::sin(b.phi));
  if (std::abs(bz) > 1e-8) {
    b.dlen = (Lb + La * cosphi + (b.R + 0.5 * w) * sinphi);
    b.dwid = ((b.R - 0.5 * w) * (1 - cosphi) + w + La * sinphi);
  } else {
    b.dlen = La + Lb;
    b.dwid = w;
  }
  b.hr0 = b.dlen / (Nx - 2);
  b.hr1 = b.dwid / (Ny - 2);
  if (bz <= 0.0) {
    b.org0 = 0 - b.hr0; b.org1 = (w - b.dwid) - b.hr1;
    b.cen0 = Lb; b.cen1 = 0.5 * w - b.R;
  } else {
    b.org0 = -b.hr0; b.org1 = -b.hr1;
    b.cen0 = Lb; b.cen1 = 0.5 * w + b.R;
  }
  b.cphi = std::cos(b.phi);
  b.sphi = std::sin(b.phi);
}

bool bend_inside(const Bend &b, double x0, double x1) {
  const double cosphi = b.cphi, sinphi = b.sphi;
  const double rmin_sq = (b.R - 0.5 * b.w) * (b.R - 0.5 * b.w);
  const double rmax_sq = (b.R + 0.5 * b.w) * (b.R + 0.5 * b.w);
  double D0 = x0 - b.cen0, D1 = x1 - b.cen1;
  if (D0 < 0.0) {
    if (x0 < SPACE_EPS || x1 < SPACE_EPS || x1 > b.w - SPACE_EPS) return false;
  } else if (D1 * sinphi > D0 * cosphi) {
    double l = D0 * D0 + D1 * D1;
    if (l <= rmin_sq || l >= rmax_sq) return false;
  } else {
    double p0, p1;
    if (std::abs(b.phi) > SPACE_EPS) {
      p0 = cosphi * D0 + (-sinphi) * D1 + b.cen0;
      p1 = sinphi * D0 + cosphi * D1 + b.cen1;
    } else {
      p0 = x0; p1 = x1;
    }
    if (p1 < SPACE_EPS || p1 > b.w - SPACE_EPS || p0 > b.Lb + b.La - SPACE_EPS) return false;
  }
  return true;
}

// Bend::crossBoundary; returns false where the reference's PAssert would abort.
bool bend_cross(const Bend &b, double base0, double base1, double dir0, double dir1, double &out) {
  const double cosphi = b.cphi, sinphi = b.sphi;
  const double x0 = base0 + b.org0, x1 = base1 + b.org1;
  const double D0 = x0 - b.cen0, D1 = x1 - b.cen1;
  if (D0 < 0.0) {
    double t = 99.9;
    if (x1 < b.w + SPACE_EPS && x1 + dir1 > b.w - SPACE_EPS)
      t = std::max(1.0, std::min(0.0, (b.w - x1) / dir1));
    if (x1 > -SPACE_EPS && x1 + dir1 < SPACE_EPS) t = std::min(t, -x1 / dir1);
    if (x0 > -SPACE_EPS && x0 + dir0 < SPACE_EPS) t = std::min(t, -x0 / dir0);
    out = t;
    return true;
  } else if (D1 * sinphi > D0 * cosphi) {
    double rmin_sq = (b.R - 0.5 * b.w) * (b.R - 0.5 * b.w);
    double rmax_sq = (b.R + 0.5 * b.w) * (b.R + 0.5 * b.w);
    double dist1 = D0 * D0 + D1 * D1;
    double e0 = D0 + dir0, e1 = D1 + dir1;
    double dist2 = e0 * e0 + e1 * e1;
    double a = dir0 * dir0 + dir1 * dir1;
    double bb = D0 * dir0 + D1 * dir1;
    double c = 0.0;
    if (dist1 < rmax_sq && dist2 > rmax_sq) c = (D0 * D0 + D1 * D1) - rmax_sq;
    else if (dist1 > rmin_sq && dist2 < rmin_sq) c = (D0 * D0 + D1 * D1) - rmin_sq;
    else { out = 99.9; return true; }
    double t = 99.9;
    double tau = (-bb + std::sqrt(bb * bb - a * c)) / a;
    if (std::abs(tau - 0.5) < 0.5) t = tau;
    tau = -tau - 2 * bb / a;
    if (std::abs(tau - 0.5) < 0.5) t = std::min(t, tau);
    out = t;
    return true;
  } else {
    double xr0, xr1, dr0, dr1;
    if (std::abs(b.phi) > SPACE_EPS) {
      xr0 = cosphi * D0 - sinphi * D1 + b.cen0;
      xr1 = sinphi * D0 + cosphi * D1 + b.cen1;
      dr0 = cosphi * dir0 - sinphi * dir1;
      dr1 = sinphi * dir0 + cosphi * dir1;
    } else {
      xr0 = x0; xr1 = x1; dr0 = dir0; dr1 = dir1;
    }
    double t0 = 99.9, t1 = 99.9, t2 = 99.9;
    if (std::abs(dr1) > SPACE_EPS) {
      t0 = -xr1 / dr1; if (t0 < 0.0) t0 = 99.9;
      t1 = (b.w - xr1) / dr1; if (t1 < 0.0) t1 = 99.9;
    }
    if (std::abs(dr0) > SPACE_EPS) {
      t2 = (b.Lb + b.La - xr0) / dr0; if (t2 < 0.0) t2 = 99.9;
    }
    double t = std::min(t0, std::min(t1, t2));
    if (t > 1 + SPACE_EPS && t < 1.001) t = 1.0;
    if (!(t < 1 + SPACE_EPS) || !(t >= 0)) return false;
    out = std::min(1.0, std::max(0.0, t));
    return true;
  }
}

double area_cases(int cc, double l0, double l1, double n0, double n1) {
  switch (cc) {
    case 1: return l0 * l1 / 2;
    case 2: return l0 * n1 / 2;
    case 3: return (l1 + n1) / 2;
    case 4: return n0 * l1 / 2;
    case 5: return (l0 + n0) / 2;
    case 7: return 1 - (1 - n0) * (1 - n1) / 2;
    case 8: return n0 * n1 / 2;
    case 10: return (l0 + n0) / 2;
    case 11: return 1 - (1 - l1) * (1 - n0) / 2;
    case 12: return (l1 + n1) / 2;
    case 13: return 1 - (1 - l0) * (1 - n1) / 2;
    case 14: return 1 - (1 - l0) * (1 - l1) / 2;
    default: return 0.0;
  }
}

struct CutCell { int i, j; double l0, l1, area, n0, n1; };

// Inside mask + cut-cell list (Bend::fillCellProperties minus the unused dual grid).
int bend_cells(const Bend &b, std::vector<uint8_t> &inside, std::vector<CutCell> &cells,
               std::vector<int> &inv) {
  const int Nx = b.Nx, Ny = b.Ny, G = 2, W = Nx + 2 * G;
  std::vector<char> iv((size_t)W * (Ny + 2 * G), 0);
  auto IV = [&](int i, int j) -> char & { return iv[(size_t)(j + G) * W + (i + G)]; };
  for (int cy = 0; cy < Ny; ++cy) {
    double x1 = b.org1 + cy * b.hr1;
    for (int cx = 0; cx < Nx; ++cx) {
      double x0 = b.org0 + cx * b.hr0;
      IV(cx, cy) = bend_inside(b, x0, x1) ? 1 : 0;
    }
  }
  std::vector<double> lam((size_t)W * (Ny + 2 * G) * 2, 0.0);
  auto L = [&](int i, int j, int c) -> double & { return lam[((size_t)(j + G) * W + (i + G)) * 2 + c]; };
  inside.assign((size_t)Nx * Ny, 0);
  std::vector<std::pair<int, int>> bc;
  const double h0 = b.hr0, h1 = b.hr1;
  for (int cy = 0; cy < Ny; ++cy) {
    for (int cx = 0; cx < Nx; ++cx) {
      int cc = IV(cx, cy) + (IV(cx + 1, cy) << 1) + (IV(cx, cy + 1) << 2) + (IV(cx + 1, cy + 1) << 3);
      if (cc == 15) { L(cx, cy, 0) = 1.0; L(cx, cy, 1) = 1.0; inside[(size_t)cy * Nx + cx] = 1; continue; }
      if (cc == 0) continue;
      bc.push_back({cx, cy});
      double &l0 = L(cx, cy, 0), &l1 = L(cx, cy, 1);
      bool ok = true;
      switch (cc) {
        case 1: ok &= bend_cross(b, cx * h0, cy * h1, h0, 0.0, l0); ok &= bend_cross(b, cx * h0, cy * h1, 0.0, h1, l1); break;
        case 2: ok &= bend_cross(b, (cx + 1) * h0, cy * h1, -h0, 0.0, l0); l1 = 0.0; break;
        case 3: l0 = 1.0; ok &= bend_cross(b, cx * h0, cy * h1, 0.0, h1, l1); break;
        case 4: l0 = 0.0; ok &= bend_cross(b, cx * h0, (cy + 1) * h1, 0.0, -h1, l1); break;
        case 5: ok &= bend_cross(b, cx * h0, cy * h1, h0, 0.0, l0); l1 = 1.0; break;
        case 7: l0 = 1.0; l1 = 1.0; break;
        case 8: l0 = 0.0; l1 = 0.0; break;
        case 10: ok &= bend_cross(b, (cx + 1) * h0, cy * h1, -h0, 0.0, l0); l1 = 0.0; break;
        case 11: l0 = 1.0; ok &= bend_cross(b, cx * h0, cy * h1, 0.0, h1, l1); break;
        case 12: l0 = 0.0; ok &= bend_cross(b, cx * h0, (cy + 1) * h1, 0.0, -h1, l1); break;
        case 13: ok &= bend_cross(b, cx * h0, cy * h1, h0, 0.0, l0); l1 = 1.0; break;
        case 14: ok &= bend_cross(b, (cx + 1) * h0, cy * h1, -h0, 0.0, l0);
                 ok &= bend_cross(b, cx * h0, (cy + 1) * h1, 0.0, -h1, l1); break;
        default: break;
      }
      if (!ok) return -3;
    }
  }
  cells.clear();
  inv.assign((size_t)Nx * Ny, -1);
  for (auto &p : bc) {
    int cx = p.first, cy = p.second;
    int cc = IV(cx, cy) + (IV(cx + 1, cy) << 1) + (IV(cx, cy + 1) << 2) + (IV(cx + 1, cy + 1) << 3);
    double l0 = L(cx, cy, 0), l1 = L(cx, cy, 1);
    double n0 = L(cx, cy + 1, 0), n1 = L(cx + 1, cy, 1);
    double area = area_cases(cc, l0, l1, n0, n1);
    if (!(area < 1.0 + SPACE_EPS) || !(area >= 0.0)) return -3;
    if (area < SPACE_EPS) continue;
    // SCBoundaryCondition::limitArea
    area = std::max(area, l0 / 2);
    area = std::max(area, l1 / 2);
    area = std::max(area, n0 / 2);
    area = std::max(area, n1 / 2);
    inv[(size_t)cy * Nx + cx] = (int)cells.size();
    cells.push_back({cx, cy, l0, l1, area, n0, n1});
  }
  return 0;
}

// ---------------------------------------------------------------------------
struct Sim {
  int order = 0;          // 0: IntCIC + ZerothOrder, 1: IntS1 + FirstOrder, 2: IntS2 + SecondOrder
  double dt = 0, qm = 0;  // time step, charge-to-mass ratio (PartBunch ctor, main.cpp:223)
  Bend b{};
  std::vector<uint8_t> inside;
  std::vector<CutCell> cells;
  std::vector<int> inv;
  Grid Ex, Ey, Hx, Hy;                   // static mesh (Hx, Hy = split Hz)
  Grid mEx, mEy, mHx, mHy, mJx, mJy;     // mini mesh
  int P0 = 0, P1 = 0, L0 = 0, L1 = 0;    // window position (ddim.first) and size
  double mo0 = 0, mo1 = 0;               // window origin
  std::vector<double> x, y, ox, oy, px, py, q;
  int gb[4] = {0, -1, 0, -1};            // global bounds (PartBunch::setGlobalBounds)
  bool fixed = false;                    // fixed-point deposit mode
  double fscale = 0;
  int err = 0;
  // absorbing layers at the open ends (no reference counterpart in use:
  // Bend::calculatePMLCoefficients is zeroed by TETMSolver::initMaps)
  // convolutional PML (kappa = 1): psi <- b psi + a (curl difference), the
  // difference used in the update is (curl difference + psi)
  struct Pml { int i, j; double bhx, ahx, bhy, ahy, bex, aex, bey, aey; };
  std::vector<Pml> pml;
  std::vector<double> psi;  // 4 per layer cell: Hzx, Hzy, Ex, Ey
  std::vector<int> plo, phi;  // per row: columns [lo, hi) of the regular update
};

// PartBunch::getLocalPDomain / getLocalPDomainInclOld relative to the window origin.
void pdomain(const Sim &s, bool incl_old, int out[4]) {
  size_t n = s.x.size();
  if (n == 0) {
    if (incl_old) { out[0] = 0; out[1] = -1; out[2] = 0; out[3] = -1; return; }
    double r[2] = {0.0, 0.0};
    out[0] = (int)std::floor((r[0] - s.mo0) / s.b.hr0); out[1] = (int)std::floor((r[0] - s.mo0) / s.b.hr0);
    out[2] = (int)std::floor((r[1] - s.mo1) / s.b.hr1); out[3] = (int)std::floor((r[1] - s.mo1) / s.b.hr1);
    return;
  }
  double mn0 = s.x[0], mx0 = s.x[0], mn1 = s.y[0], mx1 = s.y[0];
  for (size_t i = 0; i < n; ++i) {
    if (s.x[i] < mn0) mn0 = s.x[i];
    if (incl_old && s.ox[i] < mn0) mn0 = s.ox[i];
    if (s.x[i] > mx0) mx0 = s.x[i];
    if (incl_old && s.ox[i] > mx0) mx0 = s.ox[i];
    if (s.y[i] < mn1) mn1 = s.y[i];
    if (incl_old && s.oy[i] < mn1) mn1 = s.oy[i];
    if (s.y[i] > mx1) mx1 = s.y[i];
    if (incl_old && s.oy[i] > mx1) mx1 = s.oy[i];
  }
  out[0] = (int)std::floor((mn0 - s.mo0) / s.b.hr0);
  out[1] = (int)std::floor((mx0 - s.mo0) / s.b.hr0);
  out[2] = (int)std::floor((mn1 - s.mo1) / s.b.hr1);
  out[3] = (int)std::floor((mx1 - s.mo1) / s.b.hr1);
}

// PartBunch::drift_particles, PartBunch.cpp:179-187
void drift(Sim &s, double dt) {
  double full = dt * C;
  for (size_t i = 0; i < s.x.size(); ++i) {
    double r = (double)q_rsqrt((float)(1 + (s.px[i] * s.px[i] + s.py[i] * s.py[i])));
    s.x[i] += full * s.px[i] * r;
    s.y[i] += full * s.py[i] * r;
  }
}

// margins: ShapeFunction getExtraMarginEdge / getExtraMarginCell per order
void margins(int order, int edge[4], int cell[2]) {
  if (order == 0) { int e[4] = {-1, 1, 0, 1}; std::memcpy(edge, e, sizeof(e)); cell[0] = -1; cell[1] = 1; }
  else if (order == 1) { int e[4] = {-1, 1, -1, 2}; std::memcpy(edge, e, sizeof(e)); cell[0] = -1; cell[1] = 1; }
  else { int e[4] = {-2, 2, -1, 2}; std::memcpy(edge, e, sizeof(e)); cell[0] = -2; cell[1] = 2; }
}

// PartBunch::push_particles, PartBunch.cpp:215-519 (one rank; deposit of
// Jcomp over all particles once).
void push(Sim &s, int jcomp) {
  const size_t n = s.x.size();
  const double half = 0.5 * s.dt * C;
  for (size_t i = 0; i < n; ++i) {
    s.ox[i] = s.x[i]; s.oy[i] = s.y[i];
    double r = (double)q_rsqrt((float)(1.0 + (s.px[i] * s.px[i] + s.py[i] * s.py[i])));
    s.x[i] += half * s.px[i] * r;
    s.y[i] += half * s.py[i] * r;
  }
  int lp[4];
  pdomain(s, false, lp);
  int em[4], cm[2];
  margins(s.order, em, cm);
  const double h0 = s.b.hr0, h1 = s.b.hr1;
  // getFields, PartBunch.cpp:957-1111: patch origins and the absolute index of
  // relative (0,0) for Hz, Ex, Ey.
  const double po0 = s.mo0 + lp[0] * h0, po1 = s.mo1 + lp[2] * h1;
  const double hzo0 = po0 + cm[0] * h0, hzo1 = po1 + cm[0] * h1;
  const double exo0 = po0 + em[0] * h0, exo1 = po1 + em[2] * h1;
  const double eyo0 = po0 + em[2] * h0, eyo1 = po1 + em[0] * h1;
  const int hzI = lp[0] + cm[0], hzJ = lp[2] + cm[0];
  const int exI = lp[0] + em[0], exJ = lp[2] + em[2];
  const int eyI = lp[0] + em[2], eyJ = lp[2] + em[0];
  // Dense copies of the window (incl. guards) so the patch reads are plain.
  const int W0 = s.L0 + 2, W1 = s.L1 + 2;
  std::vector<double> hz((size_t)W0 * W1), ex((size_t)W0 * W1), ey((size_t)W0 * W1);
  for (int j = -1; j <= s.L1; ++j)
    for (int i = -1; i <= s.L0; ++i) {
      size_t k = (size_t)(j + 1) * W0 + (i + 1);
      hz[k] = s.mHx.at(i, j) + s.mHy.at(i, j);
      ex[k] = s.mEx.at(i, j);
      ey[k] = s.mEy.at(i, j);
    }
  // A patch whose relative (0,0) is absolute (I0, J0) reads the dense window at +1 guard.
  auto mk = [&](const std::vector<double> &a, int I0, int J0, double o0, double o1) {
    Patch p;
    p.p = a.data() + (ptrdiff_t)(J0 + 1) * W0 + (I0 + 1);
    p.nx = W0; p.ny = W1; p.o0 = o0; p.o1 = o1; p.h0 = h0; p.h1 = h1;
    return p;
  };
  Patch pex = mk(ex, exI, exJ, exo0, exo1), pey = mk(ey, eyI, eyJ, eyo0, eyo1), phz = mk(hz, hzI, hzJ, hzo0, hzo1);
  // Bend::getExternalField, Bend.cpp:865-907
  const double chh = std::cos(0.5 * s.b.phi), shh = std::sin(0.5 * s.b.phi);
  const double hw = 0.5 * s.b.w, bw = 2 * s.b.R * std::abs(shh);
  const double fact1 = half * s.qm, fact2 = fact1 * C;
  for (size_t i = 0; i < n; ++i) {
    double E0 = gather_edge(s.order, pex, s.x[i], s.y[i], 0);
    double E1 = gather_edge(s.order, pey, s.x[i], s.y[i], 1);
    double Hf = gather_cell(s.order, phz, s.x[i], s.y[i]);
    double D0 = s.x[i] - s.b.Lb, D1 = s.y[i] - hw;
    double dist = chh * D0 - shh * D1;
    double bext = (dist > 0.0 && dist < bw) ? s.b.bz : 0.0;
    double B = MU0 * Hf + 0.5 * bext;
    double k0 = fact1 * E0, k1 = fact1 * E1;
    double u0 = s.px[i] + k0, u1 = s.py[i] + k1;
    double a = fact2 * B * (double)q_rsqrt((float)(1.0 + (u0 * u0 + u1 * u1)));
    double s0 = u0 + a * u1, s1 = u1 + a * (-u0);
    double tmp = 1.0 + a * a;
    u0 = ((1.0 + a * a) * s0 + a * s1) / tmp;
    u1 = ((1.0 + a * a) * s1 - a * s0) / tmp;
    s.px[i] = u0 + k0; s.py[i] = u1 + k1;
    double r = (double)q_rsqrt((float)(1.0 + (s.px[i] * s.px[i] + s.py[i] * s.py[i])));
    s.x[i] += half * s.px[i] * r;
    s.y[i] += half * s.py[i] * r;
  }
  // Current deposit into the window (ShapeFunction getCurrentDensity{Base}{X,Y}).
  Grid &J = jcomp == 0 ? s.mJx : s.mJy;
  pdomain(s, true, s.gb);
  for (int jj = 0; jj < s.L1; ++jj)
    for (int ii = 0; ii < s.L0; ++ii) J.at(ii, jj) = 0.0;
  if (n == 0) return;
  // The patch is gPDom + margin, clipped to the local domain [0, L-1].
  const int cur[4] = {-1, 1, -1, 2};  // getExtraMarginCurrent for orders 1 and 2
  int lo0, hi0, lo1, hi1;
  if (s.order == 0) {
    // ZerothOrder margin (Index(0,0), Index(0,1)); Y deposit swaps the axes.
    int m[4] = {0, 0, 0, 1};
    int a = jcomp == 0 ? 0 : 2, bq = jcomp == 0 ? 2 : 0;
    lo0 = s.gb[0] + m[a]; hi0 = s.gb[1] + m[a + 1]; lo1 = s.gb[2] + m[bq]; hi1 = s.gb[3] + m[bq + 1];
  } else {
    int a = jcomp == 0 ? 0 : 2, bq = jcomp == 0 ? 2 : 0;
    lo0 = s.gb[0] + cur[a]; hi0 = s.gb[1] + cur[a + 1]; lo1 = s.gb[2] + cur[bq]; hi1 = s.gb[3] + cur[bq + 1];
  }
  Grid tmp; tmp.init(s.L0, s.L1, 3);
  JSink sink{&tmp, s.fixed, s.fscale, {}, 0, 0};
  if (s.fixed) sink.acc.assign(tmp.v.size(), 0);
  for (size_t i = 0; i < n; ++i)
    deposit(s.order, sink, jcomp, s.q[i], s.ox[i], s.oy[i], s.x[i], s.y[i], h0, h1, s.mo0, s.mo1, s.dt);
  if (s.fixed)
    for (size_t k = 0; k < tmp.v.size(); ++k) tmp.v[k] = (double)sink.acc[k] / s.fscale;
  lo0 = std::max(lo0, 0); hi0 = std::min(hi0, s.L0 - 1);
  lo1 = std::max(lo1, 0); hi1 = std::min(hi1, s.L1 - 1);
  for (int jj = lo1; jj <= hi1; ++jj)
    for (int ii = lo0; ii <= hi0; ++ii) J.at(ii, jj) = tmp.at(ii, jj);
}

// Communicator::exchangeBoundaries, Communicator.hh:575-876 (one rank).
// which: 0 = H (sum split 1/2 1/2), 1 = Ex, 2 = Ey.  All values are read first.
void exchange(Sim &s, int which) {
  struct W { bool to_window; int i, j; double v; };
  std::vector<W> todo;
  const int P0 = s.P0, P1 = s.P1, L0 = s.L0, L1 = s.L1;
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  auto sval = [&](int i, int j) {
    if (which == 0) return s.Hx.at(i, j) + s.Hy.at(i, j);
    return which == 1 ? s.Ex.at(i, j) : s.Ey.at(i, j);
  };
  auto mval = [&](int i, int j) {
    if (which == 0) return s.mHx.at(i, j) + s.mHy.at(i, j);
    return which == 1 ? s.mEx.at(i, j) : s.mEy.at(i, j);
  };
  // HFieldToDouble / ExFieldToDouble / EyFieldToDouble::sides (Communicator.cpp:640-642)
  unsigned sides = which == 0 ? (1u << 4 | 1u << 5 | 1u << 2 | 1u << 3)
                 : which == 1 ? (1u << 7 | 1u << 1) : (1u << 6 | 1u << 0);
  for (int side = 0; side < 8; ++side) {
    if (!(sides & (1u << side))) continue;
    const int d = side % 2;
    if (side < 4) {
      // window boundary strip -> static mesh (clipped to the static domain +-1)
      int i0 = 0, i1 = L0 - 1, j0 = 0, j1 = L1 - 1;
      if (d == 0) i0 = i1 = (side < 2 ? 0 : L0 - 1);
      else j0 = j1 = (side < 2 ? 0 : L1 - 1);
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) {
          const int si = i + P0, sj = j + P1;
          if (si < -1 || si > Nx || sj < -1 || sj > Ny) continue;
          todo.push_back({false, si, sj, mval(i, j)});
        }
    } else {
      // static ring just outside the window -> window guard layer
      int i0 = P0 - 1, i1 = P0 + L0, j0 = P1 - 1, j1 = P1 + L1;
      if (d == 0) i0 = i1 = (side < 6 ? P0 - 1 : P0 + L0);
      else j0 = j1 = (side < 6 ? P1 - 1 : P1 + L1);
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) {
          if (i < 0 || i >= Nx || j < 0 || j >= Ny) continue;
          todo.push_back({true, i - P0, j - P1, sval(i, j)});
        }
    }
  }
  for (auto &t : todo) {
    if (which == 0) {
      Grid &a = t.to_window ? s.mHx : s.Hx, &b = t.to_window ? s.mHy : s.Hy;
      a.at(t.i, t.j) = 0.5 * t.v; b.at(t.i, t.j) = 0.5 * t.v;
    } else if (which == 1) {
      (t.to_window ? s.mEx : s.Ex).at(t.i, t.j) = t.v;
    } else {
      (t.to_window ? s.mEy : s.Ey).at(t.i, t.j) = t.v;
    }
  }
}

// Convolutional PML (kappa = 1) of thickness W at the two open ends of the
// pipe, restated independently of the GPU library: the entry plane x = 0
// (axis +x) and the end plane of the second straight section (the
// centreline's end after the arc of radius R and angle |phi| about the bend
// centre and length_after along the outgoing axis).  Each layer stops kPmlGap
// cells before its end plane, so that no layer cell neighbours the conformal
// cut cells of a slanted end wall.  sigma(depth) = smax (depth / W)^m, split
// along the axis into sx, sy.
constexpr double kPmlGap = 2.0;
void pml_sigma(const Bend &b, double W, int m, double smax, double x, double y, double &sx, double &sy) {
  sx = 0.0; sy = 0.0;
  const double gap = kPmlGap * b.hr0;
  const double sin_ = x - gap;  // distance from the entry plane, past the gap
  if (sin_ >= 0.0 && sin_ < W) sx += smax * std::pow((W - sin_) / W, m);
  const double ph = std::fabs(b.phi);
  const double ry = 0.5 * b.w - b.cen1;
  const double sg = ry > 0.0 ? -1.0 : 1.0;
  const double t0 = std::cos(ph), t1 = sg * std::sin(ph);
  const double e0 = b.cen0 + b.R * std::sin(ph) + b.La * t0;
  const double e1 = b.cen1 - sg * b.R * std::cos(ph) + b.La * t1;
  const double sout = (e0 - x) * t0 + (e1 - y) * t1 - gap;
  if (sout >= 0.0 && sout < W) {
    const double v = smax * std::pow((W - sout) / W, m);
    sx += v * std::fabs(t0);
    sy += v * std::fabs(t1);
  }
}

// CPML recursion over the update interval dt': b = exp(-sigma dt'/eps0), a = b - 1
void pml_coef(double sigma, double dtp, double &b, double &a) {
  if (!(sigma > 0.0)) { b = 1.0; a = 0.0; return; }
  b = std::exp(-sigma * dtp / EPS0);
  a = b - 1.0;
}

// Static + window H half update (TETMSolver.hh:142-149) followed by the
// exchange and the cut-cell correction (:154-163).
void half_h(Sim &s) {
  const double h0 = s.b.hr0, h1 = s.b.hr1;
  const double etax = C * s.dt / h0, etay = C * s.dt / h1;
  const double Z0 = std::sqrt(MU0 / EPS0);
  const double cx = 0.5 * etax / Z0, cy = 0.5 * etay / Z0;
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  const bool layers = !s.plo.empty();
  for (int j = 0; j < Ny; ++j)
    for (int i = 0; i < Nx; ++i) {
      if (!s.inside[(size_t)j * Nx + i]) continue;
      if (layers && (i < s.plo[j] || i >= s.phi[j])) continue;
      s.Hx.at(i, j) = s.Hx.at(i, j) - cx * (s.Ey.at(i + 1, j) - s.Ey.at(i, j));
      s.Hy.at(i, j) = s.Hy.at(i, j) + cy * (s.Ex.at(i, j + 1) - s.Ex.at(i, j));
    }
  for (size_t k = 0; k < s.pml.size(); ++k) {
    const Sim::Pml &c = s.pml[k];
    double *ps = &s.psi[4 * k];
    const double dey = s.Ey.at(c.i + 1, c.j) - s.Ey.at(c.i, c.j);
    const double dex = s.Ex.at(c.i, c.j + 1) - s.Ex.at(c.i, c.j);
    ps[0] = c.bhx * ps[0] + c.ahx * dey;
    ps[1] = c.bhy * ps[1] + c.ahy * dex;
    s.Hx.at(c.i, c.j) = s.Hx.at(c.i, c.j) - cx * (dey + ps[0]);
    s.Hy.at(c.i, c.j) = s.Hy.at(c.i, c.j) + cy * (dex + ps[1]);
  }
  for (int j = 0; j < s.L1; ++j)
    for (int i = 0; i < s.L0; ++i) {
      s.mHx.at(i, j) = s.mHx.at(i, j) - cx * (s.mEy.at(i + 1, j) - s.mEy.at(i, j));
      s.mHy.at(i, j) = s.mHy.at(i, j) + cy * (s.mEx.at(i, j + 1) - s.mEx.at(i, j));
    }
  exchange(s, 0);
  // SCBoundaryCondition::updateHz + TETMSolver::updateHz (TETMSolver.cpp:87-103)
  const double ex_ = s.dt / (h0 * MU0), ey_ = s.dt / (h1 * MU0);
  for (auto &c : s.cells) {
    double u0 = -0.5 * ex_ * (c.n1 * s.Ey.at(c.i + 1, c.j) - c.l1 * s.Ey.at(c.i, c.j)) / c.area;
    double u1 = +0.5 * ey_ * (c.n0 * s.Ex.at(c.i, c.j + 1) - c.l0 * s.Ex.at(c.i, c.j)) / c.area;
    s.Hx.at(c.i, c.j) += u0;
    s.Hy.at(c.i, c.j) += u1;
  }
}

// TETMSolver.hh:165-184 (Ex) and :241-261 (Ey).  The static J is identically
// zero in the reference loop (main.cpp:388, :494), so it enters as 0.0.
void update_e(Sim &s, int comp) {
  const double h0 = s.b.hr0, h1 = s.b.hr1;
  const double Z0 = std::sqrt(MU0 / EPS0);
  const double dteps = C * s.dt * Z0;
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  const double zeroJ = 0.0;
  if (comp == 0) {
    const double k = (C * s.dt / h1) * Z0;
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        if (!s.inside[(size_t)j * Nx + i]) continue;
        if (!s.plo.empty() && (i < s.plo[j] || i >= s.phi[j])) continue;
        s.Ex.at(i, j) = s.Ex.at(i, j) + (k * (s.Hx.at(i, j) - s.Hx.at(i, j - 1) + s.Hy.at(i, j) - s.Hy.at(i, j - 1)) - dteps * zeroJ);
      }
    for (size_t q = 0; q < s.pml.size(); ++q) {
      const Sim::Pml &c = s.pml[q];
      double &ps = s.psi[4 * q + 2];
      const double dh = s.Hx.at(c.i, c.j) - s.Hx.at(c.i, c.j - 1) + s.Hy.at(c.i, c.j) - s.Hy.at(c.i, c.j - 1);
      ps = c.bex * ps + c.aex * dh;
      s.Ex.at(c.i, c.j) = s.Ex.at(c.i, c.j) + (k * (dh + ps) - dteps * zeroJ);
    }
    for (int j = 0; j < s.L1; ++j)
      for (int i = 0; i < s.L0; ++i)
        s.mEx.at(i, j) = s.mEx.at(i, j) + (k * (s.mHx.at(i, j) - s.mHx.at(i, j - 1) + s.mHy.at(i, j) - s.mHy.at(i, j - 1)) - dteps * s.mJx.at(i, j));
    exchange(s, 1);
    const double de = s.dt / EPS0;
    for (auto &c : s.cells) {
      if (c.area < MINAREA) continue;
      if (c.l0 > SPACE_EPS) {
        double u0 = (s.Hx.at(c.i, c.j) - s.Hx.at(c.i, c.j - 1)) / h1;
        double u1 = (s.Hy.at(c.i, c.j) - s.Hy.at(c.i, c.j - 1)) / h1;
        s.Ex.at(c.i, c.j) += de * (u0 + u1 - zeroJ);
      }
    }
  } else {
    const double k = (C * s.dt / h0) * Z0;
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        if (!s.inside[(size_t)j * Nx + i]) continue;
        if (!s.plo.empty() && (i < s.plo[j] || i >= s.phi[j])) continue;
        s.Ey.at(i, j) = s.Ey.at(i, j) - (k * (s.Hx.at(i, j) - s.Hx.at(i - 1, j) + s.Hy.at(i, j) - s.Hy.at(i - 1, j)) + dteps * zeroJ);
      }
    for (size_t q = 0; q < s.pml.size(); ++q) {
      const Sim::Pml &c = s.pml[q];
      double &ps = s.psi[4 * q + 3];
      const double dh = s.Hx.at(c.i, c.j) - s.Hx.at(c.i - 1, c.j) + s.Hy.at(c.i, c.j) - s.Hy.at(c.i - 1, c.j);
      ps = c.bey * ps + c.aey * dh;
      s.Ey.at(c.i, c.j) = s.Ey.at(c.i, c.j) - (k * (dh + ps) + dteps * zeroJ);
    }
    for (int j = 0; j < s.L1; ++j)
      for (int i = 0; i < s.L0; ++i)
        s.mEy.at(i, j) = s.mEy.at(i, j) - (k * (s.mHx.at(i, j) - s.mHx.at(i - 1, j) + s.mHy.at(i, j) - s.mHy.at(i - 1, j)) + dteps * s.mJy.at(i, j));
    exchange(s, 2);
    const double de = s.dt / EPS0;
    for (auto &c : s.cells) {
      if (c.area < MINAREA) continue;
      if (c.l1 > SPACE_EPS) {
        double u0 = -(s.Hx.at(c.i, c.j) - s.Hx.at(c.i - 1, c.j)) / h0;
        double u1 = -(s.Hy.at(c.i, c.j) - s.Hy.at(c.i - 1, c.j)) / h0;
        s.Ey.at(c.i, c.j) += de * (u0 + u1 - zeroJ);
      }
    }
  }
}

// main.cpp:562-652 moveMesh + Communicator.cpp:123-642 exchangeBoundariesMovingMesh.
int move_window(Sim &s) {
  const int L[2] = {s.L0, s.L1};
  int ideal[2][2];
  for (int d = 0; d < 2; ++d) {
    int len = s.gb[2 * d + 1] - s.gb[2 * d] + 1;
    if (len >= L[d]) return -5;  // PAssert(fits)
    unsigned diff = (unsigned)(L[d] - len);
    unsigned up = (unsigned)std::floor(diff / 2.0);
    unsigned lo = diff - up;
    ideal[d][0] = (int)lo - 1;
    ideal[d][1] = L[d] - (int)up - 2;
  }
  int moveI = s.gb[1] - ideal[0][1] - 1;
  int dj = s.gb[3] - ideal[1][1] - 1;
  int maxJ = std::max(0, dj), minJ = std::min(0, dj);
  if (moveI < 0 || moveI > 1 || dj < -1 || dj > 1) return -6;
  int m1 = minJ + maxJ;
  // In-place shift (reads always run ahead of writes for these orders).
  int i0 = -moveI, i1 = s.L0 - 1;
  int j0 = -maxJ, j1 = s.L1 - 1 - minJ;
  if (m1 == 0) { j0 -= 1; j1 += 1; }
  Grid *fs[6] = {&s.mEx, &s.mEy, &s.mHx, &s.mHy, &s.mJx, &s.mJy};
  auto mv = [&](int j) {
    for (int i = i0; i <= i1; ++i)
      for (Grid *g : fs) g->at(i, j) = g->at(i + moveI, j + m1);
  };
  if (minJ == -1) { for (int j = j1; j >= j0; --j) mv(j); }
  else { for (int j = j0; j <= j1; ++j) mv(j); }
  s.P0 += moveI; s.P1 += m1;
  s.mo0 += moveI * s.b.hr0;
  s.mo1 += m1 * s.b.hr1;
  // Moving-mesh strip exchange: layer lists in embedded (E2S) or surrounding (S2E) coordinates.
  struct Lay { int type; int a0, a1, b0, b1; };  // type 0..2 E2S (Hz, Ex, Ey), 3..5 S2E
  std::vector<Lay> lays[6];
  const int Ld0 = s.L0 - 1, Ld1 = s.L1 - 1, P0 = s.P0, P1 = s.P1;
  const int mv0 = moveI, mvv = m1;
  if (mv0 == 1) {
    lays[0].push_back({0, -mv0, -mv0, 0 - mvv, Ld1 - mvv - 1});
    lays[1].push_back({1, -mv0, -mv0, 0 - mvv + 1, Ld1 - mvv});
    lays[2].push_back({2, 1 - mv0, 1 - mv0, 0 - mvv, Ld1 - mvv});
    lays[3].push_back({3, Ld0 + P0, Ld0 + P0, P1, Ld1 + P1});
    lays[4].push_back({4, Ld0 + P0, Ld0 + P0, P1, Ld1 + P1 + 1});
    lays[5].push_back({5, Ld0 + P0 + 1, Ld0 + P0 + 1, P1, Ld1 + P1});
  }
  if (mvv == 1) {
    lays[0].push_back({0, 0 - mv0, Ld0 - 1 - mv0, -mvv, -mvv});
    lays[1].push_back({1, 0 - mv0, Ld0 - mv0, 1 - mvv, 1 - mvv});
    lays[2].push_back({2, 1 - mv0, Ld0 - mv0, -mvv, -mvv});
    lays[3].push_back({3, P0, Ld0 + P0, Ld1 + P1, Ld1 + P1});
    lays[4].push_back({4, P0, Ld0 + P0, Ld1 + 1 + P1, Ld1 + 1 + P1});
    lays[5].push_back({5, P0, Ld0 + P0 + 1, Ld1 + P1, Ld1 + P1});
  } else if (mvv == -1) {
    lays[0].push_back({0, 0 - mv0, Ld0 - mv0 - 1, Ld1 - 1 - mvv, Ld1 - mvv - 1});
    lays[1].push_back({1, 0 - mv0, Ld0 - mv0, Ld1 - mvv, Ld1 - mvv});
    lays[2].push_back({2, 0 - mv0 + 1, Ld0 - mv0, Ld1 - mvv, Ld1 - mvv});
    lays[3].push_back({3, P0, Ld0 + P0, 0 - 1 + P1, 0 - 1 + P1});
    lays[4].push_back({4, P0, Ld0 + P0, 0 + P1, 0 + P1});
    lays[5].push_back({5, P0, Ld0 + P0 + 1, 0 + P1, 0 + P1});
  }
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  struct W { int type, i, j; double v; };
  std::vector<W> todo;
  for (int t = 0; t < 6; ++t)
    for (auto &ly : lays[t]) {
      if (t < 3) {
        // embedded extended domain [-1, L] clipped, then to the surrounding domain
        int a0 = std::max(ly.a0, -1), a1 = std::min(ly.a1, s.L0), b0 = std::max(ly.b0, -1), b1 = std::min(ly.b1, s.L1);
        a0 = std::max(a0, 0 - P0); a1 = std::min(a1, Nx - 1 - P0);
        b0 = std::max(b0, 0 - P1); b1 = std::min(b1, Ny - 1 - P1);
        for (int j = b0; j <= b1; ++j)
          for (int i = a0; i <= a1; ++i) {
            double v = t == 0 ? s.mHx.at(i, j) + s.mHy.at(i, j) : t == 1 ? s.mEx.at(i, j) : s.mEy.at(i, j);
            todo.push_back({t, i + P0, j + P1, v});
          }
      } else {
        int a0 = std::max(ly.a0, 0), a1 = std::min(ly.a1, Nx - 1), b0 = std::max(ly.b0, 0), b1 = std::min(ly.b1, Ny - 1);
        a0 = std::max(a0, -1 + P0); a1 = std::min(a1, s.L0 + P0);
        b0 = std::max(b0, -1 + P1); b1 = std::min(b1, s.L1 + P1);
        for (int j = b0; j <= b1; ++j)
          for (int i = a0; i <= a1; ++i) {
            double v = t == 3 ? s.Hx.at(i, j) + s.Hy.at(i, j) : t == 4 ? s.Ex.at(i, j) : s.Ey.at(i, j);
            todo.push_back({t, i - P0, j - P1, v});
          }
      }
    }
  for (auto &w : todo) {
    switch (w.type) {
      case 0: s.Hx.at(w.i, w.j) = 0.5 * w.v; s.Hy.at(w.i, w.j) = 0.5 * w.v; break;
      case 1: s.Ex.at(w.i, w.j) = w.v; break;
      case 2: s.Ey.at(w.i, w.j) = w.v; break;
      case 3: s.mHx.at(w.i, w.j) = 0.5 * w.v; s.mHy.at(w.i, w.j) = 0.5 * w.v; break;
      case 4: s.mEx.at(w.i, w.j) = w.v; break;
      case 5: s.mEy.at(w.i, w.j) = w.v; break;
    }
  }
  return 0;
}

// Vertex charge shape of one particle (getChargeDensityImpl /
// getChargeDensityDiffImpl of Zeroth/First/SecondOrderShapeFunction):
// add(i, j, sg * w) for every vertex weight w of charge qq at (X, Y).
template <class Add>
void charge_shape(int order, double X, double Y, double qq, double sg, double org0, double org1, double h0,
                  double h1, Add &&add) {
  const double onesixth = 1.0 / 6.0;
  if (order == 0) {  // ZerothOrderShapeFunction.cpp:355-366
    double xi0 = (X - org0) / h0, xi1 = (Y - org1) / h1;
    int I = (int)std::floor(xi0), J = (int)std::floor(xi1);
    double t0 = xi0 - I, t1 = xi1 - J;
    add(I, J, sg * ((1.0 - t0) * (1.0 - t1) * qq));
    add(I + 1, J, sg * (t0 * (1.0 - t1) * qq));
    add(I, J + 1, sg * ((1.0 - t0) * t1 * qq));
    add(I + 1, J + 1, sg * (t0 * t1 * qq));
  } else if (order == 1) {  // FirstOrderShapeFunction.cpp:391-416
    double n0 = (X - org0) / h0, n1 = (Y - org1) / h1;
    int I = (int)std::floor(n0 + 0.5), J = (int)std::floor(n1 + 0.5);
    double a = n0 - I, b = n1 - J;
    double sxm = qq * (0.5 - a) * (0.5 - a) * 0.5, sxp = qq * (0.5 + a) * (0.5 + a) * 0.5;
    double sx = qq - sxm - sxp;
    double sym = (0.5 - b) * (0.5 - b) * 0.5, syp = (0.5 + b) * (0.5 + b) * 0.5;
    double sy = 1.0 - sym - syp;
    double wx[3] = {sxm, sx, sxp}, wy[3] = {sym, sy, syp};
    for (int bb = 0; bb < 3; ++bb)
      for (int aa = 0; aa < 3; ++aa) add(I - 1 + aa, J - 1 + bb, sg * (wx[aa] * wy[bb]));
  } else {  // SecondOrderShapeFunction.cpp:408-441
    double n0 = (X - org0) / h0, n1 = (Y - org1) / h1;
    int I = (int)std::floor(n0), J = (int)std::floor(n1);
    double a = n0 - I, b = n1 - J;
    auto p3 = [](double v) { return v * v * v; };
    double wx[4] = {onesixth * p3(1.0 - a), onesixth * (4.0 - 3.0 * a * a * (2.0 - a)),
                    onesixth * (4.0 - 3.0 * (1.0 - a) * (1.0 - a) * (1.0 + a)), onesixth * p3(a)};
    double wy[4] = {onesixth * p3(1.0 - b), onesixth * (4.0 - 3.0 * b * b * (2.0 - b)),
                    onesixth * (4.0 - 3.0 * (1.0 - b) * (1.0 - b) * (1.0 + b)), onesixth * p3(b)};
    for (int bb = 0; bb < 4; ++bb)
      for (int aa = 0; aa < 4; ++aa) add(I - 1 + aa, J - 1 + bb, sg * (qq * wx[aa] * wy[bb]));
  }
}

// ---- initial fields: boosted electrostatic solve ---------------------------
// PoissonSolver::computeField (PoissonSolver.cpp:85-201) with the matrix of
// cutoffStencil (:678-766).  The reference solves with Trilinos ML-preconditioned
// BlockCG; here the same matrix is solved by CG with a y-line Jacobi
// preconditioner (an independent method, so that it checks the GPU solver).
struct PoissonSys {
  int Nx = 0, Ny = 0;
  double EW = 0, NS = 0, D = 0;
  std::vector<uint8_t> good, act;  // good: inside or cut area > 0.5; act: good and i < maxX
};

void poisson_setup(const Sim &s, double gamma, PoissonSys &p) {
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  p.Nx = Nx; p.Ny = Ny;
  const double hr0 = s.b.hr0 * gamma, hr1 = s.b.hr1;  // PoissonSolver ctor, :70-71
  p.EW = -1 / (hr0 * hr0);
  p.NS = -1 / (hr1 * hr1);
  p.D = -2 * (p.EW + p.NS);
  const long maxX = (long)(size_t)(s.b.Lb / s.b.hr0);  // Bend::getLengthStraightSection
  p.good.assign((size_t)Nx * Ny, 0);
  p.act.assign((size_t)Nx * Ny, 0);
  for (int j = 0; j < Ny; ++j)
    for (int i = 0; i < Nx; ++i) {
      const size_t k = (size_t)j * Nx + i;
      const int c = s.inv[k];
      p.good[k] = s.inside[k] || (c > -1 && s.cells[c].area > 0.5);
      p.act[k] = p.good[k] && i < maxX;
    }
}

// Out-of-domain neighbours count as not good (Dirichlet zero).
inline bool pgood(const PoissonSys &p, int i, int j) {
  return i >= 0 && j >= 0 && i < p.Nx && j < p.Ny && p.good[(size_t)j * p.Nx + i];
}
inline bool pact(const PoissonSys &p, int i, int j) {
  return i >= 0 && j >= 0 && i < p.Nx && j < p.Ny && p.act[(size_t)j * p.Nx + i];
}

// Solve A phi = b.  Rows that are not active are identity rows, so
// phi = b there; their values move to the right-hand side of the active rows
// they couple to.  x holds the initial guess on entry (active entries used).
// Returns the iteration count; relres receives ||r|| / ||b_active||.
int poisson_solve(const PoissonSys &p, const std::vector<double> &b, std::vector<double> &x, double tol,
                  int maxit, double *relres) {
  const int Nx = p.Nx, Ny = p.Ny;
  const size_t n = (size_t)Nx * Ny;
  std::vector<double> f(n, 0.0), r(n, 0.0), z(n, 0.0), d(n, 0.0), q(n, 0.0);
  for (int j = 0; j < Ny; ++j)
    for (int i = 0; i < Nx; ++i) {
      const size_t k = (size_t)j * Nx + i;
      if (!p.act[k]) { x[k] = b[k]; continue; }
      double v = b[k];
      const int di[4] = {0, -1, 1, 0}, dj[4] = {-1, 0, 0, 1};
      for (int t = 0; t < 4; ++t) {
        const int a = i + di[t], c = j + dj[t];
        if (pgood(p, a, c) && !pact(p, a, c)) v -= (dj[t] ? p.NS : p.EW) * b[(size_t)c * Nx + a];
      }
      f[k] = v;
    }
  auto apply = [&](const std::vector<double> &u, std::vector<double> &out) {
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        const size_t k = (size_t)j * Nx + i;
        if (!p.act[k]) { out[k] = 0.0; continue; }
        double v = p.D * u[k];
        if (pact(p, i - 1, j)) v += p.EW * u[k - 1];
        if (pact(p, i + 1, j)) v += p.EW * u[k + 1];
        if (pact(p, i, j - 1)) v += p.NS * u[k - Nx];
        if (pact(p, i, j + 1)) v += p.NS * u[k + Nx];
        out[k] = v;
      }
  };
  // y-line Jacobi: one tridiagonal solve per column (Thomas algorithm)
  std::vector<double> cp(Ny), dp(Ny);
  auto precond = [&](const std::vector<double> &rr, std::vector<double> &zz) {
    for (int i = 0; i < Nx; ++i) {
      double cprev = 0.0, dprev = 0.0;
      for (int j = 0; j < Ny; ++j) {
        const size_t k = (size_t)j * Nx + i;
        if (!p.act[k]) { cp[j] = 0.0; dp[j] = 0.0; cprev = 0.0; dprev = 0.0; continue; }
        const double a = pact(p, i, j - 1) ? p.NS : 0.0, c = pact(p, i, j + 1) ? p.NS : 0.0;
        const double m = p.D - a * cprev;
        cp[j] = c / m;
        dp[j] = (rr[k] - a * dprev) / m;
        cprev = cp[j]; dprev = dp[j];
      }
      double u = 0.0;
      for (int j = Ny - 1; j >= 0; --j) {
        u = dp[j] - cp[j] * u;
        zz[(size_t)j * Nx + i] = p.act[(size_t)j * Nx + i] ? u : 0.0;
      }
    }
  };
  auto dot = [&](const std::vector<double> &a, const std::vector<double> &c) {
    double s = 0.0;
    for (size_t k = 0; k < n; ++k) s += a[k] * c[k];
    return s;
  };
  std::vector<double> u(n, 0.0);
  for (size_t k = 0; k < n; ++k) u[k] = p.act[k] ? x[k] : 0.0;
  apply(u, q);
  for (size_t k = 0; k < n; ++k) r[k] = f[k] - q[k];
  const double bn = std::sqrt(dot(f, f));
  int it = 0;
  double rn = std::sqrt(dot(r, r));
  if (bn == 0.0) {
    for (size_t k = 0; k < n; ++k) if (p.act[k]) x[k] = 0.0;
    *relres = 0.0;
    return 0;
  }
  precond(r, z);
  d = z;
  double rz = dot(r, z);
  while (rn / bn > tol && it < maxit) {
    apply(d, q);
    const double alpha = rz / dot(d, q);
    for (size_t k = 0; k < n; ++k) { u[k] += alpha * d[k]; r[k] -= alpha * q[k]; }
    ++it;
    rn = std::sqrt(dot(r, r));
    if (rn / bn <= tol) break;
    precond(r, z);
    const double rz1 = dot(r, z);
    const double beta = rz1 / rz;
    rz = rz1;
    for (size_t k = 0; k < n; ++k) d[k] = z[k] + beta * d[k];
  }
  for (size_t k = 0; k < n; ++k) if (p.act[k]) x[k] = u[k];
  *relres = rn / bn;
  return it;
}

// rho(R) / (eps0 gamma) on the Nx x Ny vertices (scatterQ + fillRHS).
void poisson_rhs(const Sim &s, const std::vector<double> &X, const std::vector<double> &Y, double gamma,
                 std::vector<double> &b) {
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  std::vector<double> r((size_t)Nx * Ny, 0.0);
  for (size_t k = 0; k < X.size(); ++k)
    charge_shape(s.order, X[k], Y[k], s.q[k], 1.0, s.b.org0, s.b.org1, s.b.hr0, s.b.hr1,
                 [&](int i, int j, double v) {
                   if (i >= 0 && j >= 0 && i < Nx && j < Ny) r[(size_t)j * Nx + i] += v;
                 });
  const double cc = 1 / (EPS0 * gamma);
  b.resize(r.size());
  for (size_t k = 0; k < r.size(); ++k) b[k] = (r[k] / (s.b.hr0 * s.b.hr1)) * cc;
}

// copyFields static -> window interior (main.cpp:335-337), then the three
// exchanges (:340-342).
void copy_to_window(Sim &s) {
  for (int j = 0; j < s.L1; ++j)
    for (int i = 0; i < s.L0; ++i) {
      int si = i + s.P0, sj = j + s.P1;
      if (si < 0 || sj < 0 || si >= s.b.Nx || sj >= s.b.Ny) continue;
      s.mEx.at(i, j) = s.Ex.at(si, sj); s.mEy.at(i, j) = s.Ey.at(si, sj);
      s.mHx.at(i, j) = s.Hx.at(si, sj); s.mHy.at(i, j) = s.Hy.at(si, sj);
    }
  exchange(s, 0); exchange(s, 1); exchange(s, 2);
}

}  // namespace

// ===========================================================================
// C ABI for ctypes (tests and bench only).
extern "C" {

struct orc_config {
  int Nx, Ny, order, fixed_point;
  double length_before, length_after, width, phi_deg, ekin_mev, bz;
  double dt;               // <= 0: dt = hx / c (main.cpp:187)
  double charge_mass;      // PartBunch charge-to-mass ratio (main.cpp:223: -1e-9 / m_e)
  double fixed_scale;      // fixed-point scale (fixed_point = 1)
};

float orc_q_rsqrt(float x) { return q_rsqrt(x); }
// The crossing split of one move (cell borders, or dual-cell borders when dual != 0).
long orc_crossings(int dual, double o0, double o1, double n0, double n1, double h0, double h1, double org0,
                   double org1, double *frac, double *s0, double *s1) {
  Xing xs[32];
  const size_t n = border_crossings(xs, o0, o1, n0, n1, h0, h1, org0, org1, dual != 0);
  for (size_t k = 0; k < n; ++k) { frac[k] = xs[k].fraction; s0[k] = xs[k].s0; s1[k] = xs[k].s1; }
  return (long)n;
}

// Bend setup: writes hr0, hr1, origin0, origin1, center0, center1, R, phi.
void orc_bend(int Nx, int Ny, double Lb, double La, double w, double phi_deg, double ekin,
              double bz, double *out8) {
  Bend b; bend_setup(b, Nx, Ny, Lb, La, w, phi_deg, ekin, bz);
  double o[8] = {b.hr0, b.hr1, b.org0, b.org1, b.cen0, b.cen1, b.R, b.phi};
  std::memcpy(out8, o, sizeof(o));
}

// Inside mask (Nx*Ny bytes) and cut cells (7 doubles each: i, j, l0, l1, area,
// n0, n1).  Returns the number of cut cells, or < 0 on a reference abort.
long orc_geometry(int Nx, int Ny, double Lb, double La, double w, double phi_deg, double ekin,
                  double bz, uint8_t *inside, double *cells, long max_cells) {
  Bend b; bend_setup(b, Nx, Ny, Lb, La, w, phi_deg, ekin, bz);
  std::vector<uint8_t> in; std::vector<CutCell> cc; std::vector<int> inv;
  int rc = bend_cells(b, in, cc, inv);
  if (rc) return rc;
  std::memcpy(inside, in.data(), in.size());
  long n = (long)cc.size();
  for (long k = 0; k < n && k < max_cells; ++k) {
    double v[7] = {(double)cc[k].i, (double)cc[k].j, cc[k].l0, cc[k].l1, cc[k].area, cc[k].n0, cc[k].n1};
    std::memcpy(cells + 7 * k, v, sizeof(v));
  }
  return n;
}

// ScatterGatherImpl<IntOp>::gather on a dense patch (row-major, x fastest).
// comp = 0/1: edge component; comp = 2: cell-centred field.
void orc_gather(int order, int comp, const double *patch, int nx, int ny, double o0, double o1,
                double h0, double h1, const double *x, const double *y, long n, double *out) {
  Patch p{patch, nx, ny, o0, o1, h0, h1};
  for (long i = 0; i < n; ++i)
    out[i] = comp < 2 ? gather_edge(order, p, x[i], y[i], comp) : gather_cell(order, p, x[i], y[i]);
}

void orc_scatter(int order, int comp, double *patch, int nx, int ny, double o0, double o1,
                 double h0, double h1, const double *x, const double *y, const double *val, long n) {
  WPatch p{patch, nx, ny, o0, o1, h0, h1};
  for (long i = 0; i < n; ++i) scatter_one(order, comp < 2, comp < 2 ? comp : 0, p, x[i], y[i], val[i]);
}

// Current deposit over a mesh with origin (org0, org1); J is a dense
// (ni x nj) patch whose element (0,0) is absolute index (i0, j0).
void orc_deposit(int order, int comp, const double *ox, const double *oy, const double *x,
                 const double *y, const double *q, long n, double org0, double org1, double h0,
                 double h1, double dt, int i0, int j0, int ni, int nj, double *J,
                 int fixed_point, double fixed_scale) {
  Grid g; g.init(ni, nj, 0);
  JSink s{&g, fixed_point != 0, fixed_scale, {}, i0, j0};
  if (s.fixed) s.acc.assign(g.v.size(), 0);
  for (long i = 0; i < n; ++i)
    deposit(order, s, comp, q[i], ox[i], oy[i], x[i], y[i], h0, h1, org0, org1, dt);
  for (size_t k = 0; k < g.v.size(); ++k) J[k] = s.fixed ? (double)s.acc[k] / fixed_scale : g.v[k];
}

// Charge difference rho(R) - rho(oldR) at vertices for the matching charge
// shape (Zeroth/First/SecondOrderShapeFunction::getChargeDensityDiffImpl),
// divided by the cell area.  rho is a dense (ni x nj) patch at absolute (i0, j0).
void orc_charge_diff(int order, const double *ox, const double *oy, const double *x,
                     const double *y, const double *q, long n, double org0, double org1,
                     double h0, double h1, int i0, int j0, int ni, int nj, double *rho) {
  std::vector<double> r((size_t)ni * nj, 0.0);
  auto add = [&](int i, int j, double v) {
    int a = i - i0, b = j - j0;
    if (a >= 0 && b >= 0 && a < ni && b < nj) r[(size_t)b * ni + a] += v;
  };
  for (long k = 0; k < n; ++k) {
    charge_shape(order, x[k], y[k], q[k], 1.0, org0, org1, h0, h1, add);
    charge_shape(order, ox[k], oy[k], q[k], -1.0, org0, org1, h0, h1, add);
  }
  for (size_t k = 0; k < r.size(); ++k) rho[k] = r[k] / (h0 * h1);
}

// ---- whole-loop simulation ----
void *orc_create(const orc_config *c) {
  Sim *s = new Sim;
  s->order = c->order;
  s->fixed = c->fixed_point != 0;
  s->fscale = c->fixed_scale;
  bend_setup(s->b, c->Nx, c->Ny, c->length_before, c->length_after, c->width, c->phi_deg,
             c->ekin_mev, c->bz);
  s->dt = c->dt > 0 ? c->dt : s->b.hr0 / C;
  s->qm = c->charge_mass;
  s->err = bend_cells(s->b, s->inside, s->cells, s->inv);
  s->Ex.init(c->Nx, c->Ny); s->Ey.init(c->Nx, c->Ny);
  s->Hx.init(c->Nx, c->Ny); s->Hy.init(c->Nx, c->Ny);
  return s;
}
void orc_destroy(void *h) { delete (Sim *)h; }
int orc_error(void *h) { return ((Sim *)h)->err; }
double orc_dt(void *h) { return ((Sim *)h)->dt; }

// Static fields: each array is Nx*Ny, row-major (x fastest), no guards.
void orc_set_static(void *h, const double *ex, const double *ey, const double *hx, const double *hy) {
  Sim &s = *(Sim *)h;
  for (int j = 0; j < s.b.Ny; ++j)
    for (int i = 0; i < s.b.Nx; ++i) {
      size_t k = (size_t)j * s.b.Nx + i;
      s.Ex.at(i, j) = ex[k]; s.Ey.at(i, j) = ey[k]; s.Hx.at(i, j) = hx[k]; s.Hy.at(i, j) = hy[k];
    }
}
void orc_get_static(void *h, double *ex, double *ey, double *hx, double *hy) {
  Sim &s = *(Sim *)h;
  for (int j = 0; j < s.b.Ny; ++j)
    for (int i = 0; i < s.b.Nx; ++i) {
      size_t k = (size_t)j * s.b.Nx + i;
      ex[k] = s.Ex.at(i, j); ey[k] = s.Ey.at(i, j); hx[k] = s.Hx.at(i, j); hy[k] = s.Hy.at(i, j);
    }
}

// SCBoundaryCondition::resetOutsideDomain, SCBoundaryCondition.hh:163-195.
void orc_reset_outside(void *h) {
  Sim &s = *(Sim *)h;
  for (int j = 0; j < s.b.Ny; ++j)
    for (int i = 0; i < s.b.Nx; ++i) {
      size_t k = (size_t)j * s.b.Nx + i;
      if (s.inside[k]) continue;
      int n = s.inv[k];
      if (n == -1) { s.Ex.at(i, j) = 0.0; s.Ey.at(i, j) = 0.0; continue; }
      const CutCell &c = s.cells[n];
      if (c.l0 < SPACE_EPS) s.Ex.at(i, j) = 0.0;
      if (c.l1 < SPACE_EPS) s.Ey.at(i, j) = 0.0;
      if (c.area < MINAREA) { s.Ex.at(i, j) = 0.0; s.Ey.at(i, j) = 0.0; }
    }
}

// Load particles, sort them (PartBunch::sortParticles) and open the window
// (main.cpp:198-217, :335-342).  Returns 0 or a negative error.
int orc_load(void *h, const double *x, const double *y, const double *px, const double *py,
             const double *q, long n) {
  Sim &s = *(Sim *)h;
  s.x.assign(x, x + n); s.y.assign(y, y + n); s.px.assign(px, px + n); s.py.assign(py, py + n);
  s.q.assign(q, q + n); s.ox = s.x; s.oy = s.y;
  if (n == 0) return -2;
  // Distribution::getDomain on the static mesh, then +-5 cells.
  double mn0 = x[0], mn1 = y[0], mx0 = x[0], mx1 = y[0];
  for (long i = 0; i < n; ++i) {
    mn0 = std::min(mn0, x[i]); mn1 = std::min(mn1, y[i]);
    mx0 = std::max(mx0, x[i]); mx1 = std::max(mx1, y[i]);
  }
  int d[4] = {(int)std::floor((mn0 - s.b.org0) / s.b.hr0), (int)std::floor((mx0 - s.b.org0) / s.b.hr0),
              (int)std::floor((mn1 - s.b.org1) / s.b.hr1), (int)std::floor((mx1 - s.b.org1) / s.b.hr1)};
  d[0] -= 5; d[1] += 5; d[2] -= 5; d[3] += 5;
  s.P0 = d[0]; s.P1 = d[2];
  s.L0 = d[1] - d[0] + 1; s.L1 = d[3] - d[2] + 1;
  s.mo0 = s.b.org0 + d[0] * s.b.hr0;
  s.mo1 = s.b.org1 + d[2] * s.b.hr1;
  for (Grid *g : {&s.mEx, &s.mEy, &s.mHx, &s.mHy, &s.mJx, &s.mJy}) g->init(s.L0, s.L1);
  // PartBunch::sortParticles: y slices of the window, x ascending inside a slice.
  int lp[4]; pdomain(s, false, lp);
  std::vector<std::vector<size_t>> sl((size_t)(lp[3] - lp[2] + 1));
  for (long i = 0; i < n; ++i) {
    unsigned idy = (unsigned)((int)std::floor((s.y[i] - s.mo1) / s.b.hr1) - lp[2]);
    sl[idy].push_back((size_t)i);
  }
  std::vector<size_t> order;
  for (auto &v : sl) {
    std::stable_sort(v.begin(), v.end(), [&](size_t a, size_t b) { return s.x[a] < s.x[b]; });
    order.insert(order.end(), v.begin(), v.end());
  }
  auto perm = [&](std::vector<double> &a) {
    std::vector<double> t(a.size());
    for (size_t k = 0; k < order.size(); ++k) t[k] = a[order[k]];
    a.swap(t);
  };
  perm(s.x); perm(s.y); perm(s.px); perm(s.py); perm(s.q);
  s.ox = s.x; s.oy = s.y;
  copy_to_window(s);
  return 0;
}

// Initial fields of the loaded bunch (main.cpp:232-248): the three boosted
// electrostatic solves of PoissonSolver::computeField (PoissonSolver.cpp:85-201)
// fill Ey, Hz and Ex of the static mesh (fillFields, :441-507), then
// SCBoundaryCondition::resetOutsideDomain and the window copy.  The first solve
// starts from zero (the reference starts from a random vector), the others
// from the shifted previous solution (shiftLHS, :270-303).
// stats: gamma, then (iterations, relative residual) for each solve.
int orc_initial_fields(void *h, double tol_first, double tol_rest, int maxit, double *stats) {
  Sim &s = *(Sim *)h;
  const size_t n = s.x.size();
  if (n == 0) return -2;
  double pm0 = 0.0, pm1 = 0.0;  // Distribution::get_pmean (Distribution.cpp:136-143)
  for (size_t k = 0; k < n; ++k) { pm0 += s.px[k]; pm1 += s.py[k]; }
  pm0 /= (double)n; pm1 /= (double)n;
  const double gamma = std::sqrt((pm0 * pm0 + pm1 * pm1) + 1);
  PoissonSys p;
  poisson_setup(s, gamma, p);
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  const size_t m = (size_t)Nx * Ny;
  const double hr0 = s.b.hr0 * gamma, hr1 = s.b.hr1;
  // positions of the three charge densities
  std::vector<double> X1(n), Y1(n), X2(n), Y2(n);
  const double full = (s.dt / 2) * C, back = (-s.dt / 2) * C, mv = -0.5 * hr0 / gamma;
  for (size_t k = 0; k < n; ++k) {
    const double r = (double)q_rsqrt((float)(1 + (s.px[k] * s.px[k] + s.py[k] * s.py[k])));
    X1[k] = s.x[k] + full * s.px[k] * r;
    Y1[k] = s.y[k] + full * s.py[k] * r;
    X2[k] = (X1[k] + back * s.px[k] * r) + mv;
    Y2[k] = (Y1[k] + back * s.py[k] * r) + 0.0;
  }
  std::vector<double> b, phi1(m, 0.0), phi2(m), phi3(m);
  double rr[3];
  int its[3];
  poisson_rhs(s, X1, Y1, gamma, b);
  its[0] = poisson_solve(p, b, phi1, tol_first, maxit, &rr[0]);
  // shiftLHS(+1): phi(i) + (phi(i+1) - phi(i))
  for (int j = 0; j < Ny; ++j)
    for (int i = 0; i < Nx; ++i) {
      const size_t k = (size_t)j * Nx + i;
      const double nb = i + 1 < Nx ? phi1[k + 1] : 0.0;
      phi2[k] = phi1[k] + (1.0 * nb - 1.0 * phi1[k]);
    }
  poisson_rhs(s, X2, Y2, gamma, b);
  its[1] = poisson_solve(p, b, phi2, tol_rest, maxit, &rr[1]);
  // shiftLHS(-0.5): phi(i) + 0.5 (phi(i-1) - phi(i))
  for (int j = 0; j < Ny; ++j)
    for (int i = 0; i < Nx; ++i) {
      const size_t k = (size_t)j * Nx + i;
      const double nb = i > 0 ? phi2[k - 1] : 0.0;
      phi3[k] = phi2[k] + (0.5 * nb - 0.5 * phi2[k]);
    }
  poisson_rhs(s, s.x, s.y, gamma, b);
  its[2] = poisson_solve(p, b, phi3, tol_rest, maxit, &rr[2]);
  // fillFields: Ey (component 1), Hz (2), Ex (0); the guard beyond the last
  // row / column holds zero.
  const double bg = std::sqrt(gamma * gamma - 1);
  const double hden = 2 * C * MU0 * hr1;
  for (int j = 0; j < Ny; ++j)
    for (int i = 0; i < Nx; ++i) {
      const size_t k = (size_t)j * Nx + i;
      const double ey0 = gamma * phi1[k] / hr1;
      const double ey1 = j + 1 < Ny ? gamma * phi1[k + Nx] / hr1 : 0.0;
      s.Ey.at(i, j) = ey0 - ey1;
      const double h0v = bg * phi2[k] / hden;
      const double h1v = j + 1 < Ny ? bg * phi2[k + Nx] / hden : 0.0;
      s.Hx.at(i, j) = h0v - h1v;
      s.Hy.at(i, j) = h0v - h1v;
      const double ex0 = phi3[k] / hr0;
      const double ex1 = i + 1 < Nx ? phi3[k + 1] / hr0 : 0.0;
      s.Ex.at(i, j) = ex0 - ex1;
    }
  orc_reset_outside(h);
  copy_to_window(s);
  if (stats) {
    stats[0] = gamma;
    for (int t = 0; t < 3; ++t) { stats[1 + 2 * t] = its[t]; stats[2 + 2 * t] = rr[t]; }
  }
  return 0;
}


void orc_get_particles(void *h, double *x, double *y, double *px, double *py) {
  Sim &s = *(Sim *)h;
  std::memcpy(x, s.x.data(), s.x.size() * 8); std::memcpy(y, s.y.data(), s.y.size() * 8);
  std::memcpy(px, s.px.data(), s.px.size() * 8); std::memcpy(py, s.py.data(), s.py.size() * 8);
}
void orc_get_old(void *h, double *ox, double *oy) {
  Sim &s = *(Sim *)h;
  std::memcpy(ox, s.ox.data(), s.ox.size() * 8); std::memcpy(oy, s.oy.data(), s.oy.size() * 8);
}
// window: P0, P1, L0, L1 and origin; global bounds gb[4]
void orc_get_window(void *h, int *w4, double *o2, int *gb4) {
  Sim &s = *(Sim *)h;
  w4[0] = s.P0; w4[1] = s.P1; w4[2] = s.L0; w4[3] = s.L1;
  o2[0] = s.mo0; o2[1] = s.mo1;
  std::memcpy(gb4, s.gb, sizeof(s.gb));
}
// which: 0 Ex, 1 Ey, 2 Hzx, 3 Hzy, 4 Jx, 5 Jy; out is (L0+2)*(L1+2) incl. guards.
void orc_get_window_field(void *h, int which, double *out) {
  Sim &s = *(Sim *)h;
  Grid *g[6] = {&s.mEx, &s.mEy, &s.mHx, &s.mHy, &s.mJx, &s.mJy};
  std::memcpy(out, g[which]->v.data(), g[which]->v.size() * 8);
}

// Fine-grained pieces of the loop.
void orc_push(void *h, int jcomp) { push(*(Sim *)h, jcomp); }
void orc_drift(void *h, double dt) { drift(*(Sim *)h, dt); }
void orc_half_h(void *h) { half_h(*(Sim *)h); }
// Absorbing layers (width cells, grading order, normal-incidence reflection); width 0 = off.
void orc_set_pml(void *h, int width, int order, double reflection) {
  Sim &s = *(Sim *)h;
  s.pml.clear(); s.plo.clear(); s.phi.clear(); s.psi.clear();
  if (width <= 0) return;
  const int Nx = s.b.Nx, Ny = s.b.Ny;
  const double h0 = s.b.hr0, h1 = s.b.hr1, o0 = s.b.org0, o1 = s.b.org1, dt = s.dt;
  const double W = width * h0;
  const double smax = -(order + 1) * EPS0 * C * std::log(reflection) / (2.0 * W);
  s.plo.assign(Ny, 0);
  s.phi.assign(Ny, Nx);
  for (int j = 0; j < Ny; ++j) {
    auto sig = [&](int i, double &sx, double &sy, double &tx, double &ty, double &ux, double &uy) {
      pml_sigma(s.b, W, order, smax, o0 + (i + 0.5) * h0, o1 + (j + 0.5) * h1, sx, sy);
      pml_sigma(s.b, W, order, smax, o0 + (i + 0.5) * h0, o1 + j * h1, tx, ty);
      pml_sigma(s.b, W, order, smax, o0 + i * h0, o1 + (j + 0.5) * h1, ux, uy);
    };
    int lo = 0, hi = Nx;
    for (int i = 0; i < Nx; ++i) {
      if (!s.inside[(size_t)j * Nx + i]) continue;
      double sx, sy, tx, ty, ux, uy;
      sig(i, sx, sy, tx, ty, ux, uy);
      if (sx > 0 || sy > 0 || ty > 0 || ux > 0) {
        if (i < Nx / 2) lo = std::max(lo, i + 1);
        else hi = std::min(hi, i);
      }
    }
    if (hi < lo) hi = lo;
    s.plo[j] = lo; s.phi[j] = hi;
    for (int i = 0; i < Nx; ++i) {
      if (!s.inside[(size_t)j * Nx + i] || (i >= lo && i < hi)) continue;
      double sx, sy, tx, ty, ux, uy;
      sig(i, sx, sy, tx, ty, ux, uy);
      Sim::Pml c{};
      c.i = i; c.j = j;
      pml_coef(sx, 0.5 * dt, c.bhx, c.ahx);
      pml_coef(sy, 0.5 * dt, c.bhy, c.ahy);
      pml_coef(ty, dt, c.bex, c.aex);
      pml_coef(ux, dt, c.bey, c.aey);
      s.pml.push_back(c);
    }
  }
  s.psi.assign(4 * s.pml.size(), 0.0);
}
int orc_pml_cells(void *h) { return (int)((Sim *)h)->pml.size(); }
void orc_update_e(void *h, int comp) { update_e(*(Sim *)h, comp); }
int orc_move(void *h) { return move_window(*(Sim *)h); }

// TETMSolver::updateField_firstStep + updateField_secondStep + moveMesh
// (main.cpp:390-506), nsteps times.
int orc_step(void *h, int nsteps) {
  Sim &s = *(Sim *)h;
  for (int k = 0; k < nsteps; ++k) {
    push(s, 0);
    half_h(s);
    update_e(s, 0);
    half_h(s);
    drift(s, -0.5 * s.dt);
    push(s, 1);
    update_e(s, 1);
    drift(s, -0.5 * s.dt);
    if (s.x.empty()) continue;
    int rc = move_window(s);
    if (rc) return rc;
  }
  return 0;
}

// IntegrateElongCommand::execute (IntegrateElong.cpp:38-89) for one step: the
// samples i = 2 .. L0-3 along the mean momentum; out[k] = E_s or NaN when the
// sample lies outside the window.  rmean/pmean come from the caller.
void orc_wake(void *h, double r0, double r1, double p0, double p1, double *out) {
  Sim &s = *(Sim *)h;
  const double lenP = std::sqrt(p0 * p0 + p1 * p1);
  const double cP = p0 / lenP, sP = p1 / lenP;
  const int W0 = s.L0 + 2;
  std::vector<double> ex((size_t)W0 * (s.L1 + 2)), ey(ex.size());
  for (int j = -1; j <= s.L1; ++j)
    for (int i = -1; i <= s.L0; ++i) {
      ex[(size_t)(j + 1) * W0 + i + 1] = s.mEx.at(i, j);
      ey[(size_t)(j + 1) * W0 + i + 1] = s.mEy.at(i, j);
    }
  Patch pex{ex.data() + W0 + 1, W0, s.L1 + 2, s.mo0, s.mo1, s.b.hr0, s.b.hr1};
  Patch pey{ey.data() + W0 + 1, W0, s.L1 + 2, s.mo0, s.mo1, s.b.hr0, s.b.hr1};
  for (int i = 2; i <= s.L0 - 3; ++i) {
    double l0 = s.mo0 + i * s.b.hr0 - r0;
    double a0 = cP * l0 + sP * 0.0 + r0;
    double a1 = -sP * l0 + cP * 0.0 + r1;
    int ci = (int)std::floor((a0 - s.mo0) / s.b.hr0), cj = (int)std::floor((a1 - s.mo1) / s.b.hr1);
    if (ci < 0 || cj < 0 || ci >= s.L0 || cj >= s.L1) { out[i - 2] = NAN; continue; }
    double e0 = gather_cic_edge(pex, a0, a1, 0), e1 = gather_cic_edge(pey, a0, a1, 1);
    out[i - 2] = cP * e0 + sP * e1;
  }
}

// SaveEMFieldsCommand::execute (src/Commands/SaveEMFields.cpp:34-189) after copyFields
// (main.cpp:468-476): the static mesh with the mini mesh's values over the points it covers
// (the current only with with_current; the loop's static current is zero), gathered with the
// run's shape order at one point per static column on the line through the centroid along the
// mean momentum.  Points beyond the static guard ring read zero.  out: 7 values per sample.
void orc_moments(void *h, double *out);
void orc_line_fields(void *h, int with_current, double *out, int cap, int *count) {
  Sim &s = *(Sim *)h;
  double m[18];
  orc_moments(h, m);
  const double org0 = s.b.org0, org1 = s.b.org1, h0 = s.b.hr0, h1 = s.b.hr1;
  const double g0 = std::floor((m[10] - org0) / h0), g1 = std::floor((m[12] - org0) / h0);
  const double l0 = std::floor(1.5 * g0 - 0.5 * g1), u0 = 2 * g1 - g0;
  const long i0 = (long)l0;
  const int n = (int)std::floor(u0 - l0 + 0.5) + 1;
  *count = n;
  if (!out || cap < n) return;
  const int Nx = s.b.Nx, Ny = s.b.Ny, M = 2, W = Nx + 2 * M;
  // dense overlaid copies with a 2-point margin; index (0, 0) = static point (0, 0)
  std::vector<double> ex((size_t)W * (Ny + 2 * M), 0.0), ey(ex.size(), 0.0), hz(ex.size(), 0.0),
      jx(ex.size(), 0.0), jy(ex.size(), 0.0);
  auto at = [&](std::vector<double> &v, int i, int j) -> double & { return v[(size_t)(j + M) * W + i + M]; };
  for (int j = -1; j <= Ny; ++j)
    for (int i = -1; i <= Nx; ++i) {
      const int a = i - s.P0, b = j - s.P1;
      if (a >= 0 && a < s.L0 && b >= 0 && b < s.L1) {
        at(ex, i, j) = s.mEx.at(a, b); at(ey, i, j) = s.mEy.at(a, b);
        at(hz, i, j) = s.mHx.at(a, b) + s.mHy.at(a, b);
        if (with_current) { at(jx, i, j) = s.mJx.at(a, b); at(jy, i, j) = s.mJy.at(a, b); }
      } else {
        at(ex, i, j) = s.Ex.at(i, j); at(ey, i, j) = s.Ey.at(i, j);
        at(hz, i, j) = s.Hx.at(i, j) + s.Hy.at(i, j);
      }
    }
  auto patch = [&](std::vector<double> &v) { return Patch{v.data() + (size_t)M * W + M, W, Ny + 2 * M, org0, org1, h0, h1}; };
  const Patch pex = patch(ex), pey = patch(ey), phz = patch(hz), pjx = patch(jx), pjy = patch(jy);
  const double R0 = m[0], R1 = m[1], P0 = m[2], P1 = m[3];
  const double lenP = std::sqrt(P0 * P0 + P1 * P1), cP = P0 / lenP, sP = P1 / lenP;
  for (int k = 0; k < n; ++k) {
    const long i = i0 + k;
    const double dx = (org0 + (double)i * h0) - R0, dy = dx / P0 * P1;
    double *o = out + 7 * (size_t)k;
    o[0] = std::sqrt(dx * dx + dy * dy) * (dx > 0 ? 1.0 : -1.0);
    o[5] = dx + R0;
    o[6] = dy + R1;
    const double x = org0 + (double)i * h0, y = R1 + (x - R0) / P0 * P1;
    const long cy = (long)std::floor((y - org1) * (1.0 / h1));
    if (i < 0 || i >= Nx || cy < 0 || cy >= Ny) { o[1] = o[2] = o[3] = o[4] = 0.0; continue; }
    const double e0 = gather_edge(s.order, pex, x, y, 0), e1 = gather_edge(s.order, pey, x, y, 1);
    const double j0 = gather_edge(s.order, pjx, x, y, 0), j1 = gather_edge(s.order, pjy, x, y, 1);
    o[1] = cP * e0 + sP * e1;
    o[2] = -sP * e0 + cP * e1;
    o[3] = gather_cell(s.order, phz, x, y);
    o[4] = cP * j0 + sP * j1;
  }
}

// CalcEnergyCommand::execute (src/Commands/CalcEnergy.cpp:41-120) before its time
// averaging, in the reference's order: every static point, plus every mini-mesh
// point, minus the static points the mini mesh covers; times the cell area.
void orc_field_energy(void *h, int with_window, double *out2) {
  Sim &s = *(Sim *)h;
  double ee = 0.0, hh = 0.0;
  auto add = [&](const Grid &ex, const Grid &ey, const Grid &hx, const Grid &hy, int i, int j, double sg) {
    const double a = ex.at(i, j), b = ey.at(i, j), c = hx.at(i, j) + hy.at(i, j);
    ee += sg * (a * a + b * b);
    hh += sg * c * c;
  };
  for (int j = 0; j < s.b.Ny; ++j)
    for (int i = 0; i < s.b.Nx; ++i) add(s.Ex, s.Ey, s.Hx, s.Hy, i, j, 1.0);
  if (with_window) {
    for (int j = 0; j < s.L1; ++j)
      for (int i = 0; i < s.L0; ++i) add(s.mEx, s.mEy, s.mHx, s.mHy, i, j, 1.0);
    const int i0 = std::max(0, s.P0), i1 = std::min(s.b.Nx - 1, s.P0 + s.L0 - 1);
    const int j0 = std::max(0, s.P1), j1 = std::min(s.b.Ny - 1, s.P1 + s.L1 - 1);
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) add(s.Ex, s.Ey, s.Hx, s.Hy, i, j, -1.0);
  }
  const double area = s.b.hr0 * s.b.hr1;
  out2[0] = ee * area;
  out2[1] = hh * area;
}

// PartBunch::calcBeamParameters / calcMoments (PartBunch.cpp:584-767) with
// long-double Kahan sums.  out: rmean2, pmean2, rrms2, prms2, eps2, rmin2, rmax2, Ekin, dE,
// Dy, DDy (moments (2, 1) and (3, 1) over N, PartBunch.cpp:643-644).
void orc_moments(void *h, double *out) {
  Sim &s = *(Sim *)h;
  const size_t n = s.x.size();
  std::memset(out, 0, 18 * sizeof(double));
  if (n == 0) return;
  const double m0 = 0.51099906e-03 * 1000;
  struct K { long double sum = 0, cor = 0; };
  auto ks = [](K a, double v) { K r; long double yv = v - a.cor; long double t = a.sum + yv; r.cor = (t - a.sum) - yv; r.sum = t; return r; };
  K sums[4]; K sq[16];
  double lim[4] = {s.x[0], s.y[0], s.x[0], s.y[0]};
  for (size_t k = 0; k < n; ++k) {
    double part[4] = {s.x[k], s.px[k], s.y[k], s.py[k]};
    if (s.x[k] < lim[0]) lim[0] = s.x[k];
    if (s.x[k] > lim[2]) lim[2] = s.x[k];
    if (s.y[k] < lim[1]) lim[1] = s.y[k];
    if (s.y[k] > lim[3]) lim[3] = s.y[k];
    for (int i = 0; i < 4; ++i) sums[i] = ks(sums[i], part[i]);
  }
  long double cen[4]; for (int i = 0; i < 4; ++i) cen[i] = sums[i].sum;
  double aR0 = (double)(cen[0] / n), aR1 = (double)(cen[2] / n);
  double aP0 = (double)(cen[1] / n), aP1 = (double)(cen[3] / n);
  double am = std::sqrt(aP0 * aP0 + aP1 * aP1), cph = aP0 / am, sph = aP1 / am;
  for (size_t k = 0; k < n; ++k) {
    double part[4];
    part[1] = cph * s.px[k] + sph * s.py[k];
    part[3] = -sph * s.px[k] + cph * s.py[k];
    part[0] = s.x[k] - aR0; part[2] = s.y[k] - aR1;
    double tmp = cph * part[0] + sph * part[2];
    part[2] = -sph * part[0] + cph * part[2];
    part[0] = tmp;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j <= i; ++j) sq[i * 4 + j] = ks(sq[i * 4 + j], part[i] * part[j]);
  }
  long double M[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j <= i; ++j) { M[i * 4 + j] = sq[i * 4 + j].sum; M[j * 4 + i] = M[i * 4 + j]; }
  const double N = (double)n;
  double rmean[2], pmean[2];
  for (int i = 0; i < 2; ++i) { rmean[i] = (double)(cen[2 * i] / N); pmean[i] = (double)(cen[2 * i + 1] / N); }
  double c1 = pmean[0] * pmean[0] + pmean[1] * pmean[1];
  double cc[4] = {0.0, c1, 0.0, 0.0};
  double rsq[2], psq[2], rp[2], rrms[2], prms[2], eps[2];
  for (int i = 0; i < 2; ++i) {
    rsq[i] = (double)M[(2 * i) * 4 + 2 * i];
    psq[i] = (double)(M[(2 * i + 1) * 4 + 2 * i + 1] - (long double)N * (long double)cc[2 * i + 1]);
    if (psq[i] < 0) psq[i] = 0;
    rp[i] = (double)M[(2 * i) * 4 + 2 * i + 1];
  }
  for (int i = 0; i < 2; ++i) {
    double e2 = (rsq[i] * psq[i] - rp[i] * rp[i]) / (N * N);
    rrms[i] = std::sqrt(rsq[i] / N); prms[i] = std::sqrt(psq[i] / N);
    eps[i] = std::sqrt(std::max(e2, 0.0));
  }
  double gam = 0.0;
  for (size_t k = 0; k < n; ++k) gam += std::sqrt(1.0 + (s.px[k] * s.px[k] + s.py[k] * s.py[k]));
  gam /= N;
  double ek = (gam - 1.0) * m0;
  double dE = prms[0] * std::sqrt(ek * (ek + 2. * m0) / (1. + ek * (ek + 2. * m0) / (m0 * m0)));
  double o[18] = {rmean[0], rmean[1], pmean[0], pmean[1], rrms[0], rrms[1], prms[0], prms[1],
                  eps[0], eps[1], lim[0], lim[1], lim[2], lim[3], ek, dE,
                  (double)(M[2 * 4 + 1] / (long double)N), (double)(M[3 * 4 + 1] / (long double)N)};
  std::memcpy(out, o, sizeof(o));
}

}  // extern "C"
