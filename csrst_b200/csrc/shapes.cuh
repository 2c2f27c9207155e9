// Device shape functions: field gather (ScatterGatherImpl) and the
// charge-conserving current deposit (Zeroth/First/SecondOrderShapeFunction).
//
// The arithmetic keeps the reference's operation order so that, built with
// --fmad=false, every gathered value and every deposit weight is the same
// IEEE double the reference computes.  ORDER 0 = IntCIC with the
// Villasenor-Buneman deposit, 1 = IntS1 (TSC) with the S1 x S2 deposit,
// 2 = IntS2 (cubic) with the S2 x S3 deposit.
#pragma once

#include "common.cuh"

namespace csrst {

// A read-only view of a field patch: value(I, J) for patch-relative indices.
struct PatchView {
  const double *base;  // address of patch-relative (0, 0)
  int pitch;
  __device__ __forceinline__ double operator()(int i, int j) const {
    return __ldg(base + (ptrdiff_t)j * pitch + i);
  }
};

// Hz patch built from the split components, Hz = Hzx + Hzy element by element
// (PartBunch::getFields, PartBunch.cpp:1012-1017).
struct SumView {
  PatchView a, b;
  __device__ __forceinline__ double operator()(int i, int j) const { return a(i, j) + b(i, j); }
};

// --- gather -----------------------------------------------------------------

// Edge component `comp` at patch coordinates (pp0, pp1) = (R - origin) / h.
// ScatterGatherImpl.hh:69-104 (CIC), :201-253 (S1), :406-468 (S2).  S is the
// arithmetic type: double reproduces the reference bit for bit, float is the
// FP32 mode's gather.
template <int ORDER, class F, class S>
__device__ __forceinline__ S gather_edge(const F &f, S pp0, S pp1, int comp) {
  const S one = S(1), half = S(0.5), zero = S(0);
  if (ORDER == 0) {
    long l0 = (long)floor(pp0 + (comp == 0 ? half : zero));
    long l1 = (long)floor(pp1 + (comp == 1 ? half : zero));
    if (comp == 0) l0 -= 1; else l1 -= 1;
    S g0 = (S)l0, g1 = (S)l1;
    if (comp == 0) g0 += half; else g1 += half;
    const S d0 = pp0 - g0, d1 = pp1 - g1;
    const int I = (int)l0, J = (int)l1;
    return ((one - d1) * ((one - d0) * f(I, J) + d0 * f(I + 1, J)) +
            d1 * ((one - d0) * f(I, J + 1) + d0 * f(I + 1, J + 1)));
  } else if (ORDER == 1) {
    long l0 = (long)floor(pp0 + (comp == 0 ? zero : half));
    long l1 = (long)floor(pp1 + (comp == 1 ? zero : half));
    S g0 = (S)l0, g1 = (S)l1;
    if (comp == 0) g0 += half; else g1 += half;
    const S d0 = pp0 - g0, d1 = pp1 - g1;
    const S bx = S(0.75) - d0 * d0, cx = half * (half + d0) * (half + d0), ax = one - (bx + cx);
    const S by = S(0.75) - d1 * d1, cy = half * (half + d1) * (half + d1), ay = one - (by + cy);
    const int I = (int)l0, J = (int)l1;
    return (ay * (ax * f(I - 1, J - 1) + bx * f(I, J - 1) + cx * f(I + 1, J - 1)) +
            by * (ax * f(I - 1, J) + bx * f(I, J) + cx * f(I + 1, J)) +
            cy * (ax * f(I - 1, J + 1) + bx * f(I, J + 1) + cx * f(I + 1, J + 1)));
  } else {
    long l0 = (long)floor(pp0 + (comp == 0 ? half : zero));
    long l1 = (long)floor(pp1 + (comp == 1 ? half : zero));
    if (comp == 0) l0 -= 1; else l1 -= 1;
    S g0 = (S)l0, g1 = (S)l1;
    if (comp == 0) g0 += half; else g1 += half;
    const S d0 = pp0 - g0, d1 = pp1 - g1;
    const S q0 = d0 * d0, q1 = d1 * d1;
    const S t23 = S(2.0 / 3.0), t16 = S(1.0 / 6.0);
    const S bx = t23 - q0 * (one - half * d0), cx = t23 - half * (one - d0) * (one - q0), ex = t16 * q0 * d0;
    const S ax = one - (bx + cx + ex);
    const S by = t23 - q1 * (one - half * d1), cy = t23 - half * (one - d1) * (one - q1), ey = t16 * q1 * d1;
    const S ay = one - (by + cy + ey);
    const int I = (int)l0, J = (int)l1;
    // The last term reads (I+1, J+2), as the reference does (ScatterGatherImpl.hh:467).
    return (ay * (ax * f(I - 1, J - 1) + bx * f(I, J - 1) + cx * f(I + 1, J - 1) + ex * f(I + 2, J - 1)) +
            by * (ax * f(I - 1, J) + bx * f(I, J) + cx * f(I + 1, J) + ex * f(I + 2, J)) +
            cy * (ax * f(I - 1, J + 1) + bx * f(I, J + 1) + cx * f(I + 1, J + 1) + ex * f(I + 2, J + 1)) +
            ey * (ax * f(I - 1, J + 2) + bx * f(I, J + 2) + cx * f(I + 1, J + 2) + ex * f(I + 1, J + 2)));
  }
}

// Cell-centred field.  ScatterGatherImpl.hh:106-134, :255-301, :470-527.
template <int ORDER, class F, class S>
__device__ __forceinline__ S gather_cell(const F &f, S pp0, S pp1) {
  const S one = S(1), half = S(0.5);
  if (ORDER == 0) {
    const long l0 = (long)floor(pp0 - half), l1 = (long)floor(pp1 - half);
    const S d0 = pp0 - ((S)l0 + half), d1 = pp1 - ((S)l1 + half);
    const int I = (int)l0, J = (int)l1;
    return ((one - d1) * ((one - d0) * f(I, J) + d0 * f(I + 1, J)) +
            d1 * ((one - d0) * f(I, J + 1) + d0 * f(I + 1, J + 1)));
  } else if (ORDER == 1) {
    const long l0 = (long)floor(pp0), l1 = (long)floor(pp1);
    const S d0 = pp0 - ((S)l0 + half), d1 = pp1 - ((S)l1 + half);
    const S bx = S(0.75) - d0 * d0, cx = half * (half + d0) * (half + d0), ax = one - (bx + cx);
    const S by = S(0.75) - d1 * d1, cy = half * (half + d1) * (half + d1), ay = one - (by + cy);
    const int I = (int)l0, J = (int)l1;
    return (ay * (ax * f(I - 1, J - 1) + bx * f(I, J - 1) + cx * f(I + 1, J - 1)) +
            by * (ax * f(I - 1, J) + bx * f(I, J) + cx * f(I + 1, J)) +
            cy * (ax * f(I - 1, J + 1) + bx * f(I, J + 1) + cx * f(I + 1, J + 1)));
  } else {
    const long l0 = (long)floor(pp0 - half), l1 = (long)floor(pp1 - half);
    const S d0 = pp0 - ((S)l0 + half), d1 = pp1 - ((S)l1 + half);
    const S q0 = d0 * d0, q1 = d1 * d1;
    const S t23 = S(2.0 / 3.0), t16 = S(1.0 / 6.0);
    const S bx = t23 - q0 * (one - half * d0), cx = t23 - half * (one - d0) * (one - q0), ex = t16 * q0 * d0;
    const S ax = one - (bx + cx + ex);
    const S by = t23 - q1 * (one - half * d1), cy = t23 - half * (one - d1) * (one - q1), ey = t16 * q1 * d1;
    const S ay = one - (by + cy + ey);
    const int I = (int)l0, J = (int)l1;
    return (ay * (ax * f(I - 1, J - 1) + bx * f(I, J - 1) + cx * f(I + 1, J - 1) + ex * f(I + 2, J - 1)) +
            by * (ax * f(I - 1, J) + bx * f(I, J) + cx * f(I + 1, J) + ex * f(I + 2, J)) +
            cy * (ax * f(I - 1, J + 1) + bx * f(I, J + 1) + cx * f(I + 1, J + 1) + ex * f(I + 2, J + 1)) +
            ey * (ax * f(I - 1, J + 2) + bx * f(I, J + 2) + cx * f(I + 1, J + 2) + ex * f(I + 1, J + 2)));
  }
}

// --- deposit ----------------------------------------------------------------

constexpr int kMaxCross = 12;  // end points + border crossings kept per push

struct Cross {
  double f, s0, s1;
};

// Border crossings of the segment old -> new (positions relative to the mesh
// origin): src/utils.hh:427-489 (cell borders) and :364-425 (dual cells,
// DUAL = true).  The interior entries are sorted by fraction with a stable
// insertion sort (what libstdc++ std::sort does on so few items) and merged
// when two fractions differ by less than 1e-6 (std::unique with samePos).
// Returns the number of points, or -1 if more crossings than kMaxCross.
template <bool DUAL>
__device__ __forceinline__ int border_crossings(Cross *xs, double o0, double o1, double n0, double n1,
                                                double h0, double h1) {
  int Ii, Ji, If, Jf;
  if (DUAL) {
    Ii = (int)floor(o0 / h0 - 0.5); Ji = (int)floor(o1 / h1 - 0.5);
    If = (int)floor(n0 / h0 - 0.5); Jf = (int)floor(n1 / h1 - 0.5);
  } else {
    Ii = (int)floor(o0 / h0); Ji = (int)floor(o1 / h1);
    If = (int)floor(n0 / h0); Jf = (int)floor(n1 / h1);
  }
  const int nx = abs(If - Ii), ny = abs(Jf - Ji);
  if (nx + ny + 2 > kMaxCross) return -1;
  const double D0 = n0 - o0, D1 = n1 - o1;
  int n = 0;
  xs[n++].f = 0.0;
  int I = Ii, J = Ji;
  while (I < If) {
    const double x = DUAL ? h0 * (I + 1.5) : h0 * (I + 1);
    const double f = (x - o0) / D0;
    xs[n].f = f; xs[n].s0 = x; xs[n].s1 = o1 + f * D1; ++I; ++n;
  }
  while (I > If) {
    const double x = DUAL ? h0 * (I + 0.5) : h0 * I;
    const double f = (x - o0) / D0;
    xs[n].f = f; xs[n].s0 = x; xs[n].s1 = o1 + f * D1; --I; ++n;
  }
  while (J < Jf) {
    const double y = DUAL ? h1 * (J + 1.5) : h1 * (J + 1);
    const double f = (y - o1) / D1;
    xs[n].f = f; xs[n].s0 = o0 + f * D0; xs[n].s1 = y; ++J; ++n;
  }
  while (J > Jf) {
    const double y = DUAL ? h1 * (J + 0.5) : h1 * J;
    const double f = (y - o1) / D1;
    xs[n].f = f; xs[n].s0 = o0 + f * D0; xs[n].s1 = y; --J; ++n;
  }
  xs[n++].f = 1.0;
  for (int a = 2; a < n - 1; ++a) {  // stable insertion sort of xs[1 .. n-2]
    Cross v = xs[a];
    int b = a;
    while (b > 1 && v.f < xs[b - 1].f) { xs[b] = xs[b - 1]; --b; }
    xs[b] = v;
  }
  int dest = 0;
  for (int k = 1; k < n; ++k)
    if (!(fabs(xs[dest].f - xs[k].f) < 1e-6)) xs[++dest] = xs[k];
  const int num = dest + 1;
  xs[0].s0 = o0; xs[0].s1 = o1;
  xs[num - 1].s0 = n0; xs[num - 1].s1 = n1;
  return num;
}

// Current of one straight segment a -> b (subSteps relative to the mesh
// origin) of a particle whose whole push covers the displacement dl (cells)
// and distance cov; sink(i, j, value) receives every contribution.
template <int ORDER, class Sink>
__device__ __forceinline__ void deposit_segment(int comp, double q, double a0, double a1, double b0, double b1,
                                                double ood0, double ood1, double oodt0, double oodt1,
                                                double dl0, double dl1, double cov, Sink &sink) {
  const double xi0 = a0 * ood0, xi1 = a1 * ood1;
  const double xf0 = b0 * ood0, xf1 = b1 * ood1;
  if (ORDER == 0) {
    // ZerothOrderShapeFunction.cpp:215-226 (X) and :279-290 (Y)
    const double c0 = (xi0 + xf0) * 0.5, c1 = (xi1 + xf1) * 0.5;
    const int I = (int)floor(c0), J = (int)floor(c1);
    if (comp == 0) {
      const double D0 = q * (xf0 - xi0) * oodt0;
      sink(I, J, D0 * (J + 1 - c1));
      sink(I, J + 1, D0 * (c1 - J));
    } else {
      const double D1 = q * (xf1 - xi1) * oodt1;
      sink(I, J, D1 * (I + 1 - c0));
      sink(I + 1, J, D1 * (c0 - I));
    }
    return;
  }
  const double sg0 = b0 - a0, sg1 = b1 - a1;
  const double tau = sqrt(sg0 * sg0 + sg1 * sg1) / cov;
  const double half = 0.5, onethird = 1.0 / 3.0;
  if (ORDER == 1) {
    // FirstOrderShapeFunction.cpp:225-248 with getCurrentX/Y (:540-683):
    // integral of S1 along the current times S2 across it, in tau.
    const double c0 = (xi0 + xf0) * 0.5, c1 = (xi1 + xf1) * 0.5;
    const int I = (int)floor(c0 + 0.5), J = (int)floor(c1 + 0.5);
    const double a_al = comp == 0 ? (I + 0.5 - xi0) : (J + 0.5 - xi1);   // along the current
    const double b_cr = comp == 0 ? (J - xi1) : (I - xi0);               // across it
    const double d_al = comp == 0 ? dl0 : dl1, d_cr = comp == 0 ? dl1 : dl0;
    const double cd = comp == 0 ? (q * oodt1) * dl0 : (q * oodt0) * dl1;
    const double onefourth = half * half;
    const double tp2 = tau * tau * half;
    const double tp3 = tp2 * tau * 2 * onethird;
    const double Am = a_al, Bm = -d_al * tau, A0 = 1.0 - a_al, B0 = d_al * tau;
    double A2[3], B2[3], C2[3];
    A2[0] = half * (half + b_cr) * (half + b_cr) * tau;
    B2[0] = -(half + b_cr) * d_cr * tp2;
    C2[0] = half * d_cr * d_cr * tp3;
    A2[1] = (0.75 - b_cr * b_cr) * tau;
    B2[1] = 2 * b_cr * d_cr * tp2;
    C2[1] = -d_cr * d_cr * tp3;
    A2[2] = half * (half - b_cr) * (half - b_cr) * tau;
    B2[2] = (half - b_cr) * d_cr * tp2;
    C2[2] = half * d_cr * d_cr * tp3;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const double sm = A2[t] + B2[t] + C2[t];
      const double m = half * A2[t] + onethird * B2[t] + onefourth * C2[t];
      const double jm = cd * ((Am + Bm) * sm - Bm * m);
      const double j0 = cd * ((A0 + B0) * sm - B0 * m);
      if (comp == 0) { sink(I - 1, J - 1 + t, jm); sink(I, J - 1 + t, j0); }
      else { sink(I - 1 + t, J - 1, jm); sink(I - 1 + t, J, j0); }
    }
  } else {
    // SecondOrderShapeFunction.cpp:226-251 with getCurrentX/Y (:583-826):
    // S2 along the current times S3 across it.
    const double c0 = 0.5 * (xi0 + xf0), c1 = 0.5 * (xi1 + xf1);
    const int I = (int)(long)floor(c0), J = (int)(long)floor(c1);
    const double tp2 = tau * tau / 2;
    const double tp3 = tp2 * tau * 2 / 3;
    const double tp4 = tp2 * tp2;
    const double onefourth = 0.25, onefifth = 0.2, onesixth = half * onethird;
    const double a = comp == 0 ? (I + 0.5 - xi0) : (J + 0.5 - xi1);
    const double b = comp == 0 ? (J - xi1) : (I - xi0);
    const double dl = comp == 0 ? dl0 : dl1, dl2 = dl * dl;
    const double de = comp == 0 ? dl1 : dl0;
    const double de2 = de * de, de3 = de2 * de;
    const double cd = comp == 0 ? (q * oodt1) * dl0 : (q * oodt0) * dl1;
    double sA[3], sB[3], sC[3];
    if (comp == 0) {
      sA[0] = half * (half + a) * (half + a); sC[0] = half * dl2 * tp2;
      sA[2] = half * (0.5 - a) * (0.5 - a);   sC[2] = half * dl2 * tp2;
    } else {
      sA[0] = (half + a) * (half + a) * half; sC[0] = dl2 * half * tp2;
      sA[2] = (half - a) * (half - a) * half; sC[2] = dl2 * half * tp2;
    }
    sB[0] = -(half + a) * dl * tau;
    sA[1] = 0.75 - a * a; sB[1] = 2 * a * dl * tau; sC[1] = -dl2 * tp2;
    sB[2] = (half - a) * dl * tau;
    double tA[4], tB[4], tC[4], tD[4];
    tA[0] = (1 + b) * (1 + b) * (1 + b) * onesixth * tau;
    tB[0] = -(1 + b) * (1 + b) * de * half * tp2;
    tC[0] = (1 + b) * de2 * half * tp3;
    tD[0] = -de3 * onesixth * tp4;
    tA[1] = (4 - 3 * b * b * (2 + b)) * onesixth * tau;
    tB[1] = b * de * (3 * b + 4) * half * tp2;
    tC[1] = -de2 * (2 + 3 * b) * half * tp3;
    tD[1] = de3 * half * tp4;
    tA[2] = (4 - 3 * (b + 1) * (b + 1) * (1 - b)) * onesixth * tau;
    tB[2] = (1 - 2 * b - 3 * b * b) * de * half * tp2;
    tC[2] = (1 + 3 * b) * de2 * half * tp3;
    tD[2] = -de3 * half * tp4;
    tA[3] = -b * b * b * onesixth * tau;
    tB[3] = b * b * de * half * tp2;
    tC[3] = -b * de2 * half * tp3;
    tD[3] = de3 * onesixth * tp4;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        const double v = cd * ((sA[u] + sB[u] + sC[u]) * (tD[t] + tC[t] + tB[t] + tA[t])
                               + (sC[u] * (tD[t] - tA[t]) - sB[u] * tB[t]) * onethird
                               + (sC[u] * tC[t] - sB[u] * tD[t]) * onefifth
                               - sB[u] * tC[t] * onefourth - sB[u] * tA[t] * half);
        if (comp == 0) sink(I - 1 + u, J - 1 + t, v);
        else sink(I - 1 + t, J - 1 + u, v);
      }
    }
  }
}

// Segments of a push with at most one border crossing per axis (|move| < one
// cell, i.e. CFL <= 1), enumerated without an array: the same points, order,
// 1e-6 merging and end-point substitution as border_crossings, kept in
// registers.  Returns false when a particle crosses more borders; the caller
// then takes the general path.
// floor(v / h - shift) with the IEEE quotient, as the reference computes it.
// v * (1/h) is within a few ulps of the rounded quotient, so its floor is the
// same integer unless it lies within 1e-9 of an integer; only then is the
// division carried out.
__device__ __forceinline__ int floor_div(double v, double h, double ooh, double shift) {
  const double a = v * ooh - shift;
  const double f = floor(a);
  if (a - f > 1e-9 && (f + 1.0) - a > 1e-9) return (int)f;
  return (int)floor(v / h - shift);
}

template <bool DUAL, class Seg>
__device__ __forceinline__ bool segments_fast(double o0, double o1, double n0, double n1, double h0, double h1,
                                              Seg &&seg) {
  const double sh = DUAL ? 0.5 : 0.0, ooh0 = 1.0 / h0, ooh1 = 1.0 / h1;
  const int Ii = floor_div(o0, h0, ooh0, sh), Ji = floor_div(o1, h1, ooh1, sh);
  const int If = floor_div(n0, h0, ooh0, sh), Jf = floor_div(n1, h1, ooh1, sh);
  if (abs(If - Ii) > 1 || abs(Jf - Ji) > 1) return false;
  const double D0 = n0 - o0, D1 = n1 - o1;
  const bool hx = If != Ii, hy = Jf != Ji;
  double fx = 0, x0 = 0, x1 = 0, fy = 0, y0 = 0, y1 = 0;
  if (hx) {
    x0 = If > Ii ? (DUAL ? h0 * (Ii + 1.5) : h0 * (Ii + 1)) : (DUAL ? h0 * (Ii + 0.5) : h0 * Ii);
    fx = (x0 - o0) / D0;
    x1 = o1 + fx * D1;
  }
  if (hy) {
    y1 = Jf > Ji ? (DUAL ? h1 * (Ji + 1.5) : h1 * (Ji + 1)) : (DUAL ? h1 * (Ji + 0.5) : h1 * Ji);
    fy = (y1 - o1) / D1;
    y0 = o0 + fy * D0;
  }
  const bool ysFirst = hy && (!hx || fy < fx);  // stable order: x crossing first on ties
  const int nint = (hx ? 1 : 0) + (hy ? 1 : 0);
  double af = 0.0, as0 = o0, as1 = o1;           // start of the pending segment
  double bf = 0.0, bs0 = 0.0, bs1 = 0.0;         // last kept point, not yet emitted
  bool hasb = false;
  for (int c = 0; c <= nint; ++c) {
    double cf, cs0, cs1;
    if (c == nint) { cf = 1.0; cs0 = n0; cs1 = n1; }
    else {
      const bool pickY = (c == 0) ? ysFirst : !ysFirst;
      cf = pickY ? fy : fx; cs0 = pickY ? y0 : x0; cs1 = pickY ? y1 : x1;
    }
    const double lf = hasb ? bf : af;
    if (!(fabs(lf - cf) < 1e-6)) {
      if (hasb) { seg(as0, as1, bs0, bs1); af = bf; as0 = bs0; as1 = bs1; }
      hasb = true; bf = cf; bs0 = cs0; bs1 = cs1;
    }
  }
  seg(as0, as1, n0, n1);  // the last kept point carries the new position
  return true;
}

// Calls sink(i, j, value) for every current contribution of one particle
// moving old -> new (absolute positions; the mesh origin is org; indices are
// mesh cells).  Returns false on a crossing overflow.  (h0, h1) is the
// spacing of the coordinates given; (jh0, jh1) the physical spacing that
// scales the current.  The FP64 path passes physical positions with
// jh = h; FP32 mode passes positions in cells (h = 1).  Ratios of lengths
// along one straight move do not depend on the units, so both give the
// same current up to rounding.
template <int ORDER, class Sink>
__device__ __forceinline__ bool deposit_particle(int comp, double q, double ao0, double ao1, double an0,
                                                 double an1, double org0, double org1, double h0, double h1,
                                                 double jh0, double jh1, double dt, Sink &&sink) {
  // crossings are taken relative to the mesh origin (utils.hh:435-436)
  const double o0 = ao0 - org0, o1 = ao1 - org1, n0 = an0 - org0, n1 = an1 - org1;
  const double ood0 = 1.0 / h0, ood1 = 1.0 / h1;
  double oodt0, oodt1, dl0 = 0.0, dl1 = 0.0, cov = 0.0;
  if (ORDER == 0) {
    oodt0 = 1.0 / (jh1 * dt); oodt1 = 1.0 / (jh0 * dt);
  } else {
    // the full displacement uses the absolute positions (R - oldR)
    const double Dx0 = an0 - ao0, Dx1 = an1 - ao1;
    cov = sqrt(Dx0 * Dx0 + Dx1 * Dx1);
    if (cov == 0.0) return true;  // a particle that does not move carries no current
    oodt0 = (1.0 / jh0) / dt; oodt1 = (1.0 / jh1) / dt;
    dl0 = Dx0 * ood0; dl1 = Dx1 * ood1;
  }
  auto seg = [&](double a0, double a1, double b0, double b1) {
    deposit_segment<ORDER>(comp, q, a0, a1, b0, b1, ood0, ood1, oodt0, oodt1, dl0, dl1, cov, sink);
  };
  if (segments_fast<ORDER == 1>(o0, o1, n0, n1, h0, h1, seg)) return true;
  Cross xs[kMaxCross];
  const int n = border_crossings<ORDER == 1>(xs, o0, o1, n0, n1, h0, h1);
  if (n < 0) return false;
  for (int k = 0; k + 1 < n; ++k) seg(xs[k].s0, xs[k].s1, xs[k + 1].s0, xs[k + 1].s1);
  return true;
}

// Warp-aggregated fixed-point add: lanes that target the same cell combine
// their values first (three exact 22-bit-chunk reductions that together form
// the 64-bit two's-complement sum), then one lane per cell does the atomic.
// k < 0 marks a contribution that falls outside the target and is dropped.
__device__ __forceinline__ void warp_add(unsigned long long *acc, int k, long long v) {
  const unsigned act = __activemask();
  const unsigned peers = __match_any_sync(act, k);
  const unsigned long long u = (unsigned long long)v;
  const unsigned c0 = __reduce_add_sync(peers, (unsigned)(u & 0x3FFFFFull));
  const unsigned c1 = __reduce_add_sync(peers, (unsigned)((u >> 22) & 0x3FFFFFull));
  const unsigned c2 = __reduce_add_sync(peers, (unsigned)(u >> 44));
  if (k >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) {
    const unsigned long long sum =
        (unsigned long long)c0 + ((unsigned long long)c1 << 22) + ((unsigned long long)c2 << 44);
    atomicAdd(&acc[k], sum);
  }
}

// Vertex charge shape of one particle (getChargeDensityImpl and
// getChargeDensityDiffImpl of ZerothOrderShapeFunction.cpp:355-366,
// FirstOrderShapeFunction.cpp:391-416, SecondOrderShapeFunction.cpp:408-441):
// add(i, j, w) for every vertex weight w of charge qq at (X, Y).
template <int ORDER, class Add>
__device__ __forceinline__ void charge_shape(double X, double Y, double qq, double org0, double org1, double h0,
                                             double h1, Add &&add) {
  if (ORDER == 0) {
    const double a = (X - org0) / h0, b = (Y - org1) / h1;
    const int I = (int)floor(a), J = (int)floor(b);
    const double t0 = a - I, t1 = b - J;
    add(I, J, (1.0 - t0) * (1.0 - t1) * qq);
    add(I + 1, J, t0 * (1.0 - t1) * qq);
    add(I, J + 1, (1.0 - t0) * t1 * qq);
    add(I + 1, J + 1, t0 * t1 * qq);
  } else if (ORDER == 1) {
    const double n0 = (X - org0) / h0, n1 = (Y - org1) / h1;
    const int I = (int)floor(n0 + 0.5), J = (int)floor(n1 + 0.5);
    const double a = n0 - I, b = n1 - J;
    const double sxm = qq * (0.5 - a) * (0.5 - a) * 0.5, sxp = qq * (0.5 + a) * (0.5 + a) * 0.5;
    const double sx = qq - sxm - sxp;
    const double sym = (0.5 - b) * (0.5 - b) * 0.5, syp = (0.5 + b) * (0.5 + b) * 0.5;
    const double sy = 1.0 - sym - syp;
    const double wx[3] = {sxm, sx, sxp}, wy[3] = {sym, sy, syp};
#pragma unroll
    for (int bb = 0; bb < 3; ++bb)
#pragma unroll
      for (int aa = 0; aa < 3; ++aa) add(I - 1 + aa, J - 1 + bb, wx[aa] * wy[bb]);
  } else {
    const double n0 = (X - org0) / h0, n1 = (Y - org1) / h1;
    const int I = (int)floor(n0), J = (int)floor(n1);
    const double a = n0 - I, b = n1 - J;
    const double s6 = 1.0 / 6.0;
    const double wx[4] = {s6 * ((1.0 - a) * (1.0 - a) * (1.0 - a)), s6 * (4.0 - 3.0 * a * a * (2.0 - a)),
                          s6 * (4.0 - 3.0 * (1.0 - a) * (1.0 - a) * (1.0 + a)), s6 * (a * a * a)};
    const double wy[4] = {s6 * ((1.0 - b) * (1.0 - b) * (1.0 - b)), s6 * (4.0 - 3.0 * b * b * (2.0 - b)),
                          s6 * (4.0 - 3.0 * (1.0 - b) * (1.0 - b) * (1.0 + b)), s6 * (b * b * b)};
#pragma unroll
    for (int bb = 0; bb < 4; ++bb)
#pragma unroll
      for (int aa = 0; aa < 4; ++aa) add(I - 1 + aa, J - 1 + bb, qq * wx[aa] * wy[bb]);
  }
}

}  // namespace csrst
