// FP32-mode current deposit with exact charge conservation.
//
// The reference deposits the current of every straight move old -> new as
// the path integral of its shape function (Zeroth/First/SecondOrderShape-
// Function: the segments between cell or dual-cell crossings, closed forms in
// the segment fraction tau).  That current is charge conserving: with the
// matching vertex charge shape S, rho(new) - rho(old) + dt div J = 0 holds
// per particle in exact arithmetic.  Evaluated in FP32 the identity would
// only hold to ~1e-7.  This file keeps it exact, in 64-bit integers, while the
// path integral itself runs in FP32:
//
//  1. charge: the 1D charge weights of both end points come from their exact
//     representation (integer cell + FP32 offset) in FP64 and are quantised
//     to the fixed-point unit, rows first: R(j) = round(K Sy(j)) with one
//     entry set so that the row totals sum to K exactly, then
//     rho(i, j) = round(R(j) Sx(i)) with one entry set so that every row sums
//     to R(j).  K = q * scale.  Every particle carries exactly K.
//  2. Fy: the reference's y-current path integral in FP32 (flux units,
//     Fy = Jy dt hx / q), quantised; per face row its total is corrected in
//     one entry to the integer flux that the row charges force:
//     Y(r) = Y(r - 1) - (R_new(r) - R_old(r)).
//  3. Fx: from continuity, row by row from the left edge of the stencil box:
//     Fx(c, r) = Fx(c - 1, r) - (rho_new - rho_old)(c, r) - Fy(c, r) + Fy(c, r - 1).
//     Because every row's charge change and y fluxes sum to zero (2.), Fx
//     ends at zero on the box's right edge.
//
// So rho_new - rho_old + div F = 0 holds exactly in integers for the charge
// the particle carries, which is the FP64 charge shape to one fixed-point
// unit per weight.  In exact arithmetic step 3 reproduces the reference's
// path-integral Fx exactly (continuity determines Fx from Fy and rho), so the
// FP32 rounding of Fy moves Fx only by ~1e-7 of |Fy|, which is small against
// |Fx| for bunches moving along x.  A push deposits one component (TE/TM
// split): comp 0 emits Fx, comp 1 the corrected Fy; both run steps 1-2
// identically, so the two components of one move are consistent.
//
// Stencil box: the union of both end points' charge stencils, (S + 1) x
// (S + 1) vertices for a move of at most one cell per axis (S = 2, 3, 4 for
// shape orders 0, 1, 2).  Indices below are relative to the particle's old
// cell (ci, cj); a sink receives (i, j, value) in those coordinates: Fx at the
// x-face between vertices i and i + 1 of row j, Fy at the y-face between rows
// j and j + 1 of column i (the reference's Jx(i, j), Jy(i, j) elements).
#pragma once

// Plain arithmetic only (no CUDA runtime types), so that the host can compile
// this header too (the CPU test of the construction defines __device__,
// __forceinline__ and the two rounding conversions).
#include <math.h>
#include <stdlib.h>

namespace csrst {

template <int ORDER>
struct Flux32Shape;
// S: charge stencil width; OFF: first stencil vertex relative to the base
// index; DUAL: the path integral splits at dual-cell (half-integer) borders.
template <>
struct Flux32Shape<0> { static constexpr int S = 2, OFF = 0, CEN = 0; static constexpr bool DUAL = false; };
template <>
struct Flux32Shape<1> { static constexpr int S = 3, OFF = -1, CEN = 1; static constexpr bool DUAL = true; };
template <>
struct Flux32Shape<2> { static constexpr int S = 4, OFF = -1, CEN = 1; static constexpr bool DUAL = false; };

// Base index (relative to the cell of the offset) and 1D charge weights of
// the offset o (cells): ZerothOrderShapeFunction.cpp:355-366 (CIC),
// FirstOrderShapeFunction.cpp:391-416 (quadratic), SecondOrderShapeFunction
// .cpp:408-441 (cubic), in FP64 on the exact offset.
template <int ORDER>
__device__ __forceinline__ int charge_weights(float o, double *w) {
  const double n = (double)o;
  if (ORDER == 0) {
    const double f = floor(n), t = n - f;
    w[0] = 1.0 - t; w[1] = t;
    return (int)f;
  } else if (ORDER == 1) {
    const double f = floor(n + 0.5), a = n - f;
    w[0] = 0.5 * (0.5 - a) * (0.5 - a);
    w[2] = 0.5 * (0.5 + a) * (0.5 + a);
    w[1] = 1.0 - w[0] - w[2];
    return (int)f;
  } else {
    const double f = floor(n), a = n - f, b = 1.0 - a, s6 = 1.0 / 6.0;
    w[0] = s6 * (b * b * b);
    w[1] = s6 * (4.0 - 3.0 * a * a * (2.0 - a));
    w[2] = s6 * (4.0 - 3.0 * b * b * (1.0 + a));
    w[3] = s6 * (a * a * a);
    return (int)f;
  }
}

// Quantised weights: out[k] = round(T w[k]) except out[CEN] = T - the others.
template <int ORDER>
__device__ __forceinline__ void quantise(const double *w, double T, long long Tint, long long *out) {
  constexpr int S = Flux32Shape<ORDER>::S, CEN = Flux32Shape<ORDER>::CEN;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < S; ++k)
    if (k != CEN) { out[k] = __double2ll_rn(T * w[k]); s += out[k]; }
  out[CEN] = Tint - s;
}

// FP32 y-current path integral of one segment p -> e (cells, old-cell
// relative) with vertex (I, J) and segment fraction tau of a move of total
// displacement (d0, d1), in flux units Fy = Jy dt hx / q:
// ZerothOrderShapeFunction.cpp:279-290, FirstOrderShapeFunction.cpp:629-683
// (getCurrentY), SecondOrderShapeFunction.cpp:583-826 (Y branch).
// v[t][k]: the contribution to the face of column I - 1 + t (CIC: I + t) and
// face row J - 1 + k (CIC: J), t < S across, k < S - 1 along.
template <int ORDER>
__device__ __forceinline__ void fy_segment(float p0, float p1, float e0, float e1, int I, int J, float tau, float d0,
                                           float d1, float (&v)[Flux32Shape<ORDER>::S][Flux32Shape<ORDER>::S - 1]) {
  if (ORDER == 0) {
    const float c0 = 0.5f * (p0 + e0);
    const float D = tau * d1;  // e1 - p1 without the cancellation of two O(1) coordinates
    v[0][0] = D * ((float)(I + 1) - c0);
    v[1][0] = D * (c0 - (float)I);
  } else if (ORDER == 1) {
    const float half = 0.5f, third = 1.0f / 3.0f, quarter = 0.25f;
    const float a = (float)J + half - p1;   // along y: start to the face J + 1/2
    const float b = (float)I - p0;          // across x: vertex minus start
    const float tp2 = tau * tau * half, tp3 = tp2 * tau * (2.0f * third);
    const float Bm = -d1 * tau, Am = a, A0 = 1.0f - a, B0 = d1 * tau;
    const float A2[3] = {half * (half + b) * (half + b) * tau, (0.75f - b * b) * tau,
                         half * (half - b) * (half - b) * tau};
    const float B2[3] = {-(half + b) * d0 * tp2, 2.0f * b * d0 * tp2, (half - b) * d0 * tp2};
    const float C2[3] = {half * d0 * d0 * tp3, -d0 * d0 * tp3, half * d0 * d0 * tp3};
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const float sm = A2[t] + B2[t] + C2[t];
      const float m = half * A2[t] + third * B2[t] + quarter * C2[t];
      v[t][0] = d1 * ((Am + Bm) * sm - Bm * m);
      v[t][1] = d1 * ((A0 + B0) * sm - B0 * m);
    }
  } else {
    const float half = 0.5f, third = 1.0f / 3.0f, quarter = 0.25f, fifth = 0.2f, sixth = 1.0f / 6.0f;
    const float tp2 = tau * tau * half, tp3 = tp2 * tau * (2.0f * third), tp4 = tp2 * tp2;
    const float a = (float)J + half - p1, b = (float)I - p0;
    const float dl = d1, dl2 = dl * dl, de = d0, de2 = de * de, de3 = de2 * de;
    const float sA[3] = {(half + a) * (half + a) * half, 0.75f - a * a, (half - a) * (half - a) * half};
    const float sB[3] = {-(half + a) * dl * tau, 2.0f * a * dl * tau, (half - a) * dl * tau};
    const float sC[3] = {dl2 * half * tp2, -dl2 * tp2, dl2 * half * tp2};
    const float bb = 1.0f + b;
    const float tA[4] = {bb * bb * bb * sixth * tau, (4.0f - 3.0f * b * b * (2.0f + b)) * sixth * tau,
                         (4.0f - 3.0f * bb * bb * (1.0f - b)) * sixth * tau, -b * b * b * sixth * tau};
    const float tB[4] = {-bb * bb * de * half * tp2, b * de * (3.0f * b + 4.0f) * half * tp2,
                         (1.0f - 2.0f * b - 3.0f * b * b) * de * half * tp2, b * b * de * half * tp2};
    const float tC[4] = {bb * de2 * half * tp3, -de2 * (2.0f + 3.0f * b) * half * tp3,
                         (1.0f + 3.0f * b) * de2 * half * tp3, -b * de2 * half * tp3};
    const float tD[4] = {-de3 * sixth * tp4, de3 * half * tp4, -de3 * half * tp4, de3 * sixth * tp4};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const float st = tD[t] + tC[t] + tB[t] + tA[t];
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        const float w = (sA[u] + sB[u] + sC[u]) * st + (sC[u] * (tD[t] - tA[t]) - sB[u] * tB[t]) * third +
                        (sC[u] * tC[t] - sB[u] * tD[t]) * fifth - sB[u] * tC[t] * quarter - sB[u] * tA[t] * half;
        v[t][u] = dl * w;
      }
    }
  }
}

// out[k] = in[k - sh] (zero outside in's N entries), sh in {0, 1}: an array
// moved into the stencil box's frame with compile-time indices only, so
// that it stays in registers.
template <int N, int M, class T>
__device__ __forceinline__ void shift_into(const T (&in)[N], bool sh, T (&out)[M]) {
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const T lo = k < N ? in[k] : T(0);
    const T hi = (k >= 1 && k - 1 < N) ? in[k - 1] : T(0);
    out[k] = sh ? hi : lo;
  }
}

// Border between base indices k and k + 1 of a path-integral split:
// k + 1 for cell borders, k + 1/2 for dual-cell borders.
template <bool DUAL>
__device__ __forceinline__ float split_border(int k) { return DUAL ? (float)k + 0.5f : (float)(k + 1); }

// Fraction of the move a + f d at coordinate X, clamped to [0, 1] (0 when
// the move has no extent along the axis).
__device__ __forceinline__ float cross_fraction(float X, float a, float d) {
  if (d == 0.0f) return 0.0f;
  return fminf(fmaxf((X - a) / d, 0.0f), 1.0f);
}

// Base indices of a move's end points (old-cell relative), for choosing the
// deposit's form before running it.
template <int ORDER>
__device__ __forceinline__ int base_index(float o) {
  return (int)floorf(ORDER == 1 ? o + 0.5f : o);
}

// The charge-conserving deposit of one move (see the top of the file).
// (a0, a1): start offset in cells from the old cell (ci, cj), any value;
// (dc0, dc1) = new cell - old cell, (b0, b1): end offset in the new cell;
// K = q * scale, Kint = its integer value.  COMP selects the emitted
// component; sink(i, j, v) gets old-cell-relative Jx / Jy indices.
// FAST: the move keeps its y base index and advances its x base index by 0
// or 1 (a bunch moving along +x at CFL <= 1, nearly every particle); the
// stencil box then has S + 1 columns and S rows at compile-time offsets.
// The caller checks that before choosing FAST (base_index).
// Returns false when the move spans more than one base index on an axis
// (more than one cell for CFL <= 1); nothing is emitted then.
template <int ORDER, int COMP, bool FAST, class Sink>
__device__ __forceinline__ bool flux_particle(float a0, float a1, int dc0, int dc1, float b0, float b1, double K,
                                              long long Kint, Sink &&sink) {
  using SH = Flux32Shape<ORDER>;
  constexpr int S = SH::S, OFF = SH::OFF, BX = S + 1, BY = FAST ? S : S + 1, NSEG = FAST ? 2 : 3;
  // 1. charge weights of both end points and their base indices (old-cell
  //    relative); the box starts at the lower base index of each axis
  double wAy[S], wBy[S];
  const int JA = charge_weights<ORDER>(a1, wAy);
  const int JB = dc1 + charge_weights<ORDER>(b1, wBy);
  if (!FAST && abs(JB - JA) > 1) return false;
  const int jmin = FAST ? JA : (JA < JB ? JA : JB);
  const bool syA = FAST ? false : JA != jmin, syB = FAST ? false : JB != jmin;
  long long RA[BY], RB[BY];  // row totals in the box frame
  {
    long long r[S];
    quantise<ORDER>(wAy, K, Kint, r);
    shift_into(r, syA, RA);
    quantise<ORDER>(wBy, K, Kint, r);
    shift_into(r, syB, RB);
  }
  double wAx[S], wBx[S];
  const int IA = charge_weights<ORDER>(a0, wAx);
  const int IB = dc0 + charge_weights<ORDER>(b0, wBx);
  if (!FAST && abs(IB - IA) > 1) return false;
  const int imin = FAST ? IA : (IA < IB ? IA : IB);
  const bool sxA = FAST ? false : IA != imin, sxB = IB != imin;
  const int ib = imin + OFF, jb = jmin + OFF;

  // 2. y-current path integral in FP32 over the segments between crossings,
  //    each segment's values moved into the box frame by its vertex's offset
  //    from the lower base index.  The displacement comes from the exact end
  //    points in FP64 (a difference of O(1) FP32 coordinates would carry an
  //    absolute error of their ulp).
  const float d0 = (float)((double)dc0 + ((double)b0 - (double)a0));
  const float d1 = (float)((double)dc1 + ((double)b1 - (double)a1));
  float fy[BX][BY - 1];
#pragma unroll
  for (int c = 0; c < BX; ++c)
#pragma unroll
    for (int r = 0; r < BY - 1; ++r) fy[c][r] = 0.0f;
  {
    const bool hx = IB != IA, hy = FAST ? false : JB != JA;
    const float fx = hx ? cross_fraction(split_border<SH::DUAL>(imin), a0, d0) : 2.0f;
    const float fyc = hy ? cross_fraction(split_border<SH::DUAL>(jmin), a1, d1) : 2.0f;
    // up to three segments in order of the crossing fractions; the vertex of
    // the path switches from A's to B's index at each crossing
    const float f1 = fminf(fx, fyc), f2 = fmaxf(fx, fyc);
    const bool xfirst = fx <= fyc;
    float ts = 0.0f;
    int I = IA, J = JA;
#pragma unroll
    for (int sg = 0; sg < NSEG; ++sg) {
      const float te = sg == NSEG - 1 ? 1.0f : sg == 0 ? fminf(f1, 1.0f) : fminf(f2, 1.0f);
      const float tau = te - ts;
      if (tau > 0.0f) {
        float v[S][S - 1];
        fy_segment<ORDER>(a0 + ts * d0, a1 + ts * d1, a0 + te * d0, a1 + te * d1, I, J, tau, d0, d1, v);
        float w[S][BY - 1];  // moved along the face rows
#pragma unroll
        for (int t = 0; t < S; ++t) shift_into(v[t], FAST ? false : J != jmin, w[t]);
        const bool cx = I != imin;
#pragma unroll
        for (int c = 0; c < BX; ++c)
#pragma unroll
          for (int r = 0; r < BY - 1; ++r) {
            const float lo = c < S ? w[c][r] : 0.0f, hi = c >= 1 ? w[c - 1][r] : 0.0f;
            fy[c][r] += cx ? hi : lo;
          }
      }
      if (sg == 0 && f1 <= 1.0f) { if (xfirst) I = IB; else J = JB; }
      if (sg == 1 && f2 <= 1.0f) { if (xfirst) J = JB; else I = IB; }
      ts = te;
    }
  }

  // 3. quantised Fy with the row totals set by the row charges; Fx by continuity
  const float Kf = (float)K;
  const int cstar = IA - imin - OFF;  // the box column of A's base vertex
  long long Y = 0;                    // total y flux of the face row below
  long long fyPrev[BX];               // corrected Fy of the face row below
#pragma unroll
  for (int c = 0; c < BX; ++c) fyPrev[c] = 0;
#pragma unroll
  for (int r = 0; r < BY; ++r) {
    long long fyRow[BX];
    if (r < BY - 1) {
      Y -= RB[r] - RA[r];
      long long sum = 0;
#pragma unroll
      for (int c = 0; c < BX; ++c) { fyRow[c] = __float2ll_rn(Kf * fy[c][r]); sum += fyRow[c]; }
#pragma unroll
      for (int c = 0; c < BX; ++c)
        if (c == cstar) fyRow[c] += Y - sum;
      if (COMP == 1) {
#pragma unroll
        for (int c = 0; c < BX; ++c)
          if (fyRow[c] != 0) sink(ib + c, jb + r, fyRow[c]);
      }
    } else {
#pragma unroll
      for (int c = 0; c < BX; ++c) fyRow[c] = 0;
    }
    if (COMP == 0) {
      // this row's charges in the box frame, each row summing to its R exactly
      long long qA[BX], qB[BX];
      {
        long long t[S];
        quantise<ORDER>(wAx, (double)RA[r], RA[r], t);
        shift_into(t, sxA, qA);
        quantise<ORDER>(wBx, (double)RB[r], RB[r], t);
        shift_into(t, sxB, qB);
      }
      long long fx = 0;
#pragma unroll
      for (int c = 0; c < BX - 1; ++c) {
        fx -= (qB[c] - qA[c]) + fyRow[c] - fyPrev[c];
        if (fx != 0) sink(ib + c, jb + r, fx);
      }
    }
#pragma unroll
    for (int c = 0; c < BX; ++c) fyPrev[c] = fyRow[c];
  }
  return true;
}

}  // namespace csrst
