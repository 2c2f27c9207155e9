// Field kernels: the TE/TM split Yee update on the static mesh and on the
// moving window, the conformal cut-cell corrections, the window <-> static
// strip exchange and the window move.  Every kernel is a template on the
// field type: double on the FP64 path (the reference's arithmetic, operation
// for operation), float in FP32 mode.
//
// One sub-step (half-H, Ex or Ey) is one launch: the static sweep over the
// masked regular cells, the sparse cut-cell list and the window cells are
// disjoint sets of elements that read only fields the launch does not write,
// so they run as three block ranges of the same grid
// (TETMSolver.hh:142-206, :241-261; SCBoundaryCondition.hh:391-431).
// The strip exchange that follows each sub-step is a pure copy between
// disjoint element sets (Communicator::exchangeBoundaries,
// Communicator.hh:575-876), launched separately because the next sub-step
// reads what it writes.
#include <cuda.h>

#include <algorithm>

#include "kernels.cuh"
#include "tma.cuh"

namespace csrst {

// The static sweep works on 16-byte vectors of a plane row: a thread holds
// storage columns c .. c + V - 1 of row j (V = 4 floats or 2 doubles), which
// are the cells i = c - 1 .. c + V - 2 (storage column 0 is the left guard).
// Plane rows start 256-byte aligned (pitch rounded up), so every vector load
// is aligned.  A warp lies in one row segment of 32 consecutive vectors (tx is
// a multiple of 32): the one element a cell needs from the next or previous
// vector comes from the neighbouring lane by shuffle, the warp's end lanes
// load it.  Vectors with c <= Nx + 1 are loaded (the right guard column is
// read); cells 0 <= i < Nx on the inside mask are updated with the same
// arithmetic as one cell per thread, and written back as a vector when all
// of a vector's cells are, else element by element (the cut-cell blocks of
// the same launch update the cells off the mask).
template <class T>
struct alignas(16) Vec16 {
  static constexpr int N = 16 / sizeof(T);
  T v[N];
};
template <class T>
__device__ __forceinline__ Vec16<T> ld16(const T *p) { return *reinterpret_cast<const Vec16<T> *>(p); }
template <class T>
__device__ __forceinline__ void st16(T *p, const Vec16<T> &r) { *reinterpret_cast<Vec16<T> *>(p) = r; }

// Storage column c and row j of thread t in static block b; false: no row.
template <class T>
__device__ __forceinline__ bool static_vec(const FieldArgsT<T> &a, int b, int &c, int &j) {
  constexpr int V = Vec16<T>::N;
  c = (b % a.tilesX) * a.tx * V + (threadIdx.x % a.tx) * V;
  j = (b / a.tilesX) * a.ty + threadIdx.x / a.tx;
  return j < a.Ny;  // uniform over the warp
}

// Inside-mask bits of the cells i = c - 1 + e of row j that are on the mesh
// (and, with absorbing layers, outside them: those cells have their own
// block range).
template <class T>
__device__ __forceinline__ unsigned static_mask(const FieldArgsT<T> &a, int c, int j) {
  constexpr int V = Vec16<T>::N;
  unsigned m = 0;
  const uint8_t *row = a.mask + (size_t)j * a.Nx;
  int lo = 0, hi = a.Nx;
  if (a.pml_rows) { const int2 r = a.pml_rows[j]; lo = r.x; hi = r.y; }
#pragma unroll
  for (int e = 0; e < V; ++e) {
    const int i = c - 1 + e;
    if (i >= lo && i < hi && row[i]) m |= 1u << e;
  }
  return m;
}

template <class T>
__device__ __forceinline__ void store_masked(T *p, const Vec16<T> &r, unsigned m) {
  constexpr int V = Vec16<T>::N;
  if (m == (1u << V) - 1) {
    st16(p, r);
  } else {
#pragma unroll
    for (int e = 0; e < V; ++e)
      if (m >> e & 1u) p[e] = r.v[e];
  }
}

template <class T>
__device__ __forceinline__ void half_h_static(const FieldArgsT<T> &a, int b) {
  constexpr int V = Vec16<T>::N;
  int c, j;
  if (!static_vec(a, b, c, j)) return;
  const bool live = c <= a.Nx + 1;
  const unsigned m = live ? static_mask(a, c, j) : 0u;  // in flight with the plane loads
  T *hxp = &a.Hx.at(c - 1, j), *hyp = &a.Hy.at(c - 1, j);
  Vec16<T> ey{}, ex0{}, ex1{}, hx{}, hy{};
  if (live) {
    ey = ld16(&a.Ey.at(c - 1, j));
    ex0 = ld16(&a.Ex.at(c - 1, j));
    ex1 = ld16(&a.Ex.at(c - 1, j + 1));
    hx = ld16(hxp);
    hy = ld16(hyp);
  }
  T eyn = __shfl_down_sync(0xffffffffu, ey.v[0], 1);
  if (!m) return;
  if ((threadIdx.x & 31) == 31 && c + V <= a.Nx + 1) eyn = a.Ey.at(c + V - 1, j);
#pragma unroll
  for (int e = 0; e < V; ++e) {
    const T ey1 = e + 1 < V ? ey.v[e + 1 < V ? e + 1 : 0] : eyn;
    hx.v[e] = hx.v[e] - a.chx * (ey1 - ey.v[e]);
    hy.v[e] = hy.v[e] + a.chy * (ex1.v[e] - ex0.v[e]);
  }
  store_masked(hxp, hx, m);
  store_masked(hyp, hy, m);
}

// Window cell k (x fastest) of the half H sub-step.
template <class T>
__device__ __forceinline__ void window_h(const FieldArgsT<T> &a, int k) {
  const int i = k % a.L0, j = k / a.L0;
  T &hx = a.mHx.at(i, j), &hy = a.mHy.at(i, j);
  hx = hx - a.chx * (a.mEy.at(i + 1, j) - a.mEy.at(i, j));
  hy = hy + a.chy * (a.mEx.at(i, j + 1) - a.mEx.at(i, j));
}

// Window cell k of the E sub-step: the window current comes from the
// fixed-point accumulator of the last push, which is converted, stored for
// diagnostics and cleared for the next deposit.
template <class T, int COMP>
__device__ __forceinline__ void window_e(const FieldArgsT<T> &a, int k) {
  const int i = k % a.L0, j = k / a.L0;
  const T J = (T)((double)(long long)a.acc[k] * a.acc_inv);
  a.acc[k] = 0ull;
  if (COMP == 0) {
    a.mJx.at(i, j) = J;
    T &e = a.mEx.at(i, j);
    e = e + (a.kex * (a.mHx.at(i, j) - a.mHx.at(i, j - 1) + a.mHy.at(i, j) - a.mHy.at(i, j - 1)) - a.dteps * J);
  } else {
    a.mJy.at(i, j) = J;
    T &e = a.mEy.at(i, j);
    e = e - (a.key * (a.mHx.at(i, j) - a.mHx.at(i - 1, j) + a.mHy.at(i, j) - a.mHy.at(i - 1, j)) + a.dteps * J);
  }
}

// Half H update (first and third sub-step), block b of the sub-step grid.
// Static blocks cover the mesh in tiles of tx x ty vectors (tx * ty = 256
// threads, tx a multiple of 32; the shape is a tuning parameter).
template <class T>
__device__ __forceinline__ void half_h_body(const FieldArgsT<T> &a, int b) {
  if (b < a.nbS) {
    half_h_static(a, b);
  } else if (b < a.nbS + a.nbC) {
    const int k = (b - a.nbS) * blockDim.x + threadIdx.x;
    if (k >= a.ncells) return;
    const CutCellDev c = a.cells[k];
    const T n0 = (T)c.n0, n1 = (T)c.n1, l0 = (T)c.l0, l1 = (T)c.l1, area = (T)c.area;
    const T u0 = a.mhx * (n1 * a.Ey.at(c.i + 1, c.j) - l1 * a.Ey.at(c.i, c.j)) / area;
    const T u1 = a.mhy * (n0 * a.Ex.at(c.i, c.j + 1) - l0 * a.Ex.at(c.i, c.j)) / area;
    a.Hx.at(c.i, c.j) += u0;
    a.Hy.at(c.i, c.j) += u1;
  } else if (b < a.nbS + a.nbC + a.nbP) {
    const int k = (b - a.nbS - a.nbC) * blockDim.x + threadIdx.x;
    if (k >= a.npml) return;
    const PmlCellT<T> c = a.pml[k];
    T *ps = a.psi + 4 * (size_t)k;
    const T dey = a.Ey.at(c.i + 1, c.j) - a.Ey.at(c.i, c.j);
    const T dex = a.Ex.at(c.i, c.j + 1) - a.Ex.at(c.i, c.j);
    const T p0 = c.bhx * ps[0] + c.ahx * dey, p1 = c.bhy * ps[1] + c.ahy * dex;
    ps[0] = p0; ps[1] = p1;
    T &hx = a.Hx.at(c.i, c.j), &hy = a.Hy.at(c.i, c.j);
    hx = hx - a.chx * (dey + p0);
    hy = hy + a.chy * (dex + p1);
  } else {
    const int k = (b - a.nbS - a.nbC - a.nbP) * blockDim.x + threadIdx.x;
    if (k >= a.L0 * a.L1) return;
    window_h(a, k);
  }
}

// E update: comp 0 = Ex (TETMSolver.hh:165-172), comp 1 = Ey (:241-249).  The
// static mesh carries no current in the reference loop (its J is reset to
// zero every step, main.cpp:388, :494), so it enters as 0.0.  The window
// current comes from the fixed-point accumulator of the last push, which is
// converted, stored for diagnostics and cleared for the next deposit.
template <class T, int COMP>
__device__ __forceinline__ void update_e_static(const FieldArgsT<T> &a, int b, T zeroJ) {
  constexpr int V = Vec16<T>::N;
  int c, j;
  if (!static_vec(a, b, c, j)) return;
  const bool live = c <= a.Nx + 1;
  const unsigned m = live ? static_mask(a, c, j) : 0u;  // in flight with the plane loads
  T *ep = COMP == 0 ? &a.Ex.at(c - 1, j) : &a.Ey.at(c - 1, j);
  Vec16<T> e{}, hx{}, hy{}, hxm{}, hym{};
  if (live) {
    e = ld16(ep);
    hx = ld16(&a.Hx.at(c - 1, j));
    hy = ld16(&a.Hy.at(c - 1, j));
    if (COMP == 0) {
      hxm = ld16(&a.Hx.at(c - 1, j - 1));
      hym = ld16(&a.Hy.at(c - 1, j - 1));
    }
  }
  T hxp = T(0), hyp = T(0);  // Ey: H of the cell left of the vector
  if (COMP == 1) {
    hxp = __shfl_up_sync(0xffffffffu, hx.v[V - 1], 1);
    hyp = __shfl_up_sync(0xffffffffu, hy.v[V - 1], 1);
  }
  if (!m) return;
  if (COMP == 1 && (threadIdx.x & 31) == 0 && c >= 1) {
    hxp = a.Hx.at(c - 2, j);
    hyp = a.Hy.at(c - 2, j);
  }
#pragma unroll
  for (int k = 0; k < V; ++k) {
    if (COMP == 0) {
      e.v[k] = e.v[k] + (a.kex * (hx.v[k] - hxm.v[k] + hy.v[k] - hym.v[k]) - a.dteps * zeroJ);
    } else {
      const T hxl = k > 0 ? hx.v[k > 0 ? k - 1 : 0] : hxp, hyl = k > 0 ? hy.v[k > 0 ? k - 1 : 0] : hyp;
      e.v[k] = e.v[k] - (a.key * (hx.v[k] - hxl + hy.v[k] - hyl) + a.dteps * zeroJ);
    }
  }
  store_masked(ep, e, m);
}

// E update: comp 0 = Ex (TETMSolver.hh:165-172), comp 1 = Ey (:241-249).  The
// static mesh carries no current in the reference loop (its J is reset to
// zero every step, main.cpp:388, :494), so it enters as 0.0.  The window
// current comes from the fixed-point accumulator of the last push, which is
// converted, stored for diagnostics and cleared for the next deposit.
template <class T, int COMP>
__device__ __forceinline__ void update_e_body(const FieldArgsT<T> &a, int b, T zeroJ) {
  if (b < a.nbS) {
    update_e_static<T, COMP>(a, b, zeroJ);
  } else if (b < a.nbS + a.nbC) {
    const int k = (b - a.nbS) * blockDim.x + threadIdx.x;
    if (k >= a.ncells) return;
    const CutCellDev c = a.cells[k];
    if (c.area < kMinArea) return;
    if (COMP == 0) {
      if (!(c.l0 > kSpaceEps)) return;
      const T u0 = (a.Hx.at(c.i, c.j) - a.Hx.at(c.i, c.j - 1)) / a.h1;
      const T u1 = (a.Hy.at(c.i, c.j) - a.Hy.at(c.i, c.j - 1)) / a.h1;
      a.Ex.at(c.i, c.j) += a.de * (u0 + u1 - zeroJ);
    } else {
      if (!(c.l1 > kSpaceEps)) return;
      const T u0 = -(a.Hx.at(c.i, c.j) - a.Hx.at(c.i - 1, c.j)) / a.h0;
      const T u1 = -(a.Hy.at(c.i, c.j) - a.Hy.at(c.i - 1, c.j)) / a.h0;
      a.Ey.at(c.i, c.j) += a.de * (u0 + u1 - zeroJ);
    }
  } else if (b < a.nbS + a.nbC + a.nbP) {
    const int k = (b - a.nbS - a.nbC) * blockDim.x + threadIdx.x;
    if (k >= a.npml) return;
    const PmlCellT<T> c = a.pml[k];
    T &ps = a.psi[4 * (size_t)k + 2 + COMP];
    if (COMP == 0) {
      const T dh = a.Hx.at(c.i, c.j) - a.Hx.at(c.i, c.j - 1) + a.Hy.at(c.i, c.j) - a.Hy.at(c.i, c.j - 1);
      const T p = c.bex * ps + c.aex * dh;
      ps = p;
      T &e = a.Ex.at(c.i, c.j);
      e = e + (a.kex * (dh + p) - a.dteps * zeroJ);
    } else {
      const T dh = a.Hx.at(c.i, c.j) - a.Hx.at(c.i - 1, c.j) + a.Hy.at(c.i, c.j) - a.Hy.at(c.i - 1, c.j);
      const T p = c.bey * ps + c.aey * dh;
      ps = p;
      T &e = a.Ey.at(c.i, c.j);
      e = e - (a.key * (dh + p) + a.dteps * zeroJ);
    }
  } else {
    const int k = (b - a.nbS - a.nbC - a.nbP) * blockDim.x + threadIdx.x;
    if (k >= a.L0 * a.L1) return;
    window_e<T, COMP>(a, k);
  }
}

// Strip exchange between the window and the static mesh for one field
// (which: 0 = H as the sum Hzx + Hzy split 1/2 1/2, 1 = Ex, 2 = Ey).
// Strips (Communicator.cpp:640-642):
//   H : window last column and last row -> static; static column left of and
//       row below the window (corners included) -> window guard ring.
//   Ex: window first row -> static; static row above the window -> window guard.
//   Ey: window first column -> static; static column right of the window -> window guard.
// No element is both read and written, so every thread copies one element.
template <class T>
__device__ __forceinline__ void exchange_body(const FieldArgsT<T> &a, int which, int k) {
  const WinState *ws = a.ws;
  const int P0 = ws->P0, P1 = ws->P1, L0 = a.L0, L1 = a.L1;
  // segment table: (to_window, count)
  int si, sj, wi, wj;  // static and window coordinates of the element
  bool to_window;
  if (which == 0) {
    if (k < L1) { wi = L0 - 1; wj = k; to_window = false; }
    else if ((k -= L1) < L0) { wi = k; wj = L1 - 1; to_window = false; }
    else if ((k -= L0) < L1 + 2) { wi = -1; wj = k - 1; to_window = true; }
    else if ((k -= L1 + 2) < L0 + 2) { wi = k - 1; wj = -1; to_window = true; }
    else return;
  } else if (which == 1) {
    if (k < L0) { wi = k; wj = 0; to_window = false; }
    else if ((k -= L0) < L0 + 2) { wi = k - 1; wj = L1; to_window = true; }
    else return;
  } else {
    if (k < L1) { wi = 0; wj = k; to_window = false; }
    else if ((k -= L1) < L1 + 2) { wi = L0; wj = k - 1; to_window = true; }
    else return;
  }
  si = wi + P0; sj = wj + P1;
  if (to_window) {
    if (si < 0 || si >= a.Nx || sj < 0 || sj >= a.Ny) return;
    if (which == 0) {
      const T v = a.Hx.at(si, sj) + a.Hy.at(si, sj);
      a.mHx.at(wi, wj) = T(0.5) * v; a.mHy.at(wi, wj) = T(0.5) * v;
    } else if (which == 1) {
      a.mEx.at(wi, wj) = a.Ex.at(si, sj);
    } else {
      a.mEy.at(wi, wj) = a.Ey.at(si, sj);
    }
  } else {
    if (si < -1 || si > a.Nx || sj < -1 || sj > a.Ny) return;
    if (which == 0) {
      const T v = a.mHx.at(wi, wj) + a.mHy.at(wi, wj);
      a.Hx.at(si, sj) = T(0.5) * v; a.Hy.at(si, sj) = T(0.5) * v;
    } else if (which == 1) {
      a.Ex.at(si, sj) = a.mEx.at(wi, wj);
    } else {
      a.Ey.at(si, sj) = a.mEy.at(wi, wj);
    }
  }
}

// Copy the static fields into the window interior (Communicator::copy via
// copyFields, main.cpp:335-337).
template <class T>
__global__ void k_copy_to_window(FieldArgsT<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.L0 * a.L1) return;
  const int i = k % a.L0, j = k / a.L0;
  const int si = i + a.ws->P0, sj = j + a.ws->P1;
  if (si < 0 || sj < 0 || si >= a.Nx || sj >= a.Ny) return;
  a.mEx.at(i, j) = a.Ex.at(si, sj); a.mEy.at(i, j) = a.Ey.at(si, sj);
  a.mHx.at(i, j) = a.Hx.at(si, sj); a.mHy.at(i, j) = a.Hy.at(si, sj);
}

// Set err if the window or its one-cell ring touches a cell that is not a
// regular inside cell: the fused sub-step launches assume the strip exchange
// and the cut-cell (or absorbing-layer) updates never meet.
template <class T>
__device__ void check_window_clear(const FieldArgsT<T> &a, WinState *ws) {
  const int P0 = ws->P0, P1 = ws->P1;
  const int per = 2 * (a.L0 + 2) + 2 * a.L1;
  for (int k = threadIdx.x; k < per; k += blockDim.x) {
    int i, j;
    if (k < a.L0 + 2) { i = k - 1; j = -1; }
    else if (k < 2 * (a.L0 + 2)) { i = k - (a.L0 + 2) - 1; j = a.L1; }
    else if (k < 2 * (a.L0 + 2) + a.L1) { i = -1; j = k - 2 * (a.L0 + 2); }
    else { i = a.L0; j = k - 2 * (a.L0 + 2) - a.L1; }
    const int si = i + P0, sj = j + P1;
    if (si < 0 || sj < 0 || si >= a.Nx || sj >= a.Ny || !a.mask[(size_t)sj * a.Nx + si] ||
        (a.pml_rows && (si < a.pml_rows[sj].x || si >= a.pml_rows[sj].y)))  // or an absorbing-layer cell
      set_err(ws, kErrWindowWall);
  }
}

template <class T>
__global__ void k_check_window(FieldArgsT<T> a) { check_window_clear(a, a.ws); }

// Window move (moveMesh, main.cpp:562-652, and exchangeBoundariesMovingMesh,
// Communicator.cpp:123-642): from the last deposit's particle bounds the
// window shifts by whole cells through a scratch copy, its position and
// origin are updated and the strips refreshed.

// The move of the window (main.cpp:567-600): ok, whole-cell shift (moveI in
// x, dj in y) and the error code when the bunch no longer fits or would move
// too far.  Reads only the bounds, so every CTA of a launch can take it.
struct MoveDecision {
  int ok, moveI, dj, err;
};
__device__ __forceinline__ MoveDecision move_decision(const WinState *ws, int L0, int L1) {
  MoveDecision r{1, 0, 0, kOk};
  const int L[2] = {L0, L1};
  int ideal1[2] = {0, 0};
  for (int d = 0; d < 2; ++d) {
    const int len = ws->gb[2 * d + 1] - ws->gb[2 * d] + 1;
    if (len >= L[d]) { r.ok = 0; r.err = kErrWindowFit; return r; }
    const unsigned diff = (unsigned)(L[d] - len);
    const unsigned up = (unsigned)floor(diff / 2.0);
    ideal1[d] = L[d] - (int)up - 2;
  }
  r.moveI = ws->gb[1] - ideal1[0] - 1;
  r.dj = ws->gb[3] - ideal1[1] - 1;
  if (r.moveI < 0 || r.moveI > 1 || r.dj < -1 || r.dj > 1) { r.ok = 0; r.err = kErrWindowMove; }
  return r;
}

// Window plane f (0 Ex, 1 Ey, 2 Hzx, 3 Hzy, 4 Jx, 5 Jy).
template <class T>
__device__ __forceinline__ const PlaneT<T> &wplane_of(const FieldArgsT<T> &a, int f) {
  return f == 0 ? a.mEx : f == 1 ? a.mEy : f == 2 ? a.mHx : f == 3 ? a.mHy : f == 4 ? a.mJx : a.mJy;
}

// Phase A (stage 0: the window planes into scratch) or phase B (stage 1: the
// shifted copy back, over the reference's loop ranges) of a move, items
// [tid, ...) in steps of nth.
template <class T>
__device__ __forceinline__ void move_copy(const MoveArgs<T> &m, int moveI, int m1, int stage, int tid, int nth) {
  const FieldArgsT<T> &a = m.f;
  const int W0 = a.L0 + 2, W1 = a.L1 + 2, np = W0 * W1;
  if (stage == 0) {
    for (int k = tid; k < 6 * np; k += nth) {
      const int f = k / np, r = k % np;
      m.scratch[k] = wplane_of(a, f).p[r];
    }
    return;
  }
  const int i0 = -moveI, i1 = a.L0 - 1;
  int j0 = -(m1 > 0 ? m1 : 0), j1 = a.L1 - 1 - (m1 < 0 ? m1 : 0);
  if (m1 == 0) { j0 -= 1; j1 += 1; }
  const int ni = i1 - i0 + 1, cnt = ni * (j1 - j0 + 1);
  for (int k = tid; k < 6 * cnt; k += nth) {
    const int f = k / cnt, r = k % cnt;
    const int i = i0 + r % ni, j = j0 + r / ni;
    wplane_of(a, f).at(i, j) = m.scratch[(size_t)f * np + (size_t)(j + m1 + 1) * W0 + (i + moveI + 1)];
  }
}

template <class T>
__device__ __forceinline__ void move_finish(const MoveArgs<T> &m, int moveI, int m1);

// The whole move in one CTA (batched ensembles: one CTA per member).
template <class T>
__device__ __forceinline__ void move_body(const MoveArgs<T> &m) {
  const FieldArgsT<T> &a = m.f;
  WinState *ws = a.ws;
  if (ws->err) return;
  __shared__ int s_move[3];
  if (threadIdx.x == 0) {
    const MoveDecision d = move_decision(ws, a.L0, a.L1);
    if (!d.ok) set_err(ws, d.err);
    s_move[0] = d.ok; s_move[1] = d.moveI; s_move[2] = d.dj;
    if (d.ok) { ws->moves[0] = d.moveI; ws->moves[1] = d.dj; }
  }
  __syncthreads();
  if (!s_move[0]) return;
  const int moveI = s_move[1], m1 = s_move[2];
  if (moveI == 0 && m1 == 0) return;
  move_copy(m, moveI, m1, 0, threadIdx.x, blockDim.x);
  __syncthreads();
  move_copy(m, moveI, m1, 1, threadIdx.x, blockDim.x);
  __syncthreads();
  move_finish(m, moveI, m1);
}

// Position, origin and strips after the shifted copy (one CTA).
template <class T>
__device__ __forceinline__ void move_finish(const MoveArgs<T> &m, int moveI, int m1) {
  const FieldArgsT<T> &a = m.f;
  WinState *ws = a.ws;
  if (threadIdx.x == 0) {
    ws->P0 += moveI; ws->P1 += m1;
    ws->mo0 += moveI * m.h0;
    ws->mo1 += m1 * m.h1;
  }
  __syncthreads();
  // phase C: strip layers; type 0..2 window -> static (Hz, Ex, Ey), 3..5 static -> window.
  const int P0 = ws->P0, P1 = ws->P1, Ld0 = a.L0 - 1, Ld1 = a.L1 - 1;
  int lay[12][5], nl = 0;
  auto add = [&](int t, int b0, int e0, int b1, int e1) {
    lay[nl][0] = t; lay[nl][1] = b0; lay[nl][2] = e0; lay[nl][3] = b1; lay[nl][4] = e1; ++nl;
  };
  // layers grouped by type, in the reference's list order
  for (int t = 0; t < 6; ++t) {
    if (moveI == 1) {
      switch (t) {
        case 0: add(0, -1, -1, -m1, Ld1 - m1 - 1); break;
        case 1: add(1, -1, -1, 1 - m1, Ld1 - m1); break;
        case 2: add(2, 0, 0, -m1, Ld1 - m1); break;
        case 3: add(3, Ld0 + P0, Ld0 + P0, P1, Ld1 + P1); break;
        case 4: add(4, Ld0 + P0, Ld0 + P0, P1, Ld1 + P1 + 1); break;
        case 5: add(5, Ld0 + P0 + 1, Ld0 + P0 + 1, P1, Ld1 + P1); break;
      }
    }
    if (m1 == 1) {
      switch (t) {
        case 0: add(0, -moveI, Ld0 - 1 - moveI, -1, -1); break;
        case 1: add(1, -moveI, Ld0 - moveI, 0, 0); break;
        case 2: add(2, 1 - moveI, Ld0 - moveI, -1, -1); break;
        case 3: add(3, P0, Ld0 + P0, Ld1 + P1, Ld1 + P1); break;
        case 4: add(4, P0, Ld0 + P0, Ld1 + 1 + P1, Ld1 + 1 + P1); break;
        case 5: add(5, P0, Ld0 + P0 + 1, Ld1 + P1, Ld1 + P1); break;
      }
    } else if (m1 == -1) {
      switch (t) {
        case 0: add(0, -moveI, Ld0 - moveI - 1, Ld1, Ld1); break;
        case 1: add(1, -moveI, Ld0 - moveI, Ld1 + 1, Ld1 + 1); break;
        case 2: add(2, 1 - moveI, Ld0 - moveI, Ld1 + 1, Ld1 + 1); break;
        case 3: add(3, P0, Ld0 + P0, P1 - 1, P1 - 1); break;
        case 4: add(4, P0, Ld0 + P0, P1, P1); break;
        case 5: add(5, P0, Ld0 + P0 + 1, P1, P1); break;
      }
    }
  }
  // clip each layer (window layers to [-1, L] and the static domain; static
  // layers to the static domain and the window incl. guards)
  int beg[13];
  beg[0] = 0;
  for (int l = 0; l < nl; ++l) {
    int *y = lay[l];
    if (y[0] < 3) {
      y[1] = max(max(y[1], -1), -P0); y[2] = min(min(y[2], a.L0), a.Nx - 1 - P0);
      y[3] = max(max(y[3], -1), -P1); y[4] = min(min(y[4], a.L1), a.Ny - 1 - P1);
    } else {
      y[1] = max(max(y[1], 0), P0 - 1); y[2] = min(min(y[2], a.Nx - 1), P0 + a.L0);
      y[3] = max(max(y[3], 0), P1 - 1); y[4] = min(min(y[4], a.Ny - 1), P1 + a.L1);
    }
    const int c = (y[2] >= y[1] && y[4] >= y[3]) ? (y[2] - y[1] + 1) * (y[4] - y[3] + 1) : 0;
    beg[l + 1] = beg[l] + c;
  }
  const int total = beg[nl];
  T *vals = m.scratch;  // the snapshot is no longer needed
  for (int k = threadIdx.x; k < total; k += blockDim.x) {
    int l = 0;
    while (k >= beg[l + 1]) ++l;
    const int *y = lay[l];
    const int w = y[2] - y[1] + 1, r = k - beg[l];
    const int i = y[1] + r % w, j = y[3] + r / w;
    T v;
    switch (y[0]) {
      case 0: v = a.mHx.at(i, j) + a.mHy.at(i, j); break;
      case 1: v = a.mEx.at(i, j); break;
      case 2: v = a.mEy.at(i, j); break;
      case 3: v = a.Hx.at(i, j) + a.Hy.at(i, j); break;
      case 4: v = a.Ex.at(i, j); break;
      default: v = a.Ey.at(i, j); break;
    }
    vals[k] = v;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < total; k += blockDim.x) {
    int l = 0;
    while (k >= beg[l + 1]) ++l;
    const int *y = lay[l];
    const int w = y[2] - y[1] + 1, r = k - beg[l];
    const int i = y[1] + r % w, j = y[3] + r / w;
    const T v = vals[k];
    switch (y[0]) {
      case 0: a.Hx.at(i + P0, j + P1) = T(0.5) * v; a.Hy.at(i + P0, j + P1) = T(0.5) * v; break;
      case 1: a.Ex.at(i + P0, j + P1) = v; break;
      case 2: a.Ey.at(i + P0, j + P1) = v; break;
      case 3: a.mHx.at(i - P0, j - P1) = T(0.5) * v; a.mHy.at(i - P0, j - P1) = T(0.5) * v; break;
      case 4: a.mEx.at(i - P0, j - P1) = v; break;
      default: a.mEy.at(i - P0, j - P1) = v; break;
    }
  }
  __syncthreads();
  check_window_clear(a, ws);
}

// Member of global block b: bpre holds the first block of every member (m + 1
// entries).
__device__ __forceinline__ int batch_member(const int *bpre, int m, int b) {
  int lo = 0, hi = m - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(bpre + mid) <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// --- fused static sweep: the four sub-steps of one time step in one pass ----
//
// The static mesh carries no current, and between the first and the last of
// its four sub-steps (half H, Ex, half H, Ey) it meets the rest of the step
// only through the window's strips.  So one launch (k_yee_tiles) takes every
// static cell through all four sub-steps: a CTA stages a tile of Ex, Ey, Hx,
// Hy and the cell-kind map into shared memory with TMA (a one-cell halo on
// each side and two rows above: the cells the later sub-steps of its own
// cells read), runs the sub-steps there, regular and cut cells alike, with
// the arithmetic of the sub-step kernels, and writes its cells into the
// OTHER plane set.  Reading one set and writing the other is what lets
// neighbouring tiles run in any order.  Cells within two of the window's
// footprint are left to k_yee_fixup (one cluster, beside the tiles on a
// second stream), which redoes them from the source set with the window's
// own sub-steps and the strip exchanges in between, in the reference's
// order; the window's Ey sub-step, which needs the second push's
// current, follows that push (k_window_ey) with its Ey exchange.  The static
// Ey the exchange overwrites (the window's first column) is the only static
// value the push-dependent part changes.
//
// The absorbing layers are not part of this path (their cells keep the
// sub-step kernels).

// Cell kinds of the kind map (static storage layout with guards, one byte).
enum : uint8_t { kKindNone = 0, kKindRegular = 1, kKindCut = 2 };

// Updates of one static cell, shared by the tile and the fix-up kernels: the
// same expressions as the sub-step kernels' regular-cell and cut-cell
// branches (TETMSolver.hh:142-206, :241-261; SCBoundaryCondition.hh:391-431).
template <class T, class A>
__device__ __forceinline__ void h_cell(const A &a, uint8_t kind, const CutCellDev *cc, T &hx, T &hy,
                                       T ey0, T ey1, T ex0, T ex1) {
  if (kind == kKindRegular) {
    hx = hx - a.chx * (ey1 - ey0);
    hy = hy + a.chy * (ex1 - ex0);
  } else {
    const T n0 = (T)cc->n0, n1 = (T)cc->n1, l0 = (T)cc->l0, l1 = (T)cc->l1, area = (T)cc->area;
    const T u0 = a.mhx * (n1 * ey1 - l1 * ey0) / area;
    const T u1 = a.mhy * (n0 * ex1 - l0 * ex0) / area;
    hx += u0;
    hy += u1;
  }
}

// Ex of one static cell; hxm, hym: H of the cell below.
template <class T, class A>
__device__ __forceinline__ void ex_cell(const A &a, uint8_t kind, const CutCellDev *cc, T &e, T hx, T hxm,
                                        T hy, T hym, T zeroJ) {
  if (kind == kKindRegular) {
    e = e + (a.kex * (hx - hxm + hy - hym) - a.dteps * zeroJ);
  } else {
    if (cc->area < kMinArea || !(cc->l0 > kSpaceEps)) return;
    const T u0 = (hx - hxm) / a.h1;
    const T u1 = (hy - hym) / a.h1;
    e += a.de * (u0 + u1 - zeroJ);
  }
}

// Ey of one static cell; hxl, hyl: H of the cell to the left.
template <class T, class A>
__device__ __forceinline__ void ey_cell(const A &a, uint8_t kind, const CutCellDev *cc, T &e, T hx, T hxl,
                                        T hy, T hyl, T zeroJ) {
  if (kind == kKindRegular) {
    e = e - (a.key * (hx - hxl + hy - hyl) + a.dteps * zeroJ);
  } else {
    if (cc->area < kMinArea || !(cc->l1 > kSpaceEps)) return;
    const T u0 = -(hx - hxl) / a.h0;
    const T u1 = -(hy - hyl) / a.h0;
    e += a.de * (u0 + u1 - zeroJ);
  }
}

// Tile geometry.  A tile is TX storage columns [s0, s0 + TX) (s0 a multiple
// of TX; storage column s holds cell s - 1) by TY cell rows [y0, y0 + TY).
// The plane boxes cover storage columns [s0 - V, s0 + TX + V) (V elements =
// 16 bytes, so that the box starts on a 16-byte boundary and its rows are a
// whole number of 16-byte pieces) and cell rows y0 - 1 .. y0 + TY + 1; the
// kind box covers storage columns [s0 - 16, s0 + TX + 16) of the same rows.
template <class T>
struct YeeTile {
  static constexpr int V = 16 / (int)sizeof(T);
  static constexpr int TX = sizeof(T) == 4 ? 64 : 32;
  static constexpr int TY = 32;
  static constexpr int W = TX + 2 * V;
  static constexpr int H = TY + 3;
  static constexpr int KW = TX + 32;
  static constexpr int KO = 16 - V;  // kind-box column of plane-box column c: c + KO
  static constexpr int PLANE_BYTES = (W * H * (int)sizeof(T) + 127) / 128 * 128;
  static constexpr int KIND_BYTES = (KW * H + 127) / 128 * 128;
  static constexpr uint32_t TX_BYTES = 4u * W * H * sizeof(T) + (uint32_t)KW * H;
  static constexpr int CUTS = 256;  // cut cells the tile's list holds (more: the phases scan the kinds)
  // planes, kinds, barrier (16 bytes), cut list, base alignment; 5 CTAs per SM
  static constexpr int SMEM = 4 * PLANE_BYTES + KIND_BYTES + 16 + 2 * CUTS + 128;
  static constexpr int THREADS = 256;
  static constexpr int E = V;           // cells per lane in a row: 16 bytes
  static constexpr int LPR = TX / E;    // lanes per row (16): a warp takes two rows at a time
};

template <class T>
struct alignas(64) YeeTileArgs {
  CUtensorMap map[5];   // Ex, Ey, Hx, Hy of the source set, then the kind map
  FieldArgsT<T> f;      // coefficients, cut cells, mesh size (static planes: the source set)
  PlaneT<T> out[4];     // Ex, Ey, Hx, Hy of the destination set
  const int *cutidx;    // cell -> cut-cell entry
  int tilesX;
  T zeroJ;
  long long spin;       // polls of the staging wait before it gives up (kErrStaging)
};

// The region the fix-up rewrites: the window's footprint widened by two
// cells, clipped to the mesh, cells [c0, c1) x [r0, r1).
struct FixRegion {
  int c0, c1, r0, r1;
};
__device__ __forceinline__ FixRegion fix_region(int P0, int P1, int L0, int L1, int Nx, int Ny) {
  return FixRegion{max(P0 - 2, 0), min(P0 + L0 + 2, Nx), max(P1 - 2, 0), min(P1 + L1 + 2, Ny)};
}

// E consecutive elements of a shared-memory row (E = 2 floats or 1 double:
// one 8-byte access per lane).
template <class T, int E>
struct alignas(E * sizeof(T)) Pack {
  T v[E];
};
template <class T, int E>
__device__ __forceinline__ Pack<T, E> ldp(const T *p) { return *reinterpret_cast<const Pack<T, E> *>(p); }
template <class T, int E>
__device__ __forceinline__ void stp(T *p, const Pack<T, E> &x) { *reinterpret_cast<Pack<T, E> *>(p) = x; }

// The E kinds of the cells at kind-box offset q (q a multiple of E).
template <int E>
__device__ __forceinline__ void kinds(const uint8_t *sK, int q, uint8_t *kd) {
  if (E == 4) {
    const uint32_t w = *reinterpret_cast<const uint32_t *>(sK + q);
#pragma unroll
    for (int e = 0; e < E; ++e) kd[e] = (uint8_t)(w >> (8 * e));
  } else if (E == 2) {
    const uint16_t w = *reinterpret_cast<const uint16_t *>(sK + q);
    kd[0] = (uint8_t)(w & 0xff);
    kd[E - 1] = (uint8_t)(w >> 8);
  } else {
    kd[0] = sK[q];
  }
}

// Shared-memory tile of the sweep: the four planes and the kinds, box
// column c / row r = cell (i0 + c, j0 + r).
template <class T>
struct TileSm {
  T *ex, *ey, *hx, *hy;
  const uint8_t *k;
  int i0, j0;
};

// The coefficients in registers (h_cell / ex_cell / ey_cell read them by
// name, as from FieldArgsT; the row passes use only the regular ones).
template <class T>
struct Coef {
  T chx, chy, kex, key, dteps, mhx, mhy, de, h0, h1;
};

template <class T, class G>
__device__ __forceinline__ const CutCellDev *tile_cut(const YeeTileArgs<T> &a, const TileSm<T> &t, int c, int r) {
  return a.f.cells + a.cutidx[(size_t)(t.j0 + r) * a.f.Nx + (t.i0 + c)];
}

// Regular cells of a piece: the row passes handle only kind-regular cells
// (with the regular branch of h_cell / ex_cell / ey_cell) and store only
// those elements back; cut cells have their own pass over the tile's list,
// halo-column cells their own pass, so that no store of one pass covers a
// cell another pass of the same phase writes.

// Stores a piece back: whole when every cell is regular, else the regular
// cells one by one.
template <class T, int E>
__device__ __forceinline__ void store_regular(T *p, const Pack<T, E> &x, const uint8_t *kd) {
  bool all = true;
#pragma unroll
  for (int e = 0; e < E; ++e) all &= kd[e] == kKindRegular;
  if (all) {
    stp<T, E>(p, x);
    return;
  }
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (kd[e] == kKindRegular) p[e] = x.v[e];
}

// The row passes: half-warp h of a warp takes row r = rp + h, lane l of it
// the cells [c, c + E) with c = V + l E; `valid` is false for the second
// row past the phase's last, whose lanes only take part in the shuffles
// (reading the last row).  A warp leaves a pass when none of its cells is
// regular; the cell right (left) of a lane's piece comes from the next
// (previous) lane of its half, the half's end lanes read it.

// Half H, regular cells [c, c + E) of row r.
template <class T, class G>
__device__ __forceinline__ void tile_h(const Coef<T> &k, const TileSm<T> &t, int c, int r, bool valid) {
  constexpr int E = G::E, W = G::W;
  const int o = r * W + c, l = threadIdx.x & (G::LPR - 1);
  uint8_t kd[E];
  kinds<E>(t.k, r * G::KW + c + G::KO, kd);
  bool any = false;
#pragma unroll
  for (int e = 0; e < E; ++e) any |= kd[e] == kKindRegular;
  if (!__any_sync(0xffffffffu, any && valid)) return;
  Pack<T, E> hx = ldp<T, E>(t.hx + o), hy = ldp<T, E>(t.hy + o);
  const Pack<T, E> ey = ldp<T, E>(t.ey + o), ex0 = ldp<T, E>(t.ex + o), ex1 = ldp<T, E>(t.ex + o + W);
  T eyn = __shfl_down_sync(0xffffffffu, ey.v[0], 1);
  if (l == G::LPR - 1) eyn = t.ey[o + E];
  if (!valid) return;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const T ey1 = e + 1 < E ? ey.v[e + 1 < E ? e + 1 : 0] : eyn;
    h_cell(k, kKindRegular, nullptr, hx.v[e], hy.v[e], ey.v[e], ey1, ex0.v[e], ex1.v[e]);
  }
  store_regular<T, E>(t.hx + o, hx, kd);
  store_regular<T, E>(t.hy + o, hy, kd);
}

// Ex, regular cells [c, c + E) of row r.
template <class T, class G>
__device__ __forceinline__ void tile_ex(const Coef<T> &k, T zeroJ, const TileSm<T> &t, int c, int r, bool valid) {
  constexpr int E = G::E, W = G::W;
  if (!valid) return;
  const int o = r * W + c;
  uint8_t kd[E];
  kinds<E>(t.k, r * G::KW + c + G::KO, kd);
  bool any = false;
#pragma unroll
  for (int e = 0; e < E; ++e) any |= kd[e] == kKindRegular;
  if (!any) return;
  Pack<T, E> ex = ldp<T, E>(t.ex + o);
  const Pack<T, E> hx = ldp<T, E>(t.hx + o), hxm = ldp<T, E>(t.hx + o - W);
  const Pack<T, E> hy = ldp<T, E>(t.hy + o), hym = ldp<T, E>(t.hy + o - W);
#pragma unroll
  for (int e = 0; e < E; ++e) ex_cell(k, kKindRegular, nullptr, ex.v[e], hx.v[e], hxm.v[e], hy.v[e], hym.v[e], zeroJ);
  store_regular<T, E>(t.ex + o, ex, kd);
}

// Ey, regular cells [c, c + E) of row r.
template <class T, class G>
__device__ __forceinline__ void tile_ey(const Coef<T> &k, T zeroJ, const TileSm<T> &t, int c, int r, bool valid) {
  constexpr int E = G::E, W = G::W;
  const int o = r * W + c, l = threadIdx.x & (G::LPR - 1);
  uint8_t kd[E];
  kinds<E>(t.k, r * G::KW + c + G::KO, kd);
  bool any = false;
#pragma unroll
  for (int e = 0; e < E; ++e) any |= kd[e] == kKindRegular;
  if (!__any_sync(0xffffffffu, any && valid)) return;
  Pack<T, E> ey = ldp<T, E>(t.ey + o);
  const Pack<T, E> hx = ldp<T, E>(t.hx + o), hy = ldp<T, E>(t.hy + o);
  T hxl0 = __shfl_up_sync(0xffffffffu, hx.v[E - 1], 1), hyl0 = __shfl_up_sync(0xffffffffu, hy.v[E - 1], 1);
  if (l == 0) {
    hxl0 = t.hx[o - 1];
    hyl0 = t.hy[o - 1];
  }
  if (!valid) return;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const T hxl = e > 0 ? hx.v[e > 0 ? e - 1 : 0] : hxl0, hyl = e > 0 ? hy.v[e > 0 ? e - 1 : 0] : hyl0;
    ey_cell(k, kKindRegular, nullptr, ey.v[e], hx.v[e], hxl, hy.v[e], hyl, zeroJ);
  }
  store_regular<T, E>(t.ey + o, ey, kd);
}

// One cell (box column c, row r) of a phase, of either kind; none is left alone.
template <class T, class G, int PHASE>
__device__ __forceinline__ void tile_cell(const YeeTileArgs<T> &a, const TileSm<T> &t, uint8_t kd, int c, int r) {
  constexpr int W = G::W;
  if (kd == kKindNone) return;
  const int o = r * W + c;
  const CutCellDev *cc = kd == kKindCut ? tile_cut<T, G>(a, t, c, r) : nullptr;
  if (PHASE == 2) ex_cell(a.f, kd, cc, t.ex[o], t.hx[o], t.hx[o - W], t.hy[o], t.hy[o - W], a.zeroJ);
  else if (PHASE == 4) ey_cell(a.f, kd, cc, t.ey[o], t.hx[o], t.hx[o - 1], t.hy[o], t.hy[o - 1], a.zeroJ);
  else h_cell(a.f, kd, cc, t.hx[o], t.hy[o], t.ey[o], t.ey[o + 1], t.ex[o], t.ex[o + W]);
}

// The cut cells and the halo column of a phase over rows [rlo, rhi): the
// cut cells from the tile's list (or, when the list overflowed, by a scan of
// the kinds), the halo column's regular cells; run by the threads from
// `first` on, which have the fewest rows in the row pass.
template <class T, class G, int PHASE>
__device__ __forceinline__ void tile_rest(const YeeTileArgs<T> &a, const TileSm<T> &t, const uint16_t *cuts, int ncut,
                                          int rlo, int rhi, int first) {
  const int tid = (int)threadIdx.x - first, nt = G::THREADS - first;
  if (tid < 0) return;
  constexpr int clo = PHASE == 4 ? G::V : G::V - 1;
  if (ncut <= G::CUTS) {
    for (int n = tid; n < ncut; n += nt) {
      const int c = cuts[n] & 0x7f, r = cuts[n] >> 7;
      if (r >= rlo && r < rhi && c >= clo) tile_cell<T, G, PHASE>(a, t, kKindCut, c, r);
    }
  } else {  // more cut cells than the list holds: scan the phase's cells
    constexpr int CW = G::V + G::TX - clo;
    for (int k = tid; k < CW * (rhi - rlo); k += nt) {
      const int c = clo + k % CW, r = rlo + k / CW;
      if (t.k[r * G::KW + c + G::KO] == kKindCut) tile_cell<T, G, PHASE>(a, t, kKindCut, c, r);
    }
  }
  if (PHASE != 4)
    for (int r = rlo + tid; r < rhi; r += nt) {
      constexpr int c = G::V - 1;
      if (t.k[r * G::KW + c + G::KO] == kKindRegular) tile_cell<T, G, PHASE>(a, t, kKindRegular, c, r);
    }
}

// Issues the staging copies of tile `tile` into the buffer at base (one thread).
template <class T>
__device__ __forceinline__ void yee_stage(const YeeTileArgs<T> &a, int tile, uint8_t *base) {
  using G = YeeTile<T>;
  uint8_t *sK = base + 4 * G::PLANE_BYTES;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sK + G::KIND_BYTES);
  const int s0 = (tile % a.tilesX) * G::TX, y0 = (tile / a.tilesX) * G::TY;
  mbar_expect_tx(bar, G::TX_BYTES);
  // storage row of cell row y0 - 1 is y0
  for (int p = 0; p < 4; ++p) tma_load_2d(base + p * G::PLANE_BYTES, &a.map[p], s0 - G::V, y0, bar);
  tma_load_2d(sK, &a.map[4], s0 - 16, y0, bar);
}

// One tile of the sweep (tile: its index in row-major tile order) in the
// CTA's shared memory from base (128-byte aligned; planes, kinds, barrier,
// cut list), the barrier initialised by the caller and at phase `parity`;
// staged: its copies were issued already (yee_stage), else this issues them.
// Returns 0; when the staging wait gives up, 1 if the copies arrived at the
// second wait (the barrier's phase is used up as usual), 2 if they did not
// (the barrier must not be used again).
template <class T>
__device__ __forceinline__ int yee_tile(const YeeTileArgs<T> &a, int tile, uint32_t parity, uint8_t *base,
                                        int *s_ncut, bool staged = false) {
  using G = YeeTile<T>;
  T *sEx = reinterpret_cast<T *>(base);
  T *sEy = reinterpret_cast<T *>(base + G::PLANE_BYTES);
  T *sHx = reinterpret_cast<T *>(base + 2 * G::PLANE_BYTES);
  T *sHy = reinterpret_cast<T *>(base + 3 * G::PLANE_BYTES);
  uint8_t *sK = base + 4 * G::PLANE_BYTES;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sK + G::KIND_BYTES);
  uint16_t *cuts = reinterpret_cast<uint16_t *>(sK + G::KIND_BYTES + 16);
  const FieldArgsT<T> &f = a.f;
  const int s0 = (tile % a.tilesX) * G::TX;
  const int y0 = (tile / a.tilesX) * G::TY;
  if (threadIdx.x == 0) {
    *s_ncut = 0;
    if (!staged) yee_stage(a, tile, base);
  }
  // the fix-up's region, whose cells this sweep leaves to it (read while the copies fly)
  const FixRegion R = fix_region(f.ws->P0, f.ws->P1, f.L0, f.L1, f.Nx, f.Ny);
  // a.spin < 0: the staging wait is on a barrier nothing completes (the
  // timeout test), with -a.spin polls
  uint64_t *never = bar + 1;
  const bool ok = a.spin < 0 ? mbar_wait(never, 0, -a.spin) : mbar_wait(bar, parity, a.spin);
  if (__syncthreads_or(!ok)) {  // report, wait once more for the copies, write nothing
    __shared__ int s_late;
    if (threadIdx.x == 0) {
      set_err(f.ws, kErrStaging);
      s_late = mbar_wait(bar, parity, a.spin < 0 ? -a.spin : a.spin) ? 1 : 2;
    }
    __syncthreads();
    return s_late;
  }
  // box column c, row r is cell (s0 - V - 1 + c, y0 - 1 + r)
  const TileSm<T> t{sEx, sEy, sHx, sHy, sK, s0 - G::V - 1, y0 - 1};
  // the tile's cut cells (columns [V - 1, V + TX), rows [0, TY + 2)), as 7-bit
  // column | row << 7: each thread tests 16 kinds at once (a cut kind is the
  // only one with bit 1 set) and looks at single bytes only where one is
  {
    constexpr int CH = G::KW / 16;  // 16-byte pieces of a kind row
    static_assert(CH * (G::TY + 2) <= G::THREADS, "one piece per thread");
    const int k = threadIdx.x;
    if (k < CH * (G::TY + 2)) {
      const int r = k / CH, q0 = (k % CH) * 16;
      const uint4 w = *reinterpret_cast<const uint4 *>(sK + r * G::KW + q0);
      if ((w.x | w.y | w.z | w.w) & 0x02020202u) {
        for (int b = 0; b < 16; ++b) {
          const int c = q0 + b - G::KO;  // box column
          if (c >= G::V - 1 && c < G::V + G::TX && sK[r * G::KW + q0 + b] == kKindCut) {
            const int n = atomicAdd(s_ncut, 1);
            if (n < G::CUTS) cuts[n] = (uint16_t)(c | r << 7);
          }
        }
      }
    }
  }
  __syncthreads();
  const int ncut = *s_ncut;
  // the row passes (tile_h, tile_ex, tile_ey); the halo column V - 1 and the
  // cut cells go to the warps from 2 on in the first two phases (their row
  // pairs leave warps 0 and 1 with one more)
  const int warp = threadIdx.x >> 5, half = (threadIdx.x >> 4) & 1;
  const int c = G::V + (threadIdx.x & (G::LPR - 1)) * G::E;
  const Coef<T> k{f.chx, f.chy, f.kex, f.key, f.dteps, f.mhx, f.mhy, f.de, f.h0, f.h1};
  const T zeroJ = a.zeroJ;
  for (int rp = 2 * warp; rp < G::TY + 2; rp += 16) {
    const int r = rp + half;
    tile_h<T, G>(k, t, c, min(r, G::TY + 1), r < G::TY + 2);
  }
  tile_rest<T, G, 1>(a, t, cuts, ncut, 0, G::TY + 2, 64);
  __syncthreads();
  for (int rp = 1 + 2 * warp; rp < G::TY + 2; rp += 16) {
    const int r = rp + half;
    tile_ex<T, G>(k, zeroJ, t, c, min(r, G::TY + 1), r < G::TY + 2);
  }
  tile_rest<T, G, 2>(a, t, cuts, ncut, 1, G::TY + 2, 64);
  __syncthreads();
  for (int rp = 1 + 2 * warp; rp < G::TY + 1; rp += 16) tile_h<T, G>(k, t, c, rp + half, true);
  tile_rest<T, G, 3>(a, t, cuts, ncut, 1, G::TY + 1, 0);
  __syncthreads();
  for (int rp = 1 + 2 * warp; rp < G::TY + 1; rp += 16) tile_ey<T, G>(k, zeroJ, t, c, rp + half, true);
  tile_rest<T, G, 4>(a, t, cuts, ncut, 1, G::TY + 1, 0);
  __syncthreads();
  // the tile's cells, every one (unchanged ones too) except the fix-up's,
  // into the destination set: 16-byte pieces of storage columns [s0, s0 + TX),
  // the same piece of all four planes per step
  constexpr int NV = G::TX / G::V;
  for (int k = threadIdx.x; k < G::TY * NV; k += G::THREADS) {
    const int r = 1 + k / NV, v = k % NV, j = t.j0 + r;
    if (j >= f.Ny) break;  // rows grow with k
    const int so = r * G::W + G::V + v * G::V;        // shared-memory offset of the piece
    const size_t go = (size_t)(j + 1) * a.out[0].pitch + s0 + v * G::V;  // the planes share one pitch
    const int i = s0 + v * G::V - 1;  // cell of the piece's first element
    const bool whole = j < R.r0 || j >= R.r1 || i + G::V <= R.c0 || i >= R.c1;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const T *src = (p == 0 ? sEx : p == 1 ? sEy : p == 2 ? sHx : sHy) + so;
      T *dst = a.out[p].p + go;
      if (whole) {
        st16(dst, *reinterpret_cast<const Vec16<T> *>(src));
      } else {
#pragma unroll
        for (int e = 0; e < G::V; ++e)
          if (i + e < R.c0 || i + e >= R.c1) dst[e] = src[e];
      }
    }
  }
  return 0;
}

__device__ __forceinline__ uint8_t *align128(uint8_t *p) {
  return reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(p) + 127) & ~(uintptr_t)127);
}

template <class T>
__global__ void __launch_bounds__(256, 5) k_yee_tiles(const __grid_constant__ YeeTileArgs<T> a) {
  using G = YeeTile<T>;
  extern __shared__ uint8_t smem_raw[];
  __shared__ int s_ncut;
  uint8_t *base = align128(smem_raw);
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + 4 * G::PLANE_BYTES + G::KIND_BYTES);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_init_fence();
  }
  __syncthreads();
  yee_tile(a, (int)blockIdx.x, 0u, base, &s_ncut);
}

// The fix-up of the cells around the window (one cluster of kFixCtas CTAs,
// synchronised by cluster barriers between the phases).  Its region is the
// window's footprint widened by two cells, clipped to the mesh: the strip
// exchanges change static cells at most one cell outside the footprint over
// the four sub-steps.  It copies the source set over the region and the
// cells the later sub-steps of the region read into scratch planes, runs the
// static and window sub-steps and exchanges there in the order of the
// sub-step kernels, and writes the region into the destination set.
constexpr int kFixCtas = 8, kFixThreads = 1024;

template <class T>
struct YeeFixArgs {
  PlaneT<T> out[4];   // Ex, Ey, Hx, Hy of the destination set
  T *z;               // 4 scratch planes, zpitch x zrows each
  int zpitch, zrows;
  const uint8_t *kind;
  int kpitch;
  const int *cutidx;
  T zeroJ;
};

// Orders every thread's earlier global and shared writes of the cluster
// before its later reads (release / acquire at cluster scope).
__device__ __forceinline__ void cluster_barrier() {
  __threadfence();
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ int exchange_items(int L0, int L1, int which) {
  return which == 0 ? 2 * (L0 + L1) + 4 : which == 1 ? 2 * L0 + 2 : 2 * L1 + 2;
}

// Half H of static cell (i, j) of the fix-up's scratch planes: every operand
// is loaded before the kind decides (the loads overlap the kind's).
template <class T, class Cut>
__device__ __forceinline__ void fix_h(const FieldArgsT<T> &a, const FieldArgsT<T> &z, uint8_t kd, int i, int j,
                                      const Cut &cut_of) {
  T hx = z.Hx.at(i, j), hy = z.Hy.at(i, j);
  const T ey0 = z.Ey.at(i, j), ey1 = z.Ey.at(i + 1, j), ex0 = z.Ex.at(i, j), ex1 = z.Ex.at(i, j + 1);
  if (kd == kKindNone) return;
  h_cell(a, kd, cut_of(kd, i, j), hx, hy, ey0, ey1, ex0, ex1);
  z.Hx.at(i, j) = hx;
  z.Hy.at(i, j) = hy;
}

// The fix-up's body over threads tid of nth, sync() between its phases (a
// cluster barrier over a cluster, __syncthreads in one CTA).
template <class T, class Sync>
__device__ __forceinline__ void yee_fixup(const FieldArgsT<T> &a, const YeeFixArgs<T> &x, int tid, int nth,
                                          const Sync &sync) {
  const int P0 = a.ws->P0, P1 = a.ws->P1, L0 = a.L0, L1 = a.L1;
  // the window and its ring on the mesh (as the move and the initial
  // placement check, kErrWindowWall), else the scratch box would not hold
  // the strips: nothing is done, uniformly over the cluster
  if (P0 < 1 || P1 < 1 || P0 + L0 >= a.Nx || P1 + L1 >= a.Ny) {
    if (tid == 0) set_err(a.ws, kErrWindowWall);
    return;
  }
  const FixRegion R = fix_region(P0, P1, L0, L1, a.Nx, a.Ny);
  const int c0 = R.c0, c1 = R.c1, r0 = R.r0, r1 = R.r1;
  // scratch box: cells [c0 - 1, c1 + 1) x [r0 - 1, r1 + 2); PlaneT's guard
  // offset puts cell (c0 - 1, r0 - 1) at the start of each scratch plane
  const int zw = c1 - c0 + 2, zh = r1 - r0 + 3;
  const ptrdiff_t zoff = (ptrdiff_t)r0 * x.zpitch + c0;
  const size_t zs = (size_t)x.zpitch * x.zrows;
  FieldArgsT<T> z = a;
  z.Ex = PlaneT<T>{x.z - zoff, x.zpitch};
  z.Ey = PlaneT<T>{x.z + zs - zoff, x.zpitch};
  z.Hx = PlaneT<T>{x.z + 2 * zs - zoff, x.zpitch};
  z.Hy = PlaneT<T>{x.z + 3 * zs - zoff, x.zpitch};
  const int nw = L0 * L1;
  auto kind_of = [&](int i, int j) { return x.kind[(size_t)(j + 1) * x.kpitch + (i + 1)]; };
  auto cut_of = [&](uint8_t kd, int i, int j) -> const CutCellDev * {
    return kd == kKindCut ? a.cells + x.cutidx[(size_t)j * a.Nx + i] : nullptr;
  };
  // the box from the source set (cells off the stored planes read zero, as
  // the tile kernel's staging fills them)
  {
    const int nb = zw * zh;
    for (int k = tid; k < 4 * nb; k += nth) {
      const int p = k / nb, rem = k % nb, i = c0 - 1 + rem % zw, j = r0 - 1 + rem / zw;
      const PlaneT<T> &src = p == 0 ? a.Ex : p == 1 ? a.Ey : p == 2 ? a.Hx : a.Hy;
      const PlaneT<T> &dst = p == 0 ? z.Ex : p == 1 ? z.Ey : p == 2 ? z.Hx : z.Hy;
      const bool stored = i >= -1 && i <= a.Nx && j >= -1 && j <= a.Ny;
      dst.at(i, j) = stored ? src.at(i, j) : T(0);
    }
  }
  sync();
  // 1: half H, static [c0 - 1, c1) x [r0 - 1, r1 + 1), and the window
  {
    const int w = c1 - c0 + 1, ns = w * (r1 - r0 + 2);
    for (int k = tid; k < ns + nw; k += nth) {
      if (k >= ns) { window_h(a, k - ns); continue; }
      const int i = c0 - 1 + k % w, j = r0 - 1 + k / w;
      fix_h(a, z, kind_of(i, j), i, j, cut_of);
    }
  }
  sync();
  for (int k = tid; k < exchange_items(L0, L1, 0); k += nth) exchange_body(z, 0, k);
  sync();
  // 2: Ex, static [c0 - 1, c1) x [r0, r1 + 1), and the window with the first push's current
  {
    const int w = c1 - c0 + 1, ns = w * (r1 - r0 + 1);
    for (int k = tid; k < ns + nw; k += nth) {
      if (k >= ns) { window_e<T, 0>(a, k - ns); continue; }
      const int i = c0 - 1 + k % w, j = r0 + k / w;
      const uint8_t kd = kind_of(i, j);
      T e = z.Ex.at(i, j);
      const T hx = z.Hx.at(i, j), hxm = z.Hx.at(i, j - 1), hy = z.Hy.at(i, j), hym = z.Hy.at(i, j - 1);
      if (kd == kKindNone) continue;
      ex_cell(a, kd, cut_of(kd, i, j), e, hx, hxm, hy, hym, x.zeroJ);
      z.Ex.at(i, j) = e;
    }
  }
  sync();
  for (int k = tid; k < exchange_items(L0, L1, 1); k += nth) exchange_body(z, 1, k);
  sync();
  // 3: half H, static [c0 - 1, c1) x [r0, r1), and the window
  {
    const int w = c1 - c0 + 1, ns = w * (r1 - r0);
    for (int k = tid; k < ns + nw; k += nth) {
      if (k >= ns) { window_h(a, k - ns); continue; }
      const int i = c0 - 1 + k % w, j = r0 + k / w;
      fix_h(a, z, kind_of(i, j), i, j, cut_of);
    }
  }
  sync();
  for (int k = tid; k < exchange_items(L0, L1, 0); k += nth) exchange_body(z, 0, k);
  sync();
  // 4: static Ey on [c0, c1) x [r0, r1) (the window's Ey follows the second push)
  {
    const int w = c1 - c0, ns = w * (r1 - r0);
    for (int k = tid; k < ns; k += nth) {
      const int i = c0 + k % w, j = r0 + k / w;
      const uint8_t kd = kind_of(i, j);
      T e = z.Ey.at(i, j);
      const T hx = z.Hx.at(i, j), hxl = z.Hx.at(i - 1, j), hy = z.Hy.at(i, j), hyl = z.Hy.at(i - 1, j);
      if (kd == kKindNone) continue;
      ey_cell(a, kd, cut_of(kd, i, j), e, hx, hxl, hy, hyl, x.zeroJ);
      z.Ey.at(i, j) = e;
    }
  }
  sync();
  {
    const int w = c1 - c0, nr = w * (r1 - r0);
    for (int k = tid; k < 4 * nr; k += nth) {
      const int p = k / nr, rem = k % nr, i = c0 + rem % w, j = r0 + rem / w;
      const PlaneT<T> &src = p == 0 ? z.Ex : p == 1 ? z.Ey : p == 2 ? z.Hx : z.Hy;
      const PlaneT<T> &dst = p == 0 ? x.out[0] : p == 1 ? x.out[1] : p == 2 ? x.out[2] : x.out[3];
      dst.at(i, j) = src.at(i, j);
    }
  }
}

struct ClusterSync {
  __device__ __forceinline__ void operator()() const { cluster_barrier(); }
};
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

template <class T>
__global__ void __cluster_dims__(kFixCtas, 1, 1) __launch_bounds__(kFixThreads)
    k_yee_fixup(FieldArgsT<T> a, YeeFixArgs<T> x) {
  yee_fixup(a, x, (int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(gridDim.x * blockDim.x), ClusterSync{});
}

// The window's Ey sub-step with the second push's current, and the Ey strip
// exchange: the thread of window cell (0, j) also writes it to the static
// mesh; the static column right of the window fills the window's guard
// column (the static Ey there is final since the fused sweep).
template <class T>
__device__ __forceinline__ void window_ey_body(const FieldArgsT<T> &a, int k) {
  const int nw = a.L0 * a.L1;
  if (k < nw) {
    window_e<T, 1>(a, k);
    if (k % a.L0 == 0) exchange_body(a, 2, k / a.L0);
  } else if (k - nw < a.L1 + 2) {
    exchange_body(a, 2, a.L1 + (k - nw));
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_window_ey(FieldArgsT<T> a) {
  window_ey_body(a, (int)(blockIdx.x * blockDim.x + threadIdx.x));
}

// --- the fused sweep of a batch of members: one persistent launch ------------
//
// A work queue (one counter, reset before the launch) hands out the items in
// order: first every member's window fix-up (one CTA each, the longest
// items), then every member's tiles.  Items do not depend on one another (a
// tile reads the source set only, the fix-up writes cells no tile writes), so
// no CTA waits for another; each staging wait is bounded (kErrStaging).
template <class T>
struct YeeBatchFix {
  FieldArgsT<T> a;   // static planes: the source set; the window; the first push's current
  YeeFixArgs<T> x;
};

template <class T>
__global__ void __launch_bounds__(256, 5) k_yee_batch(const YeeTileArgs<T> *targs, const YeeBatchFix<T> *fix,
                                                      const int *tpre, int m, unsigned *queue) {
  using G = YeeTile<T>;
  extern __shared__ uint8_t smem_raw[];
  __shared__ int s_ncut, s_item;
  uint8_t *base = align128(smem_raw);
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + 4 * G::PLANE_BYTES + G::KIND_BYTES);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_init_fence();
  }
  const int total = m + __ldg(tpre + m);
  uint32_t parity = 0;
  for (;;) {
    // the previous item's shared-memory reads and writes come before the
    // next staging copies overwrite it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int item = s_item;
    if (item >= total) break;
    if (item < m) {
      yee_fixup(fix[item].a, fix[item].x, (int)threadIdx.x, (int)blockDim.x, CtaSync{});
      continue;
    }
    const int t = item - m;
    int lo = 0, hi = m - 1;  // member of tile t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(tpre + mid) <= t) lo = mid; else hi = mid - 1;
    }
    const int rc = yee_tile(targs[lo], t - __ldg(tpre + lo), parity, base, &s_ncut);
    if (rc == 2) break;  // the barrier may still receive copies: this CTA stops
    parity ^= 1u;
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_window_ey_batch(const FieldArgsT<T> *args, const int *bpre, int m) {
  const int mm = batch_member(bpre, m, blockIdx.x);
  window_ey_body(args[mm], (int)((blockIdx.x - bpre[mm]) * blockDim.x + threadIdx.x));
}

// --- kernels: one member, and a batch of members in one launch --------------

template <class T>
__global__ void __launch_bounds__(256) k_half_h(FieldArgsT<T> a) { half_h_body(a, blockIdx.x); }

template <class T, int COMP>
__global__ void __launch_bounds__(256) k_update_e(FieldArgsT<T> a, T zeroJ) { update_e_body<T, COMP>(a, blockIdx.x, zeroJ); }

template <class T>
__global__ void k_exchange(FieldArgsT<T> a, int which) { exchange_body(a, which, blockIdx.x * blockDim.x + threadIdx.x); }

template <class T>
__global__ void __launch_bounds__(1024) k_move(MoveArgs<T> m) { move_body(m); }

// The move of one member as three launches: the two copy phases over many
// CTAs (each takes the decision itself; nothing it reads changes before the
// last launch), then the decision's bookkeeping and the strips in one CTA.
template <class T>
__global__ void __launch_bounds__(256) k_move_copy(MoveArgs<T> m, int stage) {
  const WinState *ws = m.f.ws;
  if (ws->err) return;
  const MoveDecision d = move_decision(ws, m.f.L0, m.f.L1);
  if (!d.ok || (d.moveI == 0 && d.dj == 0)) return;
  move_copy(m, d.moveI, d.dj, stage, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <class T>
__global__ void __launch_bounds__(1024) k_move_finish(MoveArgs<T> m) {
  WinState *ws = m.f.ws;
  if (ws->err) return;
  __shared__ int s_move[3];
  if (threadIdx.x == 0) {
    const MoveDecision d = move_decision(ws, m.f.L0, m.f.L1);
    if (!d.ok) set_err(ws, d.err);
    s_move[0] = d.ok; s_move[1] = d.moveI; s_move[2] = d.dj;
    if (d.ok) { ws->moves[0] = d.moveI; ws->moves[1] = d.dj; }
  }
  __syncthreads();
  if (!s_move[0] || (s_move[1] == 0 && s_move[2] == 0)) return;
  move_finish(m, s_move[1], s_move[2]);
}


// The member's arguments are read in place: every thread of a block reads the
// same words, which the L1 cache serves after the first.
template <class T>
__device__ __forceinline__ const FieldArgsT<T> &batch_args(const FieldArgsT<T> *args, int mm) {
  return args[mm];
}

template <class T>
__global__ void __launch_bounds__(256) k_half_h_batch(const FieldArgsT<T> *args, const int *bpre, int m) {
  const int mm = batch_member(bpre, m, blockIdx.x);
  const FieldArgsT<T> &a = batch_args(args, mm);
  half_h_body(a, blockIdx.x - bpre[mm]);
}

template <class T, int COMP>
__global__ void __launch_bounds__(256) k_update_e_batch(const FieldArgsT<T> *args, const int *bpre, int m) {
  const int mm = batch_member(bpre, m, blockIdx.x);
  const FieldArgsT<T> &a = batch_args(args, mm);
  update_e_body<T, COMP>(a, blockIdx.x - bpre[mm], T(0));
}

template <class T>
__global__ void k_exchange_batch(const FieldArgsT<T> *args, const int *bpre, int m, int which) {
  const int mm = batch_member(bpre, m, blockIdx.x);
  const FieldArgsT<T> &a = batch_args(args, mm);
  exchange_body(a, which, (blockIdx.x - bpre[mm]) * blockDim.x + threadIdx.x);
}

template <class T>
__global__ void __launch_bounds__(1024) k_move_batch(const MoveArgs<T> *args) {
  __shared__ MoveArgs<T> sm;
  if (threadIdx.x == 0) sm = args[blockIdx.x];
  __syncthreads();
  move_body(sm);
}

// SCBoundaryCondition::resetOutsideDomain (SCBoundaryCondition.hh:163-195):
// E = 0 on cells that are neither inside nor a kept cut cell, and on cut
// cells per component.  cutidx maps a cell to its cut-cell entry or -1.
template <class T>
__global__ void k_reset_outside(FieldArgsT<T> a, const int *cutidx) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)a.Nx * a.Ny) return;
  if (a.mask[k]) return;
  const int i = (int)(k % a.Nx), j = (int)(k / a.Nx);
  const int c = cutidx[k];
  if (c < 0) { a.Ex.at(i, j) = T(0); a.Ey.at(i, j) = T(0); return; }
  const CutCellDev cc = a.cells[c];
  if (cc.l0 < kSpaceEps) a.Ex.at(i, j) = T(0);
  if (cc.l1 < kSpaceEps) a.Ey.at(i, j) = T(0);
  if (cc.area < kMinArea) { a.Ex.at(i, j) = T(0); a.Ey.at(i, j) = T(0); }
}

// --- host launchers -----------------------------------------------------------

int exchange_count(int L0, int L1, int which) {
  return which == 0 ? 2 * (L0 + L1) + 4 : which == 1 ? 2 * L0 + 2 : 2 * L1 + 2;
}

template <class T>
int sub_grid(FieldArgsT<T> &a) {
  if (a.tx <= 0 || a.ty <= 0 || a.tx * a.ty != 256 || a.tx % 32) { a.tx = 32; a.ty = 8; }
  a.tilesX = (a.Nx + 2 + a.tx * (16 / (int)sizeof(T)) - 1) / (a.tx * (16 / (int)sizeof(T)));
  a.nbS = a.tilesX * ((a.Ny + a.ty - 1) / a.ty);
  a.nbC = (a.ncells + 255) / 256;
  a.nbP = a.pml ? (a.npml + 255) / 256 : 0;
  const int nbM = (a.L0 * a.L1 + 255) / 256;
  return a.nbS + a.nbC + a.nbP + nbM;
}

template <class T>
void launch_half_h(FieldArgsT<T> a, cudaStream_t s) {
  const int g = sub_grid(a);
  k_half_h<T><<<g, 256, 0, s>>>(a);
}

template <class T>
void launch_update_e(FieldArgsT<T> a, int comp, cudaStream_t s) {
  const int g = sub_grid(a);
  if (comp == 0) k_update_e<T, 0><<<g, 256, 0, s>>>(a, T(0));
  else k_update_e<T, 1><<<g, 256, 0, s>>>(a, T(0));
}

template <class T>
void launch_exchange(FieldArgsT<T> a, int which, cudaStream_t s) {
  const int n = exchange_count(a.L0, a.L1, which);
  k_exchange<T><<<(n + 127) / 128, 128, 0, s>>>(a, which);
}

template <class T>
void launch_copy_to_window(FieldArgsT<T> a, cudaStream_t s) {
  k_copy_to_window<T><<<(a.L0 * a.L1 + 255) / 256, 256, 0, s>>>(a);
}

template <class T>
void launch_check_window(FieldArgsT<T> a, cudaStream_t s) { k_check_window<T><<<1, 256, 0, s>>>(a); }

template <class T>
void launch_move(FieldArgsT<T> a, T *scratch, double h0, double h1, cudaStream_t s) {
  MoveArgs<T> m{a, scratch, h0, h1};
  const int n = 6 * (a.L0 + 2) * (a.L1 + 2), g = std::min((n + 255) / 256, 592);
  k_move_copy<T><<<g, 256, 0, s>>>(m, 0);
  k_move_copy<T><<<g, 256, 0, s>>>(m, 1);
  k_move_finish<T><<<1, 1024, 0, s>>>(m);
}

// Batched sub-steps over m members: args and bpre are device arrays (bpre:
// first block of each member, m + 1 entries, built from sub_grid / exchange
// counts); nblocks = bpre[m].
template <class T>
void launch_half_h_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, cudaStream_t s) {
  if (nblocks > 0) k_half_h_batch<T><<<nblocks, 256, 0, s>>>(args, bpre, m);
}
template <class T>
void launch_update_e_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, int comp,
                           cudaStream_t s) {
  if (nblocks <= 0) return;
  if (comp == 0) k_update_e_batch<T, 0><<<nblocks, 256, 0, s>>>(args, bpre, m);
  else k_update_e_batch<T, 1><<<nblocks, 256, 0, s>>>(args, bpre, m);
}
template <class T>
void launch_exchange_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, int which,
                           cudaStream_t s) {
  if (nblocks > 0) k_exchange_batch<T><<<nblocks, 128, 0, s>>>(args, bpre, m, which);
}
template <class T>
void launch_move_batch(const MoveArgs<T> *args, int m, cudaStream_t s) {
  if (m > 0) k_move_batch<T><<<m, 1024, 0, s>>>(args);
}


template <class T>
void launch_reset_outside(FieldArgsT<T> a, const int *cutidx, cudaStream_t s) {
  const long long n = (long long)a.Nx * a.Ny;
  k_reset_outside<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, cutidx);
}

// --- fused sweep: host side ---------------------------------------------------

EncodeTiled tensor_map_encoder() {
  static const EncodeTiled fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiled) nullptr;
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// Row-major 2-D map of w x h elements, rows pitch_bytes apart, box bw x bh;
// reads outside the tensor return zero.
static bool encode_2d(CUtensorMap *m, CUtensorMapDataType dt, const void *base, uint64_t w, uint64_t h,
                      uint64_t pitch_bytes, uint32_t bw, uint32_t bh) {
  const EncodeTiled enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {w, h};
  const cuuint64_t strides[1] = {pitch_bytes};
  const cuuint32_t box[2] = {bw, bh};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, dt, 2, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The tile arguments of one sweep (tensor maps over a's static planes, the
// source set) and its tile-grid height.
template <class T>
static int fill_tile_args(YeeTileArgs<T> &t, const FieldArgsT<T> &a, const PlaneT<T> *dst, const uint8_t *kind,
                          int kpitch, const int *cutidx, long long spin, int *tilesY) {
  using G = YeeTile<T>;
  if (kpitch < a.Nx + 2 || kpitch % 16) return kErrArg;
  for (int p = 1; p < 4; ++p)  // the tiles store the four planes with one row pitch
    if (dst[p].pitch != dst[0].pitch) return kErrArg;
  const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const PlaneT<T> *src[4] = {&a.Ex, &a.Ey, &a.Hx, &a.Hy};
  for (int p = 0; p < 4; ++p) {
    if ((src[p]->pitch * sizeof(T)) % 16 || (reinterpret_cast<uintptr_t>(src[p]->p) & 15)) return kErrArg;
    if (!encode_2d(&t.map[p], dt, src[p]->p, (uint64_t)a.Nx + 2, (uint64_t)a.Ny + 2,
                   (uint64_t)src[p]->pitch * sizeof(T), G::W, G::H))
      return kErrCuda;
  }
  if (!encode_2d(&t.map[4], CU_TENSOR_MAP_DATA_TYPE_UINT8, kind, (uint64_t)a.Nx + 2, (uint64_t)a.Ny + 2,
                 (uint64_t)kpitch, G::KW, G::H))
    return kErrCuda;
  t.f = a;
  for (int p = 0; p < 4; ++p) t.out[p] = dst[p];
  t.cutidx = cutidx;
  t.tilesX = (a.Nx + 2 + G::TX - 1) / G::TX;
  *tilesY = (a.Ny + G::TY - 1) / G::TY;
  t.zeroJ = T(0);
  t.spin = spin;
  return kOk;
}

template <class T>
static void fill_fix_args(YeeFixArgs<T> &x, const PlaneT<T> *dst, const uint8_t *kind, int kpitch,
                          const int *cutidx, T *z, int zpitch, int zrows) {
  for (int p = 0; p < 4; ++p) x.out[p] = dst[p];
  x.z = z; x.zpitch = zpitch; x.zrows = zrows;
  x.kind = kind; x.kpitch = kpitch; x.cutidx = cutidx;
  x.zeroJ = T(0);
}

template <class T>
int launch_yee_fused(const FieldArgsT<T> &a, const PlaneT<T> *dst, const uint8_t *kind, int kpitch,
                     const int *cutidx, T *z, int zpitch, int zrows, long long spin, cudaStream_t s, cudaStream_t s2,
                     cudaEvent_t fork, cudaEvent_t join) {
  using G = YeeTile<T>;
  if (zpitch < a.L0 + 6 || zrows < a.L1 + 7) return kErrArg;
  YeeTileArgs<T> t;
  int tilesY = 0;
  const int rc = fill_tile_args(t, a, dst, kind, kpitch, cutidx, spin, &tilesY);
  if (rc != kOk) return rc;
  if (cudaFuncSetAttribute(k_yee_tiles<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess)
    return kErrCuda;
  YeeFixArgs<T> x;
  fill_fix_args(x, dst, kind, kpitch, cutidx, z, zpitch, zrows);
  // the tiles and the fix-up write disjoint cells and read only the source
  // set: the fix-up runs on s2 beside the tiles, s waits for both
  if (cudaEventRecord(fork, s) != cudaSuccess || cudaStreamWaitEvent(s2, fork, 0) != cudaSuccess) return kErrCuda;
  k_yee_fixup<T><<<kFixCtas, kFixThreads, 0, s2>>>(a, x);
  k_yee_tiles<T><<<t.tilesX * tilesY, G::THREADS, G::SMEM, s>>>(t);
  if (cudaEventRecord(join, s2) != cudaSuccess || cudaStreamWaitEvent(s, join, 0) != cudaSuccess) return kErrCuda;
  return kOk;
}

template <class T>
void launch_window_ey(const FieldArgsT<T> &a, cudaStream_t s) {
  const int n = a.L0 * a.L1 + a.L1 + 2;
  k_window_ey<T><<<(n + 255) / 256, 256, 0, s>>>(a);
}

template <class T>
size_t yee_batch_bytes(int which) {
  return which == 0 ? sizeof(YeeTileArgs<T>) : sizeof(YeeBatchFix<T>);
}

template <class T>
int yee_batch_entry(const FieldArgsT<T> &a, const PlaneT<T> *dst, const uint8_t *kind, int kpitch, const int *cutidx,
                    T *z, int zpitch, int zrows, long long spin, void *tile_out, void *fix_out, int *ntiles) {
  if (zpitch < a.L0 + 6 || zrows < a.L1 + 7) return kErrArg;
  YeeTileArgs<T> &t = *static_cast<YeeTileArgs<T> *>(tile_out);
  int tilesY = 0;
  const int rc = fill_tile_args(t, a, dst, kind, kpitch, cutidx, spin, &tilesY);
  if (rc != kOk) return rc;
  *ntiles = t.tilesX * tilesY;
  YeeBatchFix<T> &f = *static_cast<YeeBatchFix<T> *>(fix_out);
  f.a = a;
  fill_fix_args(f.x, dst, kind, kpitch, cutidx, z, zpitch, zrows);
  return kOk;
}

template <class T>
int launch_yee_batch(const void *targs, const void *fix, const int *tpre, int m, unsigned *queue, cudaStream_t s) {
  using G = YeeTile<T>;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaFuncSetAttribute(k_yee_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) != cudaSuccess ||
      cudaMemsetAsync(queue, 0, sizeof(unsigned), s) != cudaSuccess)
    return kErrCuda;
  k_yee_batch<T><<<5 * sms, G::THREADS, G::SMEM, s>>>(static_cast<const YeeTileArgs<T> *>(targs),
                                                        static_cast<const YeeBatchFix<T> *>(fix), tpre, m, queue);
  return kOk;
}

template <class T>
void launch_window_ey_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, cudaStream_t s) {
  if (nblocks > 0) k_window_ey_batch<T><<<nblocks, 256, 0, s>>>(args, bpre, m);
}

// Cell kinds in the static storage layout (guards and padding stay none).
__global__ void k_build_kind(const uint8_t *mask, const int *cutidx, int Nx, int Ny, uint8_t *kind, int kpitch) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)Nx * Ny) return;
  const int i = (int)(k % Nx), j = (int)(k / Nx);
  kind[(size_t)(j + 1) * kpitch + (i + 1)] = mask[k] ? kKindRegular : cutidx[k] >= 0 ? kKindCut : kKindNone;
}

void launch_build_kind(const uint8_t *mask, const int *cutidx, int Nx, int Ny, uint8_t *kind, int kpitch,
                       cudaStream_t s) {
  const long long n = (long long)Nx * Ny;
  k_build_kind<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mask, cutidx, Nx, Ny, kind, kpitch);
}

#define CSRST_FIELDS_INSTANTIATE(T)                                                         \
  template void launch_half_h<T>(FieldArgsT<T>, cudaStream_t);                              \
  template void launch_update_e<T>(FieldArgsT<T>, int, cudaStream_t);                       \
  template void launch_exchange<T>(FieldArgsT<T>, int, cudaStream_t);                       \
  template void launch_copy_to_window<T>(FieldArgsT<T>, cudaStream_t);                      \
  template void launch_check_window<T>(FieldArgsT<T>, cudaStream_t);                        \
  template void launch_move<T>(FieldArgsT<T>, T *, double, double, cudaStream_t);           \
  template void launch_reset_outside<T>(FieldArgsT<T>, const int *, cudaStream_t);                \
  template int sub_grid<T>(FieldArgsT<T> &);                                                \
  template void launch_half_h_batch<T>(const FieldArgsT<T> *, const int *, int, int, cudaStream_t); \
  template void launch_update_e_batch<T>(const FieldArgsT<T> *, const int *, int, int, int, cudaStream_t); \
  template void launch_exchange_batch<T>(const FieldArgsT<T> *, const int *, int, int, int, cudaStream_t); \
  template void launch_move_batch<T>(const MoveArgs<T> *, int, cudaStream_t);                        \
  template int launch_yee_fused<T>(const FieldArgsT<T> &, const PlaneT<T> *, const uint8_t *, int, const int *, T *, \
                                   int, int, long long, cudaStream_t, cudaStream_t, cudaEvent_t, cudaEvent_t); \
  template void launch_window_ey<T>(const FieldArgsT<T> &, cudaStream_t);                            \
  template size_t yee_batch_bytes<T>(int);                                                          \
  template int yee_batch_entry<T>(const FieldArgsT<T> &, const PlaneT<T> *, const uint8_t *, int, const int *, T *, \
                                  int, int, long long, void *, void *, int *);                      \
  template int launch_yee_batch<T>(const void *, const void *, const int *, int, unsigned *, cudaStream_t); \
  template void launch_window_ey_batch<T>(const FieldArgsT<T> *, const int *, int, int, cudaStream_t);
CSRST_FIELDS_INSTANTIATE(double)
CSRST_FIELDS_INSTANTIATE(float)

}  // namespace csrst
