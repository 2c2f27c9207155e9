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
#include "kernels.cuh"

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
    const int i = k % a.L0, j = k / a.L0;
    T &hx = a.mHx.at(i, j), &hy = a.mHy.at(i, j);
    hx = hx - a.chx * (a.mEy.at(i + 1, j) - a.mEy.at(i, j));
    hy = hy + a.chy * (a.mEx.at(i, j + 1) - a.mEx.at(i, j));
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
// Communicator.cpp:123-642).  One CTA: reads the last deposit's particle
// bounds, shifts the window by whole cells through a scratch copy, updates
// the window position and origin, then refreshes the strips.

template <class T>
__device__ __forceinline__ void move_body(const MoveArgs<T> &m) {
  const FieldArgsT<T> &a = m.f;
  WinState *ws = a.ws;
  if (ws->err) return;
  const int L[2] = {a.L0, a.L1};
  __shared__ int s_move[3];
  if (threadIdx.x == 0) {
    int ok = 1, ideal1[2];
    for (int d = 0; d < 2; ++d) {
      const int len = ws->gb[2 * d + 1] - ws->gb[2 * d] + 1;
      if (len >= L[d]) { ok = 0; break; }
      const unsigned diff = (unsigned)(L[d] - len);
      const unsigned up = (unsigned)floor(diff / 2.0);
      ideal1[d] = L[d] - (int)up - 2;
    }
    int moveI = 0, dj = 0;
    if (!ok) set_err(ws, kErrWindowFit);
    else {
      moveI = ws->gb[1] - ideal1[0] - 1;
      dj = ws->gb[3] - ideal1[1] - 1;
      if (moveI < 0 || moveI > 1 || dj < -1 || dj > 1) { set_err(ws, kErrWindowMove); ok = 0; }
    }
    s_move[0] = ok; s_move[1] = moveI; s_move[2] = dj;
    if (ok) { ws->moves[0] = moveI; ws->moves[1] = dj; }
  }
  __syncthreads();
  if (!s_move[0]) return;
  const int moveI = s_move[1], m1 = s_move[2];
  if (moveI == 0 && m1 == 0) return;
  const int W0 = a.L0 + 2, W1 = a.L1 + 2, np = W0 * W1;
  const PlaneT<T> *pl[6] = {&a.mEx, &a.mEy, &a.mHx, &a.mHy, &a.mJx, &a.mJy};
  // phase A: snapshot
  for (int k = threadIdx.x; k < 6 * np; k += blockDim.x) {
    const int f = k / np, r = k % np;
    m.scratch[k] = pl[f]->p[r];
  }
  __syncthreads();
  // phase B: shifted copy over the reference's loop ranges
  const int i0 = -moveI, i1 = a.L0 - 1;
  int j0 = -(m1 > 0 ? m1 : 0), j1 = a.L1 - 1 - (m1 < 0 ? m1 : 0);
  if (m1 == 0) { j0 -= 1; j1 += 1; }
  const int ni = i1 - i0 + 1, cnt = ni * (j1 - j0 + 1);
  for (int k = threadIdx.x; k < 6 * cnt; k += blockDim.x) {
    const int f = k / cnt, r = k % cnt;
    const int i = i0 + r % ni, j = j0 + r / ni;
    pl[f]->at(i, j) = m.scratch[(size_t)f * np + (size_t)(j + m1 + 1) * W0 + (i + moveI + 1)];
  }
  __syncthreads();
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

// --- kernels: one member, and a batch of members in one launch --------------

template <class T>
__global__ void __launch_bounds__(256) k_half_h(FieldArgsT<T> a) { half_h_body(a, blockIdx.x); }

template <class T, int COMP>
__global__ void __launch_bounds__(256) k_update_e(FieldArgsT<T> a, T zeroJ) { update_e_body<T, COMP>(a, blockIdx.x, zeroJ); }

template <class T>
__global__ void k_exchange(FieldArgsT<T> a, int which) { exchange_body(a, which, blockIdx.x * blockDim.x + threadIdx.x); }

template <class T>
__global__ void __launch_bounds__(1024) k_move(MoveArgs<T> m) { move_body(m); }

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
  k_move<T><<<1, 1024, 0, s>>>(m);
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
  template void launch_move_batch<T>(const MoveArgs<T> *, int, cudaStream_t);
CSRST_FIELDS_INSTANTIATE(double)
CSRST_FIELDS_INSTANTIATE(float)

}  // namespace csrst
