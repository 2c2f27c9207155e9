// FP32 mode particle kernels: the same fused push as particles.cu
// (PartBunch::push_particles, PartBunch.cpp:215-519) on a bunch stored as
// FP32 offsets from FP64 cell origins and FP32 momentum deviations from an
// FP64 reference momentum.
//
// Precision split (what stays FP64 and why):
//   - 1/gamma: the reference's float Q_rsqrt of 1 + |P|^2 formed in FP64, so
//     velocities match the FP64 path's (utils.hh:491-504);
//   - positions during the push: cell-relative doubles built exactly from
//     the stored offsets, so no precision is lost to the distance from the
//     mesh origin; the stored offset is rounded to FP32 once per push;
//   - the current deposit: FP64 weights on those exact positions, so the
//     discrete continuity equation holds to FP64 rounding;
//   - the hard-edge dipole test: absolute position in FP64 (the bend frame).
// The field gather (27 taps for TSC) and the kick/rotation run in FP32; the
// gather is anchored at the particle's own window cell, so its coordinates
// are offsets of magnitude < 2 and keep FP32's full resolution.
// This file is built with FMA contraction on: FP32 mode is checked against
// the FP64 path to a tolerance, not bit for bit.
#include "accum.cuh"
#include "bbox.cuh"
#include "bunch32.cuh"
#include "kernels.cuh"
#include "shapes.cuh"

namespace csrst {
namespace {

__device__ __forceinline__ long long gtid() { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }

struct View32 {
  const float *base;  // window element of the particle's cell
  int pitch;
  __device__ __forceinline__ float operator()(int i, int j) const { return __ldg(base + (ptrdiff_t)j * pitch + i); }
};
struct SumView32 {
  View32 a, b;
  __device__ __forceinline__ float operator()(int i, int j) const { return a(i, j) + b(i, j); }
};

// Cell of the cell-relative coordinate t of cell c, as c' + 0.5 (exact).
__device__ __forceinline__ double cellc(int c, double t) { return (double)(c + (int)floor(t)) + 0.5; }

// Store a cell-relative position t (cells) of cell (ci, cj) as cell + offset.
__device__ __forceinline__ void store_pos(double t0, double t1, int ci, int cj, int &cell, float &o0, float &o1) {
  double f0 = floor(t0), f1 = floor(t1);
  float a0 = (float)(t0 - f0), a1 = (float)(t1 - f1);
  if (a0 >= 1.0f) { a0 = 0.0f; f0 += 1.0; }  // rounded up to the next cell
  if (a1 >= 1.0f) { a1 = 0.0f; f1 += 1.0; }
  cell = ((ci + (int)f0) & 0xffff) | ((cj + (int)f1) << 16);
  o0 = a0; o1 = a1;
}

// One particle's move: gather at R1, kick + rotation, drift to R2, R2 stored
// (cell + FP32 offset) and the new momentum deviation stored.  On return,
// when ok: r0 = R0 (deposit start) and e = R2 (end, as stored) in cells from
// the old cell (ci, cj); (ni, nj) the new cell and w the half drift of the
// new momentum.  Particles that fail the window-fit checks set the member's
// error and come back with ok false, unchanged.
struct Move32 {
  bool ok;
  int ci, cj, ni, nj;
  double r00, r01, e0, e1, w0, w1, q;
  float o0, o1;
};

template <int ORDER_OF_PUSH>
__device__ __forceinline__ void move32(const Push32Args &a, long long n, bool ok, int L0, int L1, int WP0, int WP1,
                                       Move32 &m) {
  WinState *ws = a.ws;
  const int wp = a.wpitch;
  const double P0 = a.P0, P1 = a.P1;
  const float Pf0 = (float)P0, Pf1 = (float)P1;
  int ci = 0, cj = 0;
  double s0 = 0.0, s1 = 0.0, q = 0.0;
  float d0 = 0.0f, d1 = 0.0f;
  if (ok) {
    unpack(a.b.cell[n], ci, cj);
    s0 = a.b.ox[n]; s1 = a.b.oy[n];
    d0 = a.b.dpx[n]; d1 = a.b.dpy[n];
    q = a.b.q[n];
    if (!(isfinite(d0) && isfinite(d1) && s0 >= 0.0 && s0 < 1.0 && s1 >= 0.0 && s1 < 1.0)) {
      set_err(ws, kErrWindowFit);
      ok = false;
    }
  }
  double p0 = 0.0, p1 = 0.0, w0 = 0.0, w1 = 0.0, r00 = 0.0, r01 = 0.0, x0 = 0.0, x1 = 0.0;
  if (ok) {
    const float r = rgam(P0, P1, d0, d1, p0, p1);
    w0 = half_drift(a.kh0, p0, r); w1 = half_drift(a.kh1, p1, r);
    r00 = s0; r01 = s1;
    if (a.pending) { r00 = dsub(s0, w0); r01 = dsub(s1, w1); }  // drift_particles(-dt/2)
    x0 = dadd(r00, w0); x1 = dadd(r01, w1);                     // R1, cells from (ci, cj)
    const int wi = ci - WP0, wj = cj - WP1;
    // gather (FieldPatch::gather x3) anchored at the window cell of R1; the
    // offset inside it is clamped below 1 so that FP32 rounding cannot move
    // the stencil to the next cell (the window-fit check counts cells in FP64)
    const double c0 = floor(x0), c1 = floor(x1);
    const int ai = wi + (int)c0, aj = wj + (int)c1;
    if (ai - 2 < -1 || ai + 2 > L0 || aj - 2 < -1 || aj + 2 > L1) {  // stencil outside the window planes
      set_err(ws, kErrWindowFit);
      ok = false;
    } else {
      const float g0 = fminf((float)(x0 - c0), 0x1.fffffep-1f), g1 = fminf((float)(x1 - c1), 0x1.fffffep-1f);
      const size_t o = (size_t)(aj + 1) * wp + (ai + 1);
      const View32 vex{a.mEx + o, wp}, vey{a.mEy + o, wp}, vhx{a.mHx + o, wp}, vhy{a.mHy + o, wp};
      const float E0 = gather_edge<ORDER_OF_PUSH>(vex, g0, g1, 0);
      const float E1 = gather_edge<ORDER_OF_PUSH>(vey, g0, g1, 1);
      const float Hf = gather_cell<ORDER_OF_PUSH>(SumView32{vhx, vhy}, g0, g1);
      // hard-edge dipole at the absolute position of R1
      const double X = a.org0 + ((double)ci + x0) * a.h0, Y = a.org1 + ((double)cj + x1) * a.h1;
      const double dist = a.chh * (X - a.Lb) - a.shh * (Y - a.hw);
      const float bext = (dist > 0.0 && dist < a.bwidth) ? (float)a.bz : 0.0f;
      const float B = (float)kMu0 * Hf + 0.5f * bext;
      // kick + rotation (PartBunch.cpp:366-383) on u - P
      const float k0 = a.f1 * E0, k1 = a.f1 * E1;
      const float du0 = d0 + k0, du1 = d1 + k1;
      double U0, U1;
      const float ru = rgam(P0, P1, du0, du1, U0, U1);
      const float aa = a.f2 * B * ru;
      const float sv0 = du0 + aa * (Pf1 + du1), sv1 = du1 - aa * (Pf0 + du0);  // s - P
      const float cf = aa / (1.0f + aa * aa);
      d0 = (sv0 + cf * (Pf1 + sv1)) + k0;
      d1 = (sv1 - cf * (Pf0 + sv0)) + k1;
      a.b.dpx[n] = d0; a.b.dpy[n] = d1;
    }
  }
  m.ok = ok;
  m.ci = ci; m.cj = cj; m.r00 = r00; m.r01 = r01; m.q = q;
  m.ni = 0; m.nj = 0; m.e0 = 0.0; m.e1 = 0.0; m.o0 = 0.0f; m.o1 = 0.0f; m.w0 = 0.0; m.w1 = 0.0;
  if (ok) {
    const float r = rgam(P0, P1, d0, d1, p0, p1);
    w0 = half_drift(a.kh0, p0, r); w1 = half_drift(a.kh1, p1, r);
    int nc;
    float o0, o1;
    store_pos(dadd(x0, w0), dadd(x1, w1), ci, cj, nc, o0, o1);  // R2
    a.b.cell[n] = nc; a.b.ox[n] = o0; a.b.oy[n] = o1;
    // the move ends at the stored (FP32-rounded) position, so that every
    // move's current conserves charge for the positions the bunch holds
    unpack(nc, m.ni, m.nj);
    m.e0 = (double)(m.ni - ci) + (double)o0; m.e1 = (double)(m.nj - cj) + (double)o1;
    m.o0 = o0; m.o1 = o1; m.w0 = w0; m.w1 = w1;
  }
}

// Boxes of one moved particle: R0 u R2 (the deposit bounds) and the next
// push's gather position.  Boxes hold cell index + 0.5: only the cells are
// used, and a cell-relative coordinate added to a large index could round
// across a cell border.
struct Boxes32 {
  double amn0 = INFINITY, amn1 = INFINITY, amx0 = -INFINITY, amx1 = -INFINITY;  // R0 u R2 (cells)
  double bmn0 = INFINITY, bmn1 = INFINITY, bmx0 = -INFINITY, bmx1 = -INFINITY;  // next R1 (cells)
  __device__ __forceinline__ void add(const Move32 &m) {
    amn0 = fmin(amn0, cellc(m.ci, fmin(m.r00, m.e0))); amn1 = fmin(amn1, cellc(m.cj, fmin(m.r01, m.e1)));
    amx0 = fmax(amx0, cellc(m.ci, fmax(m.r00, m.e0))); amx1 = fmax(amx1, cellc(m.cj, fmax(m.r01, m.e1)));
    // next push gathers at (stored R2 - w) + w
    const double n0 = cellc(m.ni, dadd(dsub((double)m.o0, m.w0), m.w0));
    const double n1 = cellc(m.nj, dadd(dsub((double)m.o1, m.w1), m.w1));
    bmn0 = fmin(bmn0, n0); bmn1 = fmin(bmn1, n1); bmx0 = fmax(bmx0, n0); bmx1 = fmax(bmx1, n1);
  }
  __device__ __forceinline__ void store(WinState *ws, PushShared &sh) {
    block_bbox(amn0, amn1, amx0, amx1, ws->bball, sh.sb);
    block_bbox(bmn0, bmn1, bmx0, bmx1, ws->bb[1 - ws->cur], sh.sb);
  }
};

// Deposit state of one CTA: the warp tiles (dynamic shared memory) over the
// member's window accumulator in global memory.
template <int ORDER>
struct Depositor32 {
  using Tile = typename TileFor<ORDER>::T;
  Tile tile;
  unsigned long long *win;
  int L0, L1;
  double scale;
  bool overflow = false;

  // Called by all threads of the CTA; ends with a barrier.
  __device__ __forceinline__ void begin(const Push32Args &a, unsigned long long *sm, int l0, int l1) {
    L0 = l0; L1 = l1; scale = a.acc_scale;
    win = a.acc;
    for (int k = threadIdx.x; k < Tile::kSize * (int)blockDim.x; k += blockDim.x) sm[k] = 0ull;
    __syncthreads();
    tile.init(sm, L0, L1);
  }

  // Current of one move R0 -> R2 (cells from the old cell, whose window cell
  // is (wi, wj)), FP64 weights summed in the warp's tile.  Called by all
  // lanes of the warp together (has: this lane has a particle).
  __device__ __forceinline__ void particle(const Push32Args &a, bool has, int wi, int wj, double q, double r00,
                                           double r01, double e0, double e1) {
    tile.template rebase<false>(has, has ? wi + (int)floor(r00) : 0, has ? wj + (int)floor(r01) : 0, win, L0, L1);
    if (has) {
      auto sink = [&](int i, int j, double v) {
        tile.template add<false>(i + wi, j + wj, __double2ll_rn(v * scale), win, L0, L1);
      };
      if (!deposit_particle<ORDER>(a.jcomp, q, r00, r01, e0, e1, 0.0, 0.0, 1.0, 1.0, a.h0, a.h1, a.dt, sink))
        overflow = true;
    }
  }

  // Called by all threads of the CTA after their last particle(); ends with
  // a barrier.
  __device__ __forceinline__ void end(const Push32Args &a) {
    tile.template flush<false>(win, L0, L1);
    if (overflow) set_err(a.ws, kErrCrossings);
    __syncthreads();
  }
};

// The member's sticky error at entry, read by one thread for the CTA; a CTA
// that sees one leaves as a whole.
__device__ __forceinline__ bool entry_error(WinState *ws, PushShared &sh) {
  if (threadIdx.x == 0) sh.err = *(volatile int *)&ws->err;
  __syncthreads();
  return sh.err != 0;
}

// Move and deposit of one CTA's share [beg, end) of one member; called by
// all threads of the CTA, each ends with a barrier, so that a CTA may run
// them for several members in turn.
template <int ORDER>
__device__ __forceinline__ void move32_range(const Push32Args &a, long long beg, long long end, PushShared &sh) {
  if (entry_error(a.ws, sh)) return;  // the whole CTA leaves together
  WinState *ws = a.ws;
  const int L0 = ws->L0, L1 = ws->L1, WP0 = ws->P0, WP1 = ws->P1;
  Boxes32 box;
  for (long long n = beg + threadIdx.x; n < end; n += blockDim.x) {
    Move32 m;
    move32<ORDER>(a, n, true, L0, L1, WP0, WP1, m);
    a.dep_r0[2 * n] = m.ok ? m.r00 : NAN;
    a.dep_r0[2 * n + 1] = m.r01;
    a.dep_cell[n] = (m.ci & 0xffff) | (m.cj << 16);
    if (m.ok) box.add(m);
  }
  box.store(ws, sh);
  __syncthreads();
}

template <int ORDER>
__device__ __forceinline__ void dep32_range(const Push32Args &a, long long beg, long long end, PushShared &sh,
                                            unsigned long long *sacc) {
  if (entry_error(a.ws, sh)) return;
  WinState *ws = a.ws;
  const int L0 = ws->L0, L1 = ws->L1, WP0 = ws->P0, WP1 = ws->P1;
  Depositor32<ORDER> dep;
  dep.begin(a, sacc, L0, L1);
  // a round's inputs are loaded together, one round ahead, so that their
  // latency overlaps the deposit of the round before
  struct In {
    double2 r0;
    int c0, c1;
    float o0, o1, q;
  };
  auto load = [&](long long n, In &v) {
    if (n < end) {
      v.r0 = reinterpret_cast<const double2 *>(a.dep_r0)[n];
      v.c0 = a.dep_cell[n]; v.c1 = a.b.cell[n];
      v.o0 = a.b.ox[n]; v.o1 = a.b.oy[n]; v.q = a.b.q[n];
    } else {
      v.r0.x = NAN; v.r0.y = 0.0; v.c0 = v.c1 = 0; v.o0 = v.o1 = v.q = 0.0f;
    }
  };
  const long long rounds = end > beg ? (end - beg + blockDim.x - 1) / blockDim.x : 0;
  In cur, nxt;
  load(beg + threadIdx.x, cur);
  for (long long it = 0; it < rounds; ++it) {  // the same rounds for every lane
    if (it + 1 < rounds) load(beg + (it + 1) * blockDim.x + threadIdx.x, nxt);
    const bool has = !isnan(cur.r0.x);
    double e0 = 0.0, e1 = 0.0;
    int ci = 0, cj = 0;
    if (has) {
      unpack(cur.c0, ci, cj);
      int ni, nj;
      unpack(cur.c1, ni, nj);
      e0 = (double)(ni - ci) + (double)cur.o0;
      e1 = (double)(nj - cj) + (double)cur.o1;
    }
    dep.particle(a, has, ci - WP0, cj - WP1, (double)cur.q, cur.r0.x, cur.r0.y, e0, e1);
    cur = nxt;
  }
  dep.end(a);
}

// The FP32 push in two launches.  The move launch moves every particle
// (gather, kick, drift, stores, boxes) with no shared memory and leaves for
// the deposit each particle's start R0 and old cell in a.dep_r0 / a.dep_cell
// (NaN for a particle it did not move); the deposit launch then adds the
// current of every move R0 -> R2, CTA by CTA over contiguous (cell-sorted)
// ranges.  Both run at three CTAs per SM and are bound by the latency of
// dependent FP64 chains, not by bytes: split, each runs at 24 warps per SM
// where the fused push's 128 registers and 98 KB of shared memory (window
// accumulator copy + tiles) allowed 16 (4e6-particle TSC bunch, 8192 x 1024
// mesh: 0.50 -> 0.40 ms per push).  The extra traffic is 20 bytes written
// and 36 read per particle.
template <int ORDER>
__global__ void __launch_bounds__(256, 3) k_push32_move(Push32Args a) {
  __shared__ PushShared sh;
  const long long per = (a.b.n + gridDim.x - 1) / gridDim.x;
  const long long beg = (long long)blockIdx.x * per;
  move32_range<ORDER>(a, beg, beg + per < a.b.n ? beg + per : a.b.n, sh);
}

template <int ORDER>
__global__ void __launch_bounds__(256, 3) k_push32_dep(Push32Args a) {
  extern __shared__ unsigned long long sacc[];
  __shared__ PushShared sh;
  const long long per = (a.b.n + gridDim.x - 1) / gridDim.x;
  const long long beg = (long long)blockIdx.x * per;
  dep32_range<ORDER>(a, beg, beg + per < a.b.n ? beg + per : a.b.n, sh, sacc);
}

// One push over a batch of FP32-mode members in two launches, as for one
// member: the members' particles form one index range (ppre: first particle
// of each member, m + 1 entries) cut into equal contiguous shares, one per
// CTA; a CTA runs the move (then, in the second launch, the deposit) of every
// member its share overlaps.
template <int ORDER>
__global__ void __launch_bounds__(256, 3) k_push32_batch_move(const Push32Args *args, const long long *ppre, int m,
                                                            long long per) {
  __shared__ PushShared sh;
  __shared__ Push32Args sa;
  const long long total = ppre[m];
  const long long g0 = (long long)blockIdx.x * per;
  const long long g1 = g0 + per < total ? g0 + per : total;
  for (int mm = 0; mm < m; ++mm) {
    const long long b0 = ppre[mm], b1 = ppre[mm + 1];
    if (b1 <= g0 || b0 >= g1) continue;
    const long long lb = (g0 > b0 ? g0 : b0) - b0, le = (g1 < b1 ? g1 : b1) - b0;
    __syncthreads();
    if (threadIdx.x == 0) sa = args[mm];
    __syncthreads();
    move32_range<ORDER>(sa, lb, le, sh);
  }
}

template <int ORDER>
__global__ void __launch_bounds__(256, 3) k_push32_batch_dep(const Push32Args *args, const long long *ppre, int m,
                                                           long long per) {
  extern __shared__ unsigned long long sacc[];
  __shared__ PushShared sh;
  __shared__ Push32Args sa;
  const long long total = ppre[m];
  const long long g0 = (long long)blockIdx.x * per;
  const long long g1 = g0 + per < total ? g0 + per : total;
  for (int mm = 0; mm < m; ++mm) {
    const long long b0 = ppre[mm], b1 = ppre[mm + 1];
    if (b1 <= g0 || b0 >= g1) continue;
    const long long lb = (g0 > b0 ? g0 : b0) - b0, le = (g1 < b1 ? g1 : b1) - b0;
    __syncthreads();
    if (threadIdx.x == 0) sa = args[mm];
    __syncthreads();
    dep32_range<ORDER>(sa, lb, le, sh, sacc);
  }
}

// Gather-patch set-up and the window-fit check from the box of the next
// push's gather positions (cells of the static mesh).
__device__ __forceinline__ void prep32_body(WinState *ws, int reach) {
  const int c = ws->cur;
  const double mn0 = ord_dbl(ws->bb[c][0]), mn1 = ord_dbl(ws->bb[c][1]);
  const double mx0 = ord_dbl(ws->bb[c][2]), mx1 = ord_dbl(ws->bb[c][3]);
  if (mn0 <= mx0) {
    const int lp[4] = {(int)floor(mn0) - ws->P0, (int)floor(mx0) - ws->P0, (int)floor(mn1) - ws->P1,
                       (int)floor(mx1) - ws->P1};
    for (int k = 0; k < 4; ++k) ws->lp[k] = lp[k];
    // every gather tap lies within [lp - reach, lp + reach]
    if (lp[0] - reach < -1 || lp[1] + reach > ws->L0 || lp[2] - reach < -1 || lp[3] + reach > ws->L1)
      set_err(ws, kErrWindowFit);
  }
  bbox_reset(ws->bb[1 - c]);
  bbox_reset(ws->bball);
}

__global__ void k_prep32(WinState *ws, int reach) {
  if (threadIdx.x == 0) prep32_body(ws, reach);
}

// Deposit bounds in window cells (PartBunch::getLocalPDomainInclOld).
__device__ __forceinline__ void bounds32_body(WinState *ws) {
  const double mn0 = ord_dbl(ws->bball[0]), mn1 = ord_dbl(ws->bball[1]);
  const double mx0 = ord_dbl(ws->bball[2]), mx1 = ord_dbl(ws->bball[3]);
  if (!(mn0 <= mx0)) { ws->gb[0] = 0; ws->gb[1] = -1; ws->gb[2] = 0; ws->gb[3] = -1; return; }
  ws->gb[0] = (int)floor(mn0) - ws->P0; ws->gb[1] = (int)floor(mx0) - ws->P0;
  ws->gb[2] = (int)floor(mn1) - ws->P1; ws->gb[3] = (int)floor(mx1) - ws->P1;
}

__global__ void k_bounds32(WinState *ws) {
  if (threadIdx.x == 0) bounds32_body(ws);
}

__global__ void k_prep32_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) prep32_body(p[k].ws, 2);
}
__global__ void k_post32_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) p[k].ws->cur = 1 - p[k].ws->cur;
}
__global__ void k_bounds32_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) bounds32_body(p[k].ws);
}

__global__ void k_post32(WinState *ws) {
  if (threadIdx.x == 0) ws->cur = 1 - ws->cur;
}

__global__ void k_bbox32_clear(WinState *ws) {
  if (threadIdx.x == 0) bbox_reset(ws->bb[ws->cur]);
}

// Box of the next push's gather positions R1 = (R - w) + w or R + w.
__global__ void k_bbox32(Bunch32 b, double P0, double P1, double kh0, double kh1, int pending, WinState *ws) {
  double mn0 = INFINITY, mn1 = INFINITY, mx0 = -INFINITY, mx1 = -INFINITY;
  for (long long n = gtid(); n < b.n; n += (long long)gridDim.x * blockDim.x) {
    int ci, cj;
    unpack(b.cell[n], ci, cj);
    double p0, p1;
    const float r = rgam(P0, P1, b.dpx[n], b.dpy[n], p0, p1);
    const double w0 = half_drift(kh0, p0, r), w1 = half_drift(kh1, p1, r);
    double s0 = b.ox[n], s1 = b.oy[n];
    if (pending) { s0 = dsub(s0, w0); s1 = dsub(s1, w1); }
    const double x0 = cellc(ci, dadd(s0, w0)), x1 = cellc(cj, dadd(s1, w1));
    mn0 = fmin(mn0, x0); mn1 = fmin(mn1, x1); mx0 = fmax(mx0, x0); mx1 = fmax(mx1, x1);
  }
  __shared__ double sb[4][32];
  block_bbox(mn0, mn1, mx0, mx1, ws->bb[ws->cur], sb);
}

// R += kd * v (cells), kd = dt c / h (PartBunch::drift_particles).
__global__ void k_drift32(Bunch32 b, double P0, double P1, double kd0, double kd1) {
  for (long long n = gtid(); n < b.n; n += (long long)gridDim.x * blockDim.x) {
    int ci, cj;
    unpack(b.cell[n], ci, cj);
    double p0, p1;
    const float r = rgam(P0, P1, b.dpx[n], b.dpy[n], p0, p1);
    int nc;
    float o0, o1;
    store_pos(dadd((double)b.ox[n], half_drift(kd0, p0, r)), dadd((double)b.oy[n], half_drift(kd1, p1, r)), ci, cj,
              nc, o0, o1);
    b.cell[n] = nc; b.ox[n] = o0; b.oy[n] = o1;
  }
}

__global__ void k_from64(const double *x, const double *y, const double *px, const double *py, const double *q,
                         long long nn, double org0, double org1, double h0, double h1, double P0, double P1,
                         Bunch32 b) {
  for (long long n = gtid(); n < nn; n += (long long)gridDim.x * blockDim.x) {
    int c;
    float o0, o1;
    store_pos((x[n] - org0) / h0, (y[n] - org1) / h1, 0, 0, c, o0, o1);
    b.cell[n] = c; b.ox[n] = o0; b.oy[n] = o1;
    b.dpx[n] = (float)(px[n] - P0);
    b.dpy[n] = (float)(py[n] - P1);
    b.q[n] = (float)q[n];
  }
}

__global__ void k_to64(Bunch32View v, double *x, double *y, double *px, double *py) {
  for (long long n = gtid(); n < v.b.n; n += (long long)gridDim.x * blockDim.x) {
    double a, c, p0, p1;
    v(n, a, c, p0, p1);
    if (x) x[n] = a;
    if (y) y[n] = c;
    if (px) px[n] = p0;
    if (py) py[n] = p1;
  }
}

__global__ void k_psum2(const double *px, const double *py, long long n, double *part) {
  __shared__ double sh[2][256];
  double a = 0.0, c = 0.0;
  for (long long k = blockIdx.x * 256ll + threadIdx.x; k < n; k += (long long)gridDim.x * 256) {
    a += px[k]; c += py[k];
  }
  sh[0][threadIdx.x] = a; sh[1][threadIdx.x] = c;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) { sh[0][threadIdx.x] += sh[0][threadIdx.x + w]; sh[1][threadIdx.x] += sh[1][threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = sh[0][0]; part[2 * blockIdx.x + 1] = sh[1][0]; }
}

__global__ void k_psum2_final(const double *part, int np, double *out) {
  if (threadIdx.x != 0) return;
  double a = 0.0, c = 0.0;
  for (int k = 0; k < np; ++k) { a += part[2 * k]; c += part[2 * k + 1]; }
  out[0] = a; out[1] = c;
}

template <class S, class D>
__global__ void k_plane_copy(const S *src, int spitch, D *dst, int dpitch, int rows, int cols) {
  const long long k = gtid();
  if (k >= (long long)rows * cols) return;
  const int r = (int)(k / cols), c = (int)(k % cols);
  dst[(size_t)r * dpitch + c] = (D)src[(size_t)r * spitch + c];
}

inline unsigned grid_for(long long n, unsigned cap = 4096) {
  const long long g = (n + 255) / 256;
  return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

// The deposit launch keeps only the warp tiles in dynamic shared memory
// (48-56 KB, above the 48 KB a launch gets without opting in) and adds into
// the window accumulator in global memory: measured on the 4e6-particle TSC
// bunch, a CTA copy of the accumulator in shared memory cost more (zeroing,
// flushing its touched box) than the global adds it saves, and its size kept
// the SM to two CTAs.
template <int ORDER>
size_t dep_smem32() {
  static int set = 0;
  const size_t tiles = (size_t)TileFor<ORDER>::T::kSize * 256 * sizeof(unsigned long long);
  if (!set) {
    cudaFuncSetAttribute(k_push32_dep<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tiles);
    cudaGetLastError();
    set = 1;
  }
  return tiles;
}

// CTAs of the move and deposit launches: three per SM.
int push_grid32() {
  static int g = 0;
  if (!g) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g = 3 * (sms > 0 ? sms : 148);
  }
  return g;
}

template <int ORDER>
void push32_order(const Push32Args &a, cudaStream_t s) {
  k_push32_move<ORDER><<<push_grid32(), 256, 0, s>>>(a);
  k_push32_dep<ORDER><<<push_grid32(), 256, dep_smem32<ORDER>(), s>>>(a);
}

}  // namespace

int launch_push32(const Push32Args &a, int order, cudaStream_t s) {
  if (order == 0) push32_order<0>(a, s);
  else if (order == 1) push32_order<1>(a, s);
  else push32_order<2>(a, s);
  k_post32<<<1, 32, 0, s>>>(a.ws);
  return 0;
}

// The batched FP32 push keeps no window copy in shared memory (0: no member
// "fits"); its deposit launch takes the warp tiles of the largest shape order.
long long push32_batch_smem_limit() {
  static int set = 0;
  if (!set) {
    cudaFuncSetAttribute(k_push32_batch_dep<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(TileFor<0>::T::kSize * 256 * sizeof(unsigned long long)));
    cudaFuncSetAttribute(k_push32_batch_dep<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(TileFor<1>::T::kSize * 256 * sizeof(unsigned long long)));
    cudaFuncSetAttribute(k_push32_batch_dep<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(TileFor<2>::T::kSize * 256 * sizeof(unsigned long long)));
    cudaGetLastError();
    set = 1;
  }
  return 0;
}

void launch_push32_batch(const PushGroup *groups, int ngroups, int m, int grid, const PrepArgs *prep, cudaStream_t s,
            int parts) {
  const int tb = (m + 127) / 128;
  if (parts & 1) k_prep32_batch<<<tb, 128, 0, s>>>(prep, m);
  for (int g = 0; g < ngroups; ++g) {
    const PushGroup &G = groups[g];
    if (G.total <= 0) continue;
    const int ctas = (int)((long long)grid * G.total / (G.all > 0 ? G.all : G.total)) + 1;
    const long long per = (G.total + ctas - 1) / ctas;
    const Push32Args *args = static_cast<const Push32Args *>(G.args);
    push32_batch_smem_limit();
    const size_t tiles = push_tile_bytes(G.order);
    if (G.order == 0) {
      k_push32_batch_move<0><<<ctas, 256, 0, s>>>(args, G.ppre, G.m, per);
      k_push32_batch_dep<0><<<ctas, 256, tiles, s>>>(args, G.ppre, G.m, per);
    } else if (G.order == 1) {
      k_push32_batch_move<1><<<ctas, 256, 0, s>>>(args, G.ppre, G.m, per);
      k_push32_batch_dep<1><<<ctas, 256, tiles, s>>>(args, G.ppre, G.m, per);
    } else {
      k_push32_batch_move<2><<<ctas, 256, 0, s>>>(args, G.ppre, G.m, per);
      k_push32_batch_dep<2><<<ctas, 256, tiles, s>>>(args, G.ppre, G.m, per);
    }
  }
  if (parts & 2) {
    k_post32_batch<<<tb, 128, 0, s>>>(prep, m);
    k_bounds32_batch<<<tb, 128, 0, s>>>(prep, m);
  }
}

void launch_prep32(WinState *ws, int order, cudaStream_t s) {
  (void)order;
  k_prep32<<<1, 32, 0, s>>>(ws, 2);
}

void launch_bounds32(WinState *ws, cudaStream_t s) { k_bounds32<<<1, 32, 0, s>>>(ws); }

void launch_bbox32(const Bunch32 &b, double P0, double P1, double kh0, double kh1, int pending, WinState *ws,
                   cudaStream_t s) {
  k_bbox32_clear<<<1, 32, 0, s>>>(ws);
  k_bbox32<<<grid_for(b.n, 1184), 256, 0, s>>>(b, P0, P1, kh0, kh1, pending, ws);
}

void launch_drift32(const Bunch32 &b, double P0, double P1, double kd0, double kd1, cudaStream_t s) {
  if (b.n > 0) k_drift32<<<grid_for(b.n), 256, 0, s>>>(b, P0, P1, kd0, kd1);
}

void launch_from64(const double *x, const double *y, const double *px, const double *py, const double *q,
                   long long n, double org0, double org1, double h0, double h1, double P0, double P1,
                   const Bunch32 &b, cudaStream_t s) {
  if (n > 0) k_from64<<<grid_for(n), 256, 0, s>>>(x, y, px, py, q, n, org0, org1, h0, h1, P0, P1, b);
}

void launch_to64(const Bunch32 &b, double P0, double P1, double kh0, double kh1, int pending, double org0,
                 double org1, double h0, double h1, double *x, double *y, double *px, double *py,
                 cudaStream_t s) {
  if (b.n > 0)
    k_to64<<<grid_for(b.n), 256, 0, s>>>(Bunch32View{b, P0, P1, kh0, kh1, pending, org0, org1, h0, h1}, x, y, px,
                                         py);
}

// Mean-momentum sums: part holds 2 x 296 doubles, out2 receives the two sums.
void launch_psum(const double *px, const double *py, long long n, double *part, double *out2, cudaStream_t s) {
  k_psum2<<<296, 256, 0, s>>>(px, py, n, part);
  k_psum2_final<<<1, 32, 0, s>>>(part, 296, out2);
}

void launch_d2f(const double *src, int spitch, float *dst, int dpitch, int rows, int cols, cudaStream_t s) {
  k_plane_copy<double, float><<<grid_for((long long)rows * cols, 1u << 30), 256, 0, s>>>(src, spitch, dst, dpitch,
                                                                                        rows, cols);
}

void launch_f2d(const float *src, int spitch, double *dst, int dpitch, int rows, int cols, cudaStream_t s) {
  k_plane_copy<float, double><<<grid_for((long long)rows * cols, 1u << 30), 256, 0, s>>>(src, spitch, dst, dpitch,
                                                                                        rows, cols);
}

}  // namespace csrst
