// FP32 mode particle kernels: the fused push of particles.cu
// (PartBunch::push_particles, PartBunch.cpp:215-519) on a bunch stored as
// FP32 offsets from FP64 cell origins and FP32 momentum deviations from an
// FP64 reference momentum, in FP32 arithmetic.
//
// Precision split:
//   - FP32: 1/gamma (the reference's float Q_rsqrt of 1 + |P|^2 formed from
//     the FP32 deviation, bunch32.cuh), the drifts, the positions during the
//     push (offsets from the particle's old cell), the field gather (anchored
//     at the particle's own window cell, so its coordinates keep FP32's full
//     resolution), the kick and rotation, and the current's path integral
//     (flux32.cuh);
//   - FP64: the hard-edge dipole test on the absolute position (the bend
//     frame), and the 1D charge weights of each move's end points from which
//     the fixed-point charge and, by exact integer continuity, the x current
//     are formed (flux32.cuh); the deposited current then satisfies the
//     discrete continuity equation exactly for the charge each particle
//     carries.
// This file is built with FMA contraction on; the bunch arithmetic shared
// with other kernels (bunch32.cuh) rounds every operation explicitly.
#include <climits>

#include "accum.cuh"
#include "bbox.cuh"
#include "bunch32.cuh"
#include "flux32.cuh"
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
__device__ __forceinline__ double cellc(int c, float t) { return (double)(c + (int)floorf(t)) + 0.5; }

// Store a position t (cells from cell (ci, cj)) as cell + offset in [0, 1).
__device__ __forceinline__ void store32(float t0, float t1, int ci, int cj, int &cell, float &o0, float &o1) {
  float f0 = floorf(t0), f1 = floorf(t1);
  float a0 = fsub(t0, f0), a1 = fsub(t1, f1);
  if (a0 >= 1.0f) { a0 = 0.0f; f0 += 1.0f; }  // a negative t rounded up to the next cell
  if (a1 >= 1.0f) { a1 = 0.0f; f1 += 1.0f; }
  cell = ((ci + (int)f0) & 0xffff) | ((cj + (int)f1) << 16);
  o0 = a0; o1 = a1;
}

// One particle's move: start A = stored position (minus the pending half
// drift), gather at R1, kick + rotation, drift to R2, R2 and the new momentum
// deviation stored.  On return, when ok: A in cells from the old cell
// (ci, cj), the stored end point as new cell (ni, nj) + offset (o0, o1).
// Particles that fail the window-fit checks set the member's error and come
// back with ok false, unchanged.
struct Move32 {
  bool ok;
  int ci, cj, ni, nj;
  float a0, a1, o0, o1, q;
};

// The stored state of particle n, read one round ahead of its move.
struct In32 {
  int cell;
  float s0, s1, d0, d1, q;
};
__device__ __forceinline__ In32 load32(const Bunch32 &b, long long n) {
  return In32{__ldcs(b.cell + n), __ldcs(b.ox + n), __ldcs(b.oy + n), __ldcs(b.dpx + n), __ldcs(b.dpy + n),
              __ldg(b.q + n)};
}

template <int ORDER_OF_PUSH>
__device__ __forceinline__ void move32(const Push32Args &a, long long n, const In32 &in, int L0, int L1, int WP0,
                                       int WP1, Move32 &m) {
  WinState *ws = a.ws;
  const int wp = a.wpitch;
  const Ref32 &R = a.R;
  int ci, cj;
  unpack(in.cell, ci, cj);
  const float s0 = in.s0, s1 = in.s1;
  float d0 = in.d0, d1 = in.d1;
  m.q = in.q;
  m.ci = ci; m.cj = cj; m.ni = ci; m.nj = cj;
  m.a0 = s0; m.a1 = s1; m.o0 = s0; m.o1 = s1;
  m.ok = isfinite(d0) && isfinite(d1) && s0 >= 0.0f && s0 < 1.0f && s1 >= 0.0f && s1 < 1.0f;
  if (!m.ok) { set_err(ws, kErrWindowFit); return; }
  // R0 and R1: with the trailing -dt/2 drift pending, the particle sits at
  // s - w and the push's first half drift brings it back to s
  float x0 = s0, x1 = s1;
  {
    const float r = rgam32(R, d0, d1);
    const float w0 = drift32(R.kh0, R.P0, d0, r), w1 = drift32(R.kh1, R.P1, d1, r);
    if (a.pending) { m.a0 = fsub(s0, w0); m.a1 = fsub(s1, w1); }
    else { x0 = fadd(s0, w0); x1 = fadd(s1, w1); }
  }
  const int wi = ci - WP0, wj = cj - WP1;
  // gather (FieldPatch::gather x3) anchored at the window cell of R1
  const float c0 = floorf(x0), c1 = floorf(x1);
  const int ai = wi + (int)c0, aj = wj + (int)c1;
  if (ai - 2 < -1 || ai + 2 > L0 || aj - 2 < -1 || aj + 2 > L1) {  // stencil outside the window planes
    set_err(ws, kErrWindowFit);
    m.ok = false;
    return;
  }
  const float g0 = x0 - c0, g1 = x1 - c1;
  const size_t o = (size_t)(aj + 1) * wp + (ai + 1);
  const View32 vex{a.mEx + o, wp}, vey{a.mEy + o, wp}, vhx{a.mHx + o, wp}, vhy{a.mHy + o, wp};
  const float E0 = gather_edge<ORDER_OF_PUSH>(vex, g0, g1, 0);
  const float E1 = gather_edge<ORDER_OF_PUSH>(vey, g0, g1, 1);
  const float Hf = gather_cell<ORDER_OF_PUSH>(SumView32{vhx, vhy}, g0, g1);
  // hard-edge dipole at the absolute position of R1 (bend frame, FP64)
  const double X = a.org0 + ((double)ci + (double)x0) * a.h0, Y = a.org1 + ((double)cj + (double)x1) * a.h1;
  const double dist = a.chh * (X - a.Lb) - a.shh * (Y - a.hw);
  const float bext = (dist > 0.0 && dist < a.bwidth) ? (float)a.bz : 0.0f;
  const float B = (float)kMu0 * Hf + 0.5f * bext;
  // kick + rotation (PartBunch.cpp:366-383) on u - P
  const float k0 = a.f1 * E0, k1 = a.f1 * E1;
  const float du0 = d0 + k0, du1 = d1 + k1;
  const float ru = rgam32(R, du0, du1);
  const float aa = a.f2 * B * ru;
  const float sv0 = du0 + aa * (R.P1 + du1), sv1 = du1 - aa * (R.P0 + du0);  // s - P
  const float cf = aa / (1.0f + aa * aa);
  d0 = (sv0 + cf * (R.P1 + sv1)) + k0;
  d1 = (sv1 - cf * (R.P0 + sv0)) + k1;
  a.b.dpx[n] = d0; a.b.dpy[n] = d1;
  // second half drift to R2, stored as cell + offset
  const float r = rgam32(R, d0, d1);
  int nc;
  store32(fadd(x0, drift32(R.kh0, R.P0, d0, r)), fadd(x1, drift32(R.kh1, R.P1, d1, r)), ci, cj, nc, m.o0, m.o1);
  a.b.cell[n] = nc; a.b.ox[n] = m.o0; a.b.oy[n] = m.o1;
  unpack(nc, m.ni, m.nj);
  if (a.old_cell) { a.old_cell[n] = (ci & 0xffff) | (cj << 16); a.old_o0[n] = m.a0; a.old_o1[n] = m.a1; }
}

// Boxes of one moved particle: R0 u R2 (the deposit bounds) and the next
// push's gather position, the stored R2, as static-mesh cell indices; they
// are merged as cell + 0.5 (only the cells are used).
struct Boxes32 {
  int amn0 = INT_MAX, amn1 = INT_MAX, amx0 = INT_MIN, amx1 = INT_MIN;  // R0 u R2
  int bmn0 = INT_MAX, bmn1 = INT_MAX, bmx0 = INT_MIN, bmx1 = INT_MIN;  // next R1
  __device__ __forceinline__ void add(const Move32 &m) {
    const int r0 = m.ci + (int)floorf(m.a0), r1 = m.cj + (int)floorf(m.a1);
    amn0 = min(amn0, min(r0, m.ni)); amn1 = min(amn1, min(r1, m.nj));
    amx0 = max(amx0, max(r0, m.ni)); amx1 = max(amx1, max(r1, m.nj));
    bmn0 = min(bmn0, m.ni); bmn1 = min(bmn1, m.nj); bmx0 = max(bmx0, m.ni); bmx1 = max(bmx1, m.nj);
  }
  __device__ __forceinline__ static double c(int v, bool lo) {
    return lo ? (v == INT_MAX ? INFINITY : v + 0.5) : (v == INT_MIN ? -INFINITY : v + 0.5);
  }
  __device__ __forceinline__ void store(WinState *ws, PushShared &sh) {
    block_bbox(c(amn0, true), c(amn1, true), c(amx0, false), c(amx1, false), ws->bball, sh.sb);
    block_bbox(c(bmn0, true), c(bmn1, true), c(bmx0, false), c(bmx1, false), ws->bb[1 - ws->cur], sh.sb);
  }
};

// The member's sticky error at entry, read by one thread for the CTA; a CTA
// that sees one leaves as a whole.
__device__ __forceinline__ bool entry_error(WinState *ws, PushShared &sh) {
  if (threadIdx.x == 0) sh.err = *(volatile int *)&ws->err;
  __syncthreads();
  return sh.err != 0;
}

// The fused push of one CTA's share [beg, end) of one member: every lane
// moves its particle, then the warp deposits the moves' flux (flux32.cuh)
// into per-lane shared-memory tiles around a base cell the warp shares,
// which drain into the member's window accumulator in global memory.  Called
// by all threads of the CTA; ends with a barrier, so a CTA may run it for
// several members in turn.
template <int ORDER, int COMP>
__device__ __forceinline__ void push32_range(const Push32Args &a, long long beg, long long end, PushShared &sh,
                                             unsigned long long *sm) {
  if (entry_error(a.ws, sh)) return;  // the whole CTA leaves together
  WinState *ws = a.ws;
  const int L0 = ws->L0, L1 = ws->L1, WP0 = ws->P0, WP1 = ws->P1;
  using Tile = typename TileFor<ORDER>::T;
  for (int k = threadIdx.x; k < Tile::kSize * (int)blockDim.x; k += blockDim.x) sm[k] = 0ull;
  __syncthreads();
  Tile tile;
  tile.init(sm, L0, L1);
  Boxes32 box;
  bool overflow = false;
  const long long rounds = end > beg ? (end - beg + blockDim.x - 1) / blockDim.x : 0;
  // each lane's next particle is read while the current one moves
  In32 next{};
  if (beg + threadIdx.x < end) next = load32(a.b, beg + threadIdx.x);
  for (long long it = 0; it < rounds; ++it) {  // the same rounds for every lane of the warp
    const long long n = beg + it * blockDim.x + threadIdx.x;
    const In32 cur = next;
    if (n + blockDim.x < end) next = load32(a.b, n + blockDim.x);
    Move32 m;
    m.ok = false;
    m.ci = WP0; m.cj = WP1;
    if (n < end) {
      move32<ORDER>(a, n, cur, L0, L1, WP0, WP1, m);
      if (m.ok) box.add(m);
    }
    const int wi = m.ci - WP0, wj = m.cj - WP1;
    tile.template rebase<false>(m.ok, wi, wj, a.acc, L0, L1);
    // the compact form when every particle of the warp keeps its y base index
    // and advances by at most one x base index
    const int dx = m.ni - m.ci + base_index<ORDER>(m.o0) - base_index<ORDER>(m.a0);
    const bool fast = !m.ok || ((unsigned)dx <= 1u && m.nj - m.cj + base_index<ORDER>(m.o1) == base_index<ORDER>(m.a1));
    const bool all_fast = __all_sync(0xffffffffu, fast);
    if (m.ok) {
      const double K = (double)m.q * a.acc_scale;
      auto sink = [&](int i, int j, long long v) { tile.template add<false>(wi + i, wj + j, v, a.acc, L0, L1); };
      const bool ok = all_fast
          ? flux_particle<ORDER, COMP, true>(m.a0, m.a1, m.ni - m.ci, m.nj - m.cj, m.o0, m.o1, K, __double2ll_rn(K), sink)
          : flux_particle<ORDER, COMP, false>(m.a0, m.a1, m.ni - m.ci, m.nj - m.cj, m.o0, m.o1, K, __double2ll_rn(K), sink);
      if (!ok) overflow = true;
    }
  }
  tile.template flush<false>(a.acc, L0, L1);
  if (overflow) set_err(ws, kErrCrossings);
  box.store(ws, sh);
  __syncthreads();
}

// CTAs per SM of the push launches: three for CIC and TSC, two for the
// cubic shape, whose 5 x 5 stencil box needs more registers.
template <int ORDER>
struct Push32Occ { static constexpr int kCtas = ORDER == 2 ? 2 : 3; };

template <int ORDER, int COMP>
__global__ void __launch_bounds__(256, Push32Occ<ORDER>::kCtas) k_push32(Push32Args a) {
  extern __shared__ unsigned long long sacc[];
  __shared__ PushShared sh;
  const long long per = (a.b.n + gridDim.x - 1) / gridDim.x;
  const long long beg = (long long)blockIdx.x * per;
  push32_range<ORDER, COMP>(a, beg, beg + per < a.b.n ? beg + per : a.b.n, sh, sacc);
}

// One push over a batch of FP32-mode members: the members' particles form one
// index range (ppre: first particle of each member, m + 1 entries) cut into
// equal contiguous shares, one per CTA; a CTA runs the push of every member
// its share overlaps.
template <int ORDER, int COMP>
__global__ void __launch_bounds__(256, Push32Occ<ORDER>::kCtas) k_push32_batch(const Push32Args *args, const long long *ppre, int m,
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
    push32_range<ORDER, COMP>(sa, lb, le, sh, sacc);
  }
}

// Stand-alone flux of n moves (csrst_flux32) into dense patches, one thread
// per move, with 64-bit atomics; err[0]: crossing overflow, err[1]: a
// non-zero contribution fell outside the patch.
template <int ORDER, int COMP>
__global__ void k_flux32(const int *cell0, const float *a0, const float *a1, const int *cell1, const float *b0,
                         const float *b1, const float *q, long long n, double scale, int i0, int j0, int ni, int nj,
                         unsigned long long *F, unsigned long long *drho, int *err) {
  using SH = Flux32Shape<ORDER>;
  for (long long k = gtid(); k < n; k += (long long)gridDim.x * blockDim.x) {
    int ci, cj, ni_, nj_;
    unpack(cell0[k], ci, cj);
    unpack(cell1[k], ni_, nj_);
    const double K = (double)q[k] * scale;
    const long long Ki = __double2ll_rn(K);
    bool dropped = false;
    auto put = [&](unsigned long long *dst, int i, int j, long long v) {
      i += ci - i0; j += cj - j0;
      if (i < 0 || j < 0 || i >= ni || j >= nj) { if (v) dropped = true; return; }
      atomicAdd(&dst[(size_t)j * ni + i], (unsigned long long)v);
    };
    auto sink = [&](int i, int j, long long v) { put(F, i, j, v); };
    if (!flux_particle<ORDER, COMP, false>(a0[k], a1[k], ni_ - ci, nj_ - cj, b0[k], b1[k], K, Ki, sink)) {
      atomicExch(&err[0], kErrCrossings);
      continue;
    }
    if (drho) {  // the charge the flux conserves: rho(end) - rho(start), rows first
      for (int e = 0; e < 2; ++e) {
        double wx[SH::S], wy[SH::S];
        long long R[SH::S], Q[SH::S];
        const int I = (e ? ni_ - ci : 0) + charge_weights<ORDER>(e ? b0[k] : a0[k], wx);
        const int J = (e ? nj_ - cj : 0) + charge_weights<ORDER>(e ? b1[k] : a1[k], wy);
        quantise<ORDER>(wy, K, Ki, R);
        for (int r = 0; r < SH::S; ++r) {
          quantise<ORDER>(wx, (double)R[r], R[r], Q);
          for (int c = 0; c < SH::S; ++c) put(drho, I + SH::OFF + c, J + SH::OFF + r, e ? Q[c] : -Q[c]);
        }
      }
    }
    if (dropped) atomicExch(&err[1], 1);
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


__global__ void k_prep32_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) prep32_body(p[k].ws, 2);
}
__global__ void k_after32_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) {
    p[k].ws->cur = 1 - p[k].ws->cur;
    bounds32_body(p[k].ws);
  }
}

// After a push: the box sets swap (the push filled the other one), the
// deposit bounds follow from the push's boxes, and, when the caller knows
// the next push reads the same particles and window (prep_next), its gather
// patch is set up here too, which saves that push its own set-up launch.
__global__ void k_after32(WinState *ws, int prep_next) {
  if (threadIdx.x != 0) return;
  ws->cur = 1 - ws->cur;
  bounds32_body(ws);
  if (prep_next) prep32_body(ws, 2);
}

__global__ void k_bbox32_clear(WinState *ws) {
  if (threadIdx.x == 0) bbox_reset(ws->bb[ws->cur]);
}

// Box of the next push's gather positions R1: the stored position when the
// trailing -dt/2 drift is pending, else stored + w.
__global__ void k_bbox32(Bunch32 b, Ref32 R, int pending, WinState *ws) {
  double mn0 = INFINITY, mn1 = INFINITY, mx0 = -INFINITY, mx1 = -INFINITY;
  for (long long n = gtid(); n < b.n; n += (long long)gridDim.x * blockDim.x) {
    int ci, cj;
    unpack(b.cell[n], ci, cj);
    float x0 = b.ox[n], x1 = b.oy[n];
    if (!pending) {
      const float d0 = b.dpx[n], d1 = b.dpy[n], r = rgam32(R, d0, d1);
      x0 = fadd(x0, drift32(R.kh0, R.P0, d0, r));
      x1 = fadd(x1, drift32(R.kh1, R.P1, d1, r));
    }
    const double c0 = cellc(ci, x0), c1 = cellc(cj, x1);
    mn0 = fmin(mn0, c0); mn1 = fmin(mn1, c1); mx0 = fmax(mx0, c0); mx1 = fmax(mx1, c1);
  }
  __shared__ double sb[4][32];
  block_bbox(mn0, mn1, mx0, mx1, ws->bb[ws->cur], sb);
}

// R += kd * v (cells), kd = dt c / h (PartBunch::drift_particles).
__global__ void k_drift32(Bunch32 b, Ref32 R, float kd0, float kd1) {
  for (long long n = gtid(); n < b.n; n += (long long)gridDim.x * blockDim.x) {
    int ci, cj;
    unpack(b.cell[n], ci, cj);
    const float d0 = b.dpx[n], d1 = b.dpy[n], r = rgam32(R, d0, d1);
    int nc;
    float o0, o1;
    store32(fadd(b.ox[n], drift32(kd0, R.P0, d0, r)), fadd(b.oy[n], drift32(kd1, R.P1, d1, r)), ci, cj, nc, o0, o1);
    b.cell[n] = nc; b.ox[n] = o0; b.oy[n] = o1;
  }
}

// FP64 bunch -> FP32 form: cell of (x - origin) / h and the offset in it.
__global__ void k_from64(const double *x, const double *y, const double *px, const double *py, const double *q,
                         long long nn, double org0, double org1, double h0, double h1, double P0, double P1,
                         Bunch32 b) {
  for (long long n = gtid(); n < nn; n += (long long)gridDim.x * blockDim.x) {
    const double t0 = (x[n] - org0) / h0, t1 = (y[n] - org1) / h1;
    double f0 = floor(t0), f1 = floor(t1);
    float a0 = (float)(t0 - f0), a1 = (float)(t1 - f1);
    if (a0 >= 1.0f) { a0 = 0.0f; f0 += 1.0; }  // rounded up to the next cell
    if (a1 >= 1.0f) { a1 = 0.0f; f1 += 1.0; }
    b.cell[n] = ((int)f0 & 0xffff) | ((int)f1 << 16);
    b.ox[n] = a0; b.oy[n] = a1;
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

// The push keeps only the warp tiles in dynamic shared memory (48-56 KB,
// above the 48 KB a launch gets without opting in) and adds into the window
// accumulator in global memory, so that three CTAs fit on an SM.
template <int ORDER, int COMP>
size_t push_smem32() {
  static int set = 0;
  const size_t tiles = (size_t)TileFor<ORDER>::T::kSize * 256 * sizeof(unsigned long long);
  if (!set) {
    cudaFuncSetAttribute(k_push32<ORDER, COMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tiles);
    cudaFuncSetAttribute(k_push32_batch<ORDER, COMP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tiles);
    cudaGetLastError();
    set = 1;
  }
  return tiles;
}

// CTAs of a push launch: three per SM.
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
  const int g = push_grid32() / 3 * Push32Occ<ORDER>::kCtas;
  if (a.jcomp == 0) k_push32<ORDER, 0><<<g, 256, push_smem32<ORDER, 0>(), s>>>(a);
  else k_push32<ORDER, 1><<<g, 256, push_smem32<ORDER, 1>(), s>>>(a);
}

template <int ORDER>
void push32_batch_order(const Push32Args *args, const long long *ppre, int m, int ctas, long long per, int jcomp,
                        cudaStream_t s) {
  if (jcomp == 0) k_push32_batch<ORDER, 0><<<ctas, 256, push_smem32<ORDER, 0>(), s>>>(args, ppre, m, per);
  else k_push32_batch<ORDER, 1><<<ctas, 256, push_smem32<ORDER, 1>(), s>>>(args, ppre, m, per);
}

template <int ORDER>
void flux32_order(int comp, const int *cell0, const float *a0, const float *a1, const int *cell1, const float *b0,
                  const float *b1, const float *q, long long n, double scale, int i0, int j0, int ni, int nj,
                  unsigned long long *F, unsigned long long *drho, int *err, cudaStream_t s) {
  const unsigned g = grid_for(n);
  if (comp == 0)
    k_flux32<ORDER, 0><<<g, 256, 0, s>>>(cell0, a0, a1, cell1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, err);
  else
    k_flux32<ORDER, 1><<<g, 256, 0, s>>>(cell0, a0, a1, cell1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, err);
}

}  // namespace

int launch_push32(const Push32Args &a, int order, cudaStream_t s) {
  if (order == 0) push32_order<0>(a, s);
  else if (order == 1) push32_order<1>(a, s);
  else push32_order<2>(a, s);
  return 0;
}

// The batched FP32 push keeps no window copy in shared memory (0: no member
// "fits"); its launches take the warp tiles of their shape order.
long long push32_batch_smem_limit() { return 0; }

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
    const int jcomp = G.jcomp;
    if (G.order == 0) push32_batch_order<0>(args, G.ppre, G.m, ctas, per, jcomp, s);
    else if (G.order == 1) push32_batch_order<1>(args, G.ppre, G.m, ctas, per, jcomp, s);
    else push32_batch_order<2>(args, G.ppre, G.m, ctas, per, jcomp, s);
  }
  if (parts & 2) k_after32_batch<<<tb, 128, 0, s>>>(prep, m);
}

void launch_flux32(int order, int comp, const int *cell0, const float *a0, const float *a1, const int *cell1,
                   const float *b0, const float *b1, const float *q, long long n, double scale, int i0, int j0,
                   int ni, int nj, unsigned long long *F, unsigned long long *drho, int *err, cudaStream_t s) {
  if (n <= 0) return;
  if (order == 0) flux32_order<0>(comp, cell0, a0, a1, cell1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, err, s);
  else if (order == 1) flux32_order<1>(comp, cell0, a0, a1, cell1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, err, s);
  else flux32_order<2>(comp, cell0, a0, a1, cell1, b0, b1, q, n, scale, i0, j0, ni, nj, F, drho, err, s);
}

void launch_prep32(WinState *ws, int order, cudaStream_t s) {
  (void)order;
  k_prep32<<<1, 32, 0, s>>>(ws, 2);
}

void launch_after32(WinState *ws, int prep_next, cudaStream_t s) { k_after32<<<1, 32, 0, s>>>(ws, prep_next); }

void launch_bbox32(const Bunch32 &b, const Ref32 &R, int pending, WinState *ws, cudaStream_t s) {
  k_bbox32_clear<<<1, 32, 0, s>>>(ws);
  k_bbox32<<<grid_for(b.n, 1184), 256, 0, s>>>(b, R, pending, ws);
}

void launch_drift32(const Bunch32 &b, const Ref32 &R, float kd0, float kd1, cudaStream_t s) {
  if (b.n > 0) k_drift32<<<grid_for(b.n), 256, 0, s>>>(b, R, kd0, kd1);
}

void launch_from64(const double *x, const double *y, const double *px, const double *py, const double *q,
                   long long n, double org0, double org1, double h0, double h1, double P0, double P1,
                   const Bunch32 &b, cudaStream_t s) {
  if (n > 0) k_from64<<<grid_for(n), 256, 0, s>>>(x, y, px, py, q, n, org0, org1, h0, h1, P0, P1, b);
}

void launch_to64(const Bunch32 &b, const Ref32 &R, double P0, double P1, int pending, double org0, double org1,
                 double h0, double h1, double *x, double *y, double *px, double *py, cudaStream_t s) {
  if (b.n > 0)
    k_to64<<<grid_for(b.n), 256, 0, s>>>(Bunch32View{b, R, P0, P1, pending, org0, org1, h0, h1}, x, y, px, py);
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
