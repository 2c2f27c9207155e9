// Particle kernels: the fused relativistic push (drift + gather + kick +
// drift + current deposit) and its window bookkeeping, plus stand-alone
// gather / scatter / deposit kernels behind ScatterGatherImpl and the shape
// functions.
//
// One push kernel replaces PartBunch::push_particles (PartBunch.cpp:215-519):
//   R0 = R (minus the trailing -dt/2 drift of the previous sub-step when it is
//        still pending), R1 = R0 + h v(P), gather E, Hz at R1, kick/rotate,
//   R2 = R1 + h v(P'), deposit J(jcomp) for R0 -> R2.
// The bounding box of R1 (which fixes the gather patch origin, exactly as
// getFields does) is produced by the previous push, so each push streams the
// particles once: 32 B in, 32 B out per particle.
//
// The current is accumulated as 64-bit fixed point: each contribution is
// rounded once to a multiple of 1/scale and integer-added, first in a
// shared-memory copy of the window per CTA, then into the global window.
// Integer addition is exact and associative, so the result is bitwise the
// same for any launch shape, CTA count or scheduling order.
#include "accum.cuh"
#include "bbox.cuh"
#include "kernels.cuh"
#include "shapes.cuh"

namespace csrst {

// Positions R1 = R0 + h v(P) of the next push; fills slot `cur` of the window
// state.  pending: the stored R still owes the -dt/2 drift.
__global__ void k_bbox_next(const double *x, const double *y, const double *px, const double *py,
                            long long n, double half, int pending, WinState *ws) {
  double mn0 = INFINITY, mn1 = INFINITY, mx0 = -INFINITY, mx1 = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double p0 = px[i], p1 = py[i];
    const double r = inv_gamma(p0, p1);
    const double w0 = half * p0 * r, w1 = half * p1 * r;
    double a0 = x[i], a1 = y[i];
    if (pending) { a0 = a0 + (-w0); a1 = a1 + (-w1); }
    a0 = a0 + w0; a1 = a1 + w1;
    mn0 = fmin(mn0, a0); mn1 = fmin(mn1, a1); mx0 = fmax(mx0, a0); mx1 = fmax(mx1, a1);
  }
  __shared__ double sb[4][32];
  block_bbox(mn0, mn1, mx0, mx1, ws->bb[ws->cur], sb);
}

__global__ void k_bbox_clear(WinState *ws, int slot) {
  if (threadIdx.x == 0) bbox_reset(ws->bb[slot < 0 ? ws->cur : slot]);
}

// Before a push: derive the gather patches from the particle box of the
// positions the push will gather at (PartBunch::getLocalPDomain and
// getFields), and reset the accumulators the push will fill.
// em: getExtraMarginEdge (x first, x last, y first, y last); cm: getExtraMarginCell.
__device__ __forceinline__ void push_prep_body(WinState *ws, double h0, double h1, int em0, int em2, int cm0) {
  const int c = ws->cur;
  const double mn0 = ord_dbl(ws->bb[c][0]), mn1 = ord_dbl(ws->bb[c][1]);
  const double mx0 = ord_dbl(ws->bb[c][2]), mx1 = ord_dbl(ws->bb[c][3]);
  int lp[4];
  if (mn0 <= mx0) {
    lp[0] = (int)floor((mn0 - ws->mo0) / h0); lp[1] = (int)floor((mx0 - ws->mo0) / h0);
    lp[2] = (int)floor((mn1 - ws->mo1) / h1); lp[3] = (int)floor((mx1 - ws->mo1) / h1);
  } else {  // no particles: PartBunch::getLocalPDomain with Rmin = Rmax = 0
    lp[0] = lp[1] = (int)floor((0.0 - ws->mo0) / h0);
    lp[2] = lp[3] = (int)floor((0.0 - ws->mo1) / h1);
  }
  for (int k = 0; k < 4; ++k) ws->lp[k] = lp[k];
  // Every gather tap lies within [lp - 2, lp + 2] (the cubic edge stencil
  // reaches furthest); the window planes hold one guard cell.  A bunch that
  // no longer fits stops the run instead of reading outside the window.
  if (mn0 <= mx0 && (lp[0] - 2 < -1 || lp[1] + 2 > ws->L0 || lp[2] - 2 < -1 || lp[3] + 2 > ws->L1))
    set_err(ws, kErrWindowFit);
  const double po0 = ws->mo0 + lp[0] * h0, po1 = ws->mo1 + lp[2] * h1;
  ws->hz_o0 = po0 + cm0 * h0; ws->hz_o1 = po1 + cm0 * h1;
  ws->ex_o0 = po0 + em0 * h0; ws->ex_o1 = po1 + em2 * h1;
  ws->ey_o0 = po0 + em2 * h0; ws->ey_o1 = po1 + em0 * h1;
  ws->hz_I = lp[0] + cm0; ws->hz_J = lp[2] + cm0;
  ws->ex_I = lp[0] + em0; ws->ex_J = lp[2] + em2;
  ws->ey_I = lp[0] + em2; ws->ey_J = lp[2] + em0;
  bbox_reset(ws->bb[1 - c]);
  bbox_reset(ws->bball);
}

__global__ void k_push_prep(WinState *ws, double h0, double h1, int em0, int em2, int cm0) {
  if (threadIdx.x == 0) push_prep_body(ws, h0, h1, em0, em2, cm0);
}

// After a push: flip the bbox slot.
__global__ void k_push_post(WinState *ws) {
  if (threadIdx.x == 0) ws->cur = 1 - ws->cur;
}

// Dynamic shared memory: [window accumulator (SMEM only)][per-thread deposit tiles].
// One CTA's share [beg, end) of one push.  All threads of the CTA call it
// together; it ends with a barrier, so a CTA can run it for several members
// in turn.
template <int ORDER, bool SMEM>
__device__ __forceinline__ void push_body(const PushArgs &a, long long beg, long long end, PushShared &sh,
                                          unsigned long long *sacc) {
  int *tb = sh.tb;  // touched box of this CTA (window cells)
  WinState *ws = a.ws;
  if (threadIdx.x == 0) sh.err = *(volatile int *)&ws->err;
  __syncthreads();
  if (sh.err) return;  // the whole CTA leaves together
  const int L0 = ws->L0, L1 = ws->L1;
  const int ncell = L0 * L1;
  using Tile = typename TileFor<ORDER>::T;
  unsigned long long *win = SMEM ? sacc : a.acc;
  unsigned long long *tmem = SMEM ? sacc + ncell : sacc;
  if (SMEM)
    for (int k = threadIdx.x; k < ncell; k += blockDim.x) sacc[k] = 0ull;
  for (int k = threadIdx.x; k < Tile::kSize * (int)blockDim.x; k += blockDim.x) tmem[k] = 0ull;
  if (threadIdx.x == 0) { tb[0] = L0; tb[1] = L1; tb[2] = -1; tb[3] = -1; }
  __syncthreads();
  Tile tile;
  tile.init(tmem, L0, L1);
  const double mo0 = ws->mo0, mo1 = ws->mo1;
  const double h0 = a.h0, h1 = a.h1;
  const double ood0 = 1.0 / h0, ood1 = 1.0 / h1;
  const int wp = a.wpitch;
  // Patch views: relative (0,0) is absolute window index (I, J); the window
  // plane stores absolute (i, j) at (j + 1) * wp + (i + 1).
  const PatchView pex{a.mEx + (ptrdiff_t)(ws->ex_J + 1) * wp + (ws->ex_I + 1), wp};
  const PatchView pey{a.mEy + (ptrdiff_t)(ws->ey_J + 1) * wp + (ws->ey_I + 1), wp};
  const PatchView phx{a.mHx + (ptrdiff_t)(ws->hz_J + 1) * wp + (ws->hz_I + 1), wp};
  const PatchView phy{a.mHy + (ptrdiff_t)(ws->hz_J + 1) * wp + (ws->hz_I + 1), wp};
  const double exo0 = ws->ex_o0, exo1 = ws->ex_o1, eyo0 = ws->ey_o0, eyo1 = ws->ey_o1;
  const double hzo0 = ws->hz_o0, hzo1 = ws->hz_o1;

  double amn0 = INFINITY, amn1 = INFINITY, amx0 = -INFINITY, amx1 = -INFINITY;  // R0 u R2
  double bmn0 = INFINITY, bmn1 = INFINITY, bmx0 = -INFINITY, bmx1 = -INFINITY;  // next R1
  bool overflow = false;
  const double scale = a.acc_scale;
  auto sink = [&](int i, int j, double v) { tile.template add<SMEM>(i, j, __double2ll_rn(v * scale), win, L0, L1); };

  // The CTA owns a contiguous slice of the (cell-ordered) particles.  The
  // rounds are the same for every lane, so that the warp re-bases its
  // deposit tile together.
  const long long rounds = end > beg ? (end - beg + blockDim.x - 1) / blockDim.x : 0;
  for (long long it = 0; it < rounds; ++it) {
    const long long i = beg + it * blockDim.x + threadIdx.x;
    bool ok = i < end;
    double x = 0.0, y = 0.0, p0 = 0.0, p1 = 0.0, q = 0.0, r0x = 0.0, r0y = 0.0, w0 = 0.0, w1 = 0.0;
    if (ok) {
      x = a.x[i]; y = a.y[i]; p0 = a.px[i]; p1 = a.py[i]; q = a.q[i];
      if (!(isfinite(x) && isfinite(y) && isfinite(p0) && isfinite(p1))) {
        set_err(ws, kErrWindowFit);
        ok = false;
      }
    }
    if (ok) {
      double r = inv_gamma(p0, p1);
      w0 = a.half * p0 * r; w1 = a.half * p1 * r;
      if (a.pending) { x = x + (-w0); y = y + (-w1); }          // drift_particles(-dt/2)
      r0x = x; r0y = y;                                          // oldR
      x = x + w0; y = y + w1;                                    // R1
      // gather (FieldPatch::gather x3; Hz = Hzx + Hzy on the fly)
      const double E0 = gather_edge<ORDER>(pex, (x - exo0) * ood0, (y - exo1) * ood1, 0);
      const double E1 = gather_edge<ORDER>(pey, (x - eyo0) * ood0, (y - eyo1) * ood1, 1);
      const double hpp0 = (x - hzo0) * ood0, hpp1 = (y - hzo1) * ood1;
      const double Hf = gather_cell<ORDER>(SumView{phx, phy}, hpp0, hpp1);
      // hard-edge dipole
      const double D0 = x - a.Lb, D1 = y - a.hw;
      const double dist = a.chh * D0 - a.shh * D1;
      const double bext = (dist > 0.0 && dist < a.bwidth) ? a.bz : 0.0;
      const double B = kMu0 * Hf + 0.5 * bext;
      // kick + rotation (PartBunch.cpp:366-383)
      const double k0 = a.fact1 * E0, k1 = a.fact1 * E1;
      double u0 = p0 + k0, u1 = p1 + k1;
      const double aa = a.fact2 * B * inv_gamma(u0, u1);
      const double s0 = u0 + aa * u1, s1 = u1 + aa * (-u0);
      const double tmp = 1.0 + aa * aa;
      u0 = ((1.0 + aa * aa) * s0 + aa * s1) / tmp;
      u1 = ((1.0 + aa * aa) * s1 - aa * s0) / tmp;
      p0 = u0 + k0; p1 = u1 + k1;
      r = inv_gamma(p0, p1);
      w0 = a.half * p0 * r; w1 = a.half * p1 * r;
      x = x + w0; y = y + w1;                                    // R2
      a.x[i] = x; a.y[i] = y; a.px[i] = p0; a.py[i] = p1;
    }
    // current deposit R0 -> R2 in window coordinates, summed in the warp's tile
    tile.template rebase<SMEM>(ok, ok ? (int)floor((r0x - mo0) * ood0) : 0, ok ? (int)floor((r0y - mo1) * ood1) : 0,
                               win, L0, L1);
    if (ok) {
      if (!deposit_particle<ORDER>(a.jcomp, q, r0x, r0y, x, y, mo0, mo1, h0, h1, h0, h1, a.dt, sink))
        overflow = true;
      amn0 = fmin(amn0, fmin(x, r0x)); amn1 = fmin(amn1, fmin(y, r0y));
      amx0 = fmax(amx0, fmax(x, r0x)); amx1 = fmax(amx1, fmax(y, r0y));
      // next push gathers at (R2 - h v) + h v
      const double nx = (x + (-w0)) + w0, ny = (y + (-w1)) + w1;
      bmn0 = fmin(bmn0, nx); bmn1 = fmin(bmn1, ny); bmx0 = fmax(bmx0, nx); bmx1 = fmax(bmx1, ny);
    }
  }
  tile.template flush<SMEM>(win, L0, L1);
  if (overflow) set_err(ws, kErrCrossings);
  block_bbox(amn0, amn1, amx0, amx1, ws->bball, sh.sb);
  block_bbox(bmn0, bmn1, bmx0, bmx1, ws->bb[1 - ws->cur], sh.sb);
  if (SMEM) {
    if (tile.ti1 >= 0) {
      atomicMin(&tb[0], tile.ti0); atomicMin(&tb[1], tile.tj0);
      atomicMax(&tb[2], tile.ti1); atomicMax(&tb[3], tile.tj1);
    }
    __syncthreads();
    const int i0 = tb[0], j0 = tb[1], i1 = tb[2], j1 = tb[3];
    if (i1 >= i0) {
      const int w = i1 - i0 + 1, cnt = w * (j1 - j0 + 1);
      for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        const int i = i0 + k % w, j = j0 + k / w;
        const unsigned long long v = sacc[j * L0 + i];
        if (v) atomicAdd(&a.acc[j * L0 + i], v);
      }
    }
  }
  __syncthreads();
}

// The single-member push: warp tiles in dynamic shared memory, the window
// accumulator in global memory, three CTAs per SM.  The push is bound by the
// latency of dependent FP64 chains; a CTA copy of the accumulator in shared
// memory held the SM to two CTAs and cost more to zero and flush than the
// global adds it saved (4e6-particle TSC bunch, 8192 x 1024 mesh: 0.55 ->
// 0.44 ms per push).  Integer sums: the result does not depend on where
// they are added.
template <int ORDER>
__global__ void __launch_bounds__(256, 3) k_push(PushArgs a) {
  extern __shared__ unsigned long long sacc[];
  __shared__ PushShared sh;
  const long long per = (a.n + gridDim.x - 1) / gridDim.x;
  const long long beg = (long long)blockIdx.x * per;
  const long long end = beg + per < a.n ? beg + per : a.n;
  push_body<ORDER, false>(a, beg, end, sh, sacc);
}

// One push over a batch of members: the members' particles form one index
// range (ppre: first particle of each member, m + 1 entries) that is cut into
// equal contiguous shares, one per CTA; a CTA runs the push of every member
// its share overlaps, with that member's shape order and accumulator.
template <int ORDER>
__global__ void __launch_bounds__(256, 2) k_push_batch(const PushArgs *args, const unsigned char *smem_ok,
                                                       const long long *ppre, int m, long long per) {
  extern __shared__ unsigned long long sacc[];
  __shared__ PushShared sh;
  __shared__ PushArgs sa;
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
    if (smem_ok[mm]) push_body<ORDER, true>(sa, lb, le, sh, sacc);
    else push_body<ORDER, false>(sa, lb, le, sh, sacc);
  }
}

// Per-member bookkeeping of a batched push, one thread per member.
__global__ void k_push_prep_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) push_prep_body(p[k].ws, p[k].h0, p[k].h1, p[k].em0, p[k].em2, p[k].cm0);
}
__global__ void k_push_post_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) p[k].ws->cur = 1 - p[k].ws->cur;
}

// After the last push of a step: the deposit's particle bounds relative to
// the window (PartBunch::getLocalPDomainInclOld -> setGlobalBounds).
__device__ __forceinline__ void global_bounds_body(WinState *ws, double h0, double h1) {
  const double mn0 = ord_dbl(ws->bball[0]), mn1 = ord_dbl(ws->bball[1]);
  const double mx0 = ord_dbl(ws->bball[2]), mx1 = ord_dbl(ws->bball[3]);
  if (!(mn0 <= mx0)) { ws->gb[0] = 0; ws->gb[1] = -1; ws->gb[2] = 0; ws->gb[3] = -1; return; }
  ws->gb[0] = (int)floor((mn0 - ws->mo0) / h0);
  ws->gb[1] = (int)floor((mx0 - ws->mo0) / h0);
  ws->gb[2] = (int)floor((mn1 - ws->mo1) / h1);
  ws->gb[3] = (int)floor((mx1 - ws->mo1) / h1);
}

__global__ void k_global_bounds(WinState *ws, double h0, double h1) {
  if (threadIdx.x == 0) global_bounds_body(ws, h0, h1);
}
__global__ void k_global_bounds_batch(const PrepArgs *p, int m) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) global_bounds_body(p[k].ws, p[k].h0, p[k].h1);
}

// Stand-alone drift (PartBunch::drift_particles, PartBunch.cpp:179-187).
__global__ void k_drift(double *x, double *y, const double *px, const double *py, long long n,
                        double full) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double p0 = px[i], p1 = py[i];
    const double r = inv_gamma(p0, p1);
    x[i] += full * p0 * r;
    y[i] += full * p1 * r;
  }
}

// --- stand-alone ScatterGatherImpl / ShapeFunction kernels --------------------

template <int ORDER>
__global__ void k_gather(int comp, const double *patch, int nx, double o0, double o1, double h0,
                         double h1, const double *x, const double *y, long long n, double *out) {
  const PatchView f{patch, nx};
  const double ood0 = 1.0 / h0, ood1 = 1.0 / h1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double pp0 = (x[i] - o0) * ood0, pp1 = (y[i] - o1) * ood1;
    out[i] = comp < 2 ? gather_edge<ORDER>(f, pp0, pp1, comp) : gather_cell<ORDER>(f, pp0, pp1);
  }
}

// Deposit of stand-alone particle arrays into a dense fixed-point patch at
// absolute index (i0, j0) of a mesh with origin (org0, org1).
template <int ORDER>
__global__ void k_deposit(int comp, const double *ox, const double *oy, const double *x,
                          const double *y, const double *q, long long n, double org0, double org1,
                          double h0, double h1, double dt, int i0, int j0, int ni, int nj,
                          unsigned long long *acc, double scale, int *err) {
  // err[0]: crossing overflow; err[1]: a non-zero contribution fell outside the patch
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    bool dropped = false;
    auto sink = [&](int a, int b, double v) {
      a -= i0; b -= j0;
      const bool in = a >= 0 && b >= 0 && a < ni && b < nj;
      const long long iv = __double2ll_rn(v * scale);
      if (!in && iv != 0) dropped = true;
      warp_add(acc, in ? b * ni + a : -1, iv);
    };
    if (!deposit_particle<ORDER>(comp, q[i], ox[i], oy[i], x[i], y[i], org0, org1, h0, h1, h0, h1, dt, sink))
      atomicExch(&err[0], kErrCrossings);
    if (dropped) atomicExch(&err[1], 1);
  }
}

__global__ void k_fixed_to_double(const unsigned long long *acc, double *out, long long n, double inv) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (double)(long long)acc[i] * inv;
}

// --- host launchers -----------------------------------------------------------

void launch_bbox_next(const double *x, const double *y, const double *px, const double *py,
                      long long n, double half, int pending, WinState *ws, cudaStream_t s) {
  k_bbox_clear<<<1, 32, 0, s>>>(ws, -1);
  const int blocks = n > 0 ? (int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184) : 1;
  k_bbox_next<<<blocks, 256, 0, s>>>(x, y, px, py, n, half, pending, ws);
}

PrepArgs prep_args(WinState *ws, double h0, double h1, int order) {
  PrepArgs p{ws, h0, h1, 0, 0, 0};
  if (order == 0) { p.em0 = -1; p.em2 = 0; p.cm0 = -1; }
  else if (order == 1) { p.em0 = -1; p.em2 = -1; p.cm0 = -1; }
  else { p.em0 = -2; p.em2 = -1; p.cm0 = -2; }
  return p;
}

void launch_push_prep(WinState *ws, double h0, double h1, int order, cudaStream_t s) {
  const PrepArgs p = prep_args(ws, h0, h1, order);
  k_push_prep<<<1, 32, 0, s>>>(ws, h0, h1, p.em0, p.em2, p.cm0);
}

size_t push_tile_bytes(int order) {
  const int k = order == 0 ? TileFor<0>::T::kSize : order == 1 ? TileFor<1>::T::kSize : TileFor<2>::T::kSize;
  return (size_t)k * 256 * sizeof(unsigned long long);
}

long long push_batch_smem_limit() {
  static long long lim = -1;
  if (lim < 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k_push_batch<1>);
    lim = (long long)v - (long long)fa.sharedSizeBytes;
    // keep two CTAs per SM: half the SM's shared memory less the static part
    // and the 1 KB the runtime reserves per CTA
    int per_sm = 0;
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    const long long two = (long long)per_sm / 2 - (long long)fa.sharedSizeBytes - 1024;
    if (two > 0 && two < lim) lim = two;
    if (cudaFuncSetAttribute(k_push_batch<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim) != cudaSuccess ||
        cudaFuncSetAttribute(k_push_batch<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim) != cudaSuccess ||
        cudaFuncSetAttribute(k_push_batch<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim) != cudaSuccess)
      lim = 0;
    cudaGetLastError();
  }
  return lim;
}

void launch_push_batch(const PushGroup *groups, int ngroups, int m, int grid, const PrepArgs *prep, cudaStream_t s,
            int parts) {
  const int tb = (m + 127) / 128;
  if (parts & 1) k_push_prep_batch<<<tb, 128, 0, s>>>(prep, m);
  for (int g = 0; g < ngroups; ++g) {
    const PushGroup &G = groups[g];
    if (G.total <= 0) continue;
    const int ctas = (int)((long long)grid * G.total / (G.all > 0 ? G.all : G.total)) + 1;
    const long long per = (G.total + ctas - 1) / ctas;
    const PushArgs *args = static_cast<const PushArgs *>(G.args);
    if (G.order == 0) k_push_batch<0><<<ctas, 256, G.smem, s>>>(args, G.smem_ok, G.ppre, G.m, per);
    else if (G.order == 1) k_push_batch<1><<<ctas, 256, G.smem, s>>>(args, G.smem_ok, G.ppre, G.m, per);
    else k_push_batch<2><<<ctas, 256, G.smem, s>>>(args, G.smem_ok, G.ppre, G.m, per);
  }
  if (parts & 2) {
    k_push_post_batch<<<tb, 128, 0, s>>>(prep, m);
    k_global_bounds_batch<<<tb, 128, 0, s>>>(prep, m);
  }
}

// Dynamic shared memory of the single-member push: its warp tiles (48-56 KB,
// above the 48 KB a launch gets without opting in).
template <int ORDER>
static size_t push_smem() {
  static int set = 0;
  const size_t tiles = (size_t)TileFor<ORDER>::T::kSize * 256 * sizeof(unsigned long long);
  if (!set) {
    cudaFuncSetAttribute(k_push<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tiles);
    cudaGetLastError();
    set = 1;
  }
  return tiles;
}

void launch_push(const PushArgs &a, int order, int grid, cudaStream_t s) {
  if (order == 0) k_push<0><<<grid, 256, push_smem<0>(), s>>>(a);
  else if (order == 1) k_push<1><<<grid, 256, push_smem<1>(), s>>>(a);
  else k_push<2><<<grid, 256, push_smem<2>(), s>>>(a);
  k_push_post<<<1, 32, 0, s>>>(a.ws);
}

void launch_global_bounds(WinState *ws, double h0, double h1, cudaStream_t s) {
  k_global_bounds<<<1, 32, 0, s>>>(ws, h0, h1);
}

void launch_drift(double *x, double *y, const double *px, const double *py, long long n, double full,
                  cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  k_drift<<<blocks, 256, 0, s>>>(x, y, px, py, n, full);
}

void launch_gather(int order, int comp, const double *patch, int nx, double o0, double o1,
                   double h0, double h1, const double *x, const double *y, long long n, double *out,
                   cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  if (order == 0) k_gather<0><<<blocks, 256, 0, s>>>(comp, patch, nx, o0, o1, h0, h1, x, y, n, out);
  else if (order == 1) k_gather<1><<<blocks, 256, 0, s>>>(comp, patch, nx, o0, o1, h0, h1, x, y, n, out);
  else k_gather<2><<<blocks, 256, 0, s>>>(comp, patch, nx, o0, o1, h0, h1, x, y, n, out);
}

void launch_deposit(int order, int comp, const double *ox, const double *oy, const double *x,
                    const double *y, const double *q, long long n, double org0, double org1,
                    double h0, double h1, double dt, int i0, int j0, int ni, int nj,
                    unsigned long long *acc, double scale, int *err, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  if (order == 0)
    k_deposit<0><<<blocks, 256, 0, s>>>(comp, ox, oy, x, y, q, n, org0, org1, h0, h1, dt, i0, j0, ni, nj, acc, scale, err);
  else if (order == 1)
    k_deposit<1><<<blocks, 256, 0, s>>>(comp, ox, oy, x, y, q, n, org0, org1, h0, h1, dt, i0, j0, ni, nj, acc, scale, err);
  else
    k_deposit<2><<<blocks, 256, 0, s>>>(comp, ox, oy, x, y, q, n, org0, org1, h0, h1, dt, i0, j0, ni, nj, acc, scale, err);
}

void launch_fixed_to_double(const unsigned long long *acc, double *out, long long n, double inv,
                            cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  k_fixed_to_double<<<blocks, 256, 0, s>>>(acc, out, n, inv);
}

}  // namespace csrst
