// Deposit accumulation of the push kernels.
//
// A thread walks the cell-sorted bunch with a stride of one CTA, so the
// particles it deposits one after another mostly start in the same cell, and
// the 32 lanes of a warp work on neighbouring particles of that cell.
// Adding every contribution straight into the CTA's window accumulator would
// make those lanes collide on the same addresses; aggregating them across the
// warp first costs more instructions than the deposit itself.
//
// Instead each thread owns a small tile of shared memory around a base cell
// shared by its warp and adds its contributions there with plain loads and
// stores: tile entry k of thread t sits at k * blockDim + t, so the lanes of a
// warp always use different banks and never contend.  When the warp moves on
// to particles that start in another cell, the warp sums each tile entry over
// its lanes and one lane adds it to the window accumulator.  Contributions
// that fall outside the tile (large moves) go to the window accumulator
// directly.  All sums are 64-bit integers, so the result does not depend on
// the order of the additions.
#pragma once

#include "common.cuh"

namespace csrst {

// TW x TH tile covering window cells [bi - OX, bi - OX + TW) x [bj - OY, bj - OY + TH)
// around a base cell that all 32 lanes of the warp share, so that a re-base
// is one collective step: every entry is summed over the warp (three exact
// 22-bit chunk reductions form the 64-bit two's-complement sum) and added to
// the destination by one lane.  rebase() and flush() must be called by all
// lanes of the warp together; add() may be called by any subset.
template <int TW, int TH, int OX, int OY>
struct TileAcc {
  static constexpr int kSize = TW * TH;
  unsigned long long *tile;  // shared memory, kSize * stride entries, zeroed
  int stride;                // threads per CTA
  int bi, bj;                // warp-uniform base cell (window cells)
  bool live;                 // warp-uniform: the tile may hold non-zero entries
  int ti0, tj0, ti1, tj1;    // window cells this lane added to (touched box)

  __device__ __forceinline__ void init(unsigned long long *t, int L0, int L1) {
    tile = t + threadIdx.x;
    stride = blockDim.x;
    bi = bj = -(1 << 28);
    live = false;
    ti0 = L0; tj0 = L1; ti1 = -1; tj1 = -1;
  }

  template <bool SHARED>
  __device__ __forceinline__ void touch(int i, int j) {
    if (SHARED) { ti0 = min(ti0, i); tj0 = min(tj0, j); ti1 = max(ti1, i); tj1 = max(tj1, j); }
  }

  // Adds everything held to dst (window cells, L0 x L1; global or shared).
  template <bool SHARED>
  __device__ __forceinline__ void flush(unsigned long long *dst, int L0, int L1) {
    if (!live) return;
    const bool lead = (threadIdx.x & 31) == 0;
#pragma unroll 4
    for (int k = 0; k < kSize; ++k) {
      const unsigned long long v = tile[k * stride];
      if (!__any_sync(0xffffffffu, v != 0ull)) continue;  // the warp never added to this entry
      tile[k * stride] = 0ull;
      const unsigned c0 = __reduce_add_sync(0xffffffffu, (unsigned)(v & 0x3FFFFFull));
      const unsigned c1 = __reduce_add_sync(0xffffffffu, (unsigned)((v >> 22) & 0x3FFFFFull));
      const unsigned c2 = __reduce_add_sync(0xffffffffu, (unsigned)(v >> 44));
      const unsigned long long sum =
          (unsigned long long)c0 + ((unsigned long long)c1 << 22) + ((unsigned long long)c2 << 44);
      const int i = bi - OX + k % TW, j = bj - OY + k / TW;
      if (lead && sum && i >= 0 && j >= 0 && i < L0 && j < L1) {
        atomicAdd(&dst[j * L0 + i], sum);
        touch<SHARED>(i, j);
      }
    }
    live = false;
  }

  // Re-bases the warp's tile on the start cell of the first lane that has a
  // particle (has) in this round.
  template <bool SHARED>
  __device__ __forceinline__ void rebase(bool has, int ci, int cj, unsigned long long *dst, int L0, int L1) {
    const unsigned m = __ballot_sync(0xffffffffu, has);
    if (!m) return;
    const int src = __ffs(m) - 1;
    const int nbi = __shfl_sync(0xffffffffu, ci, src), nbj = __shfl_sync(0xffffffffu, cj, src);
    if (nbi != bi || nbj != bj) {
      flush<SHARED>(dst, L0, L1);
      bi = nbi; bj = nbj;
    }
    live = true;
  }

  template <bool SHARED>
  __device__ __forceinline__ void add(int i, int j, long long v, unsigned long long *dst, int L0, int L1) {
    const int a = i - (bi - OX), b = j - (bj - OY);
    if ((unsigned)a < (unsigned)TW && (unsigned)b < (unsigned)TH) {
      tile[(b * TW + a) * stride] += (unsigned long long)v;
    } else if (i >= 0 && j >= 0 && i < L0 && j < L1) {
      atomicAdd(&dst[j * L0 + i], (unsigned long long)v);
      touch<SHARED>(i, j);
    }
  }
};

// Tile shape per shape order: relative to the start cell of the particle it
// holds every contribution of a particle that moves less than half a cell
// along x and a little along y (CFL <= 0.5), for both current components:
// i in [-1, 2], j in [-1, 2] for CIC and TSC, i in [-1, 3] for the cubic
// shape; one more column on each side lets the lanes of a warp start one
// cell before or after the warp's base cell.
template <int ORDER>
struct TileFor;
template <>
struct TileFor<0> { using T = TileAcc<6, 4, 2, 1>; };
template <>
struct TileFor<1> { using T = TileAcc<6, 4, 2, 1>; };
template <>
struct TileFor<2> { using T = TileAcc<7, 4, 2, 1>; };

}  // namespace csrst
