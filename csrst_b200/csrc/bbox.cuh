// Bounding boxes of particle positions reduced over a CTA and merged into
// device-wide boxes held as ordered-integer doubles (see dbl_ord).
#pragma once

#include "common.cuh"

namespace csrst {

__device__ __forceinline__ void warp_bbox(double &mn0, double &mn1, double &mx0, double &mx1) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn0 = fmin(mn0, __shfl_xor_sync(0xffffffffu, mn0, o));
    mn1 = fmin(mn1, __shfl_xor_sync(0xffffffffu, mn1, o));
    mx0 = fmax(mx0, __shfl_xor_sync(0xffffffffu, mx0, o));
    mx1 = fmax(mx1, __shfl_xor_sync(0xffffffffu, mx1, o));
  }
}

// Reduce a per-thread box over the CTA and merge it into dst[4] with atomics;
// sb is shared scratch of 4 x 32 doubles.
__device__ __forceinline__ void block_bbox(double mn0, double mn1, double mx0, double mx1, long long *dst,
                                           double (*sb)[32]) {
  warp_bbox(mn0, mn1, mx0, mx1);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) { sb[0][w] = mn0; sb[1][w] = mn1; sb[2][w] = mx0; sb[3][w] = mx1; }
  __syncthreads();
  if (w == 0) {
    mn0 = lane < nw ? sb[0][lane] : INFINITY;
    mn1 = lane < nw ? sb[1][lane] : INFINITY;
    mx0 = lane < nw ? sb[2][lane] : -INFINITY;
    mx1 = lane < nw ? sb[3][lane] : -INFINITY;
    warp_bbox(mn0, mn1, mx0, mx1);
    if (lane == 0 && mn0 <= mx0) {
      atomicMin(&dst[0], dbl_ord(mn0));
      atomicMin(&dst[1], dbl_ord(mn1));
      atomicMax(&dst[2], dbl_ord(mx0));
      atomicMax(&dst[3], dbl_ord(mx1));
    }
  }
  __syncthreads();
}

// Shared scratch of one push CTA, declared once per kernel so that a kernel
// that inlines several push variants does not hold one copy per variant.
struct PushShared {
  double sb[4][32];  // block_bbox
  int tb[4];         // touched box of the CTA (window cells)
  int err;           // the member's sticky error at entry
};

__device__ __forceinline__ void bbox_reset(long long *b) {
  b[0] = dbl_ord(INFINITY); b[1] = dbl_ord(INFINITY);
  b[2] = dbl_ord(-INFINITY); b[3] = dbl_ord(-INFINITY);
}

}  // namespace csrst
