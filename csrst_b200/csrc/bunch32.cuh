// FP32-mode bunch arithmetic shared by the particle kernels and the
// diagnostics: every operation on positions and momenta is explicitly
// rounded, so that the same inputs give the same bits in every kernel,
// whatever contraction the translation unit is compiled with.
#pragma once

#include "kernels.cuh"

namespace csrst {

__device__ __forceinline__ void unpack(int c, int &i, int &j) {
  i = c & 0xffff;
  j = (int)((unsigned)c >> 16);
}

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// 1/gamma as the FP64 path computes it, from the full momentum P + d.
__device__ __forceinline__ float rgam(double P0, double P1, float d0, float d1, double &p0, double &p1) {
  p0 = dadd(P0, (double)d0);
  p1 = dadd(P1, (double)d1);
  return q_rsqrt((float)dadd(1.0, dadd(dmul(p0, p0), dmul(p1, p1))));
}

// Drift of one half step in cells: kh * p * (1/gamma).
__device__ __forceinline__ double half_drift(double kh, double p, float r) { return dmul(dmul(kh, p), (double)r); }

// The FP32-mode bunch seen as FP64 particles: position (with a pending
// trailing half drift undone) and full momentum of particle n.
struct Bunch32View {
  Bunch32 b;
  double P0, P1, kh0, kh1;
  int pending;
  double org0, org1, h0, h1;
  __device__ __forceinline__ void operator()(long long n, double &x, double &y, double &px, double &py) const {
    int ci, cj;
    unpack(b.cell[n], ci, cj);
    const float r = rgam(P0, P1, b.dpx[n], b.dpy[n], px, py);
    double s0 = b.ox[n], s1 = b.oy[n];
    if (pending) { s0 = dsub(s0, half_drift(kh0, px, r)); s1 = dsub(s1, half_drift(kh1, py, r)); }
    x = dadd(org0, dmul(dadd((double)ci, s0), h0));
    y = dadd(org1, dmul(dadd((double)cj, s1), h1));
  }
};

// Beam moments of the FP32-mode bunch read in place (diag.cu); the same
// out[18] layout and summation order as launch_moments on its FP64 copy.
void launch_moments32(const Bunch32View &v, double *part, double *mean, double *out, cudaStream_t s);

}  // namespace csrst
