// FP32-mode bunch arithmetic shared by the particle kernels and the
// diagnostics: every operation on positions and momenta is an explicitly
// rounded FP32 operation, so that the same inputs give the same bits in every
// kernel, whatever contraction the translation unit is compiled with.
#pragma once

#include "kernels.cuh"

namespace csrst {

__device__ __forceinline__ void unpack(int c, int &i, int &j) {
  i = c & 0xffff;
  j = (int)((unsigned)c >> 16);
}

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }

// 1/gamma of the momentum P + d with the reference's float Q_rsqrt
// (utils.hh:491-504, PartBunch.cpp:173-184): its argument 1 + |P + d|^2 is
// formed as (1 + |P|^2) + (2 P.d + |d|^2) in FP32, within an FP32 rounding of
// the FP64 path's argument (the deviation d stays below ~1 while P is ~1e3).
__device__ __forceinline__ float rgam32(const Ref32 &R, float d0, float d1) {
  const float dev = fadd(fmul(2.0f, fadd(fmul(R.P0, d0), fmul(R.P1, d1))), fadd(fmul(d0, d0), fmul(d1, d1)));
  return q_rsqrt(fadd(R.G2, dev));
}

// Drift in cells: kh * (P + d) * (1/gamma) (kh = c dt' / h for the step dt').
__device__ __forceinline__ float drift32(float kh, float P, float d, float r) { return fmul(fmul(kh, fadd(P, d)), r); }

// Start of the next push for a particle stored at offset o (cells in its
// cell): with the trailing -dt/2 drift still pending the particle sits at
// o - w, else at o.
__device__ __forceinline__ void start32(const Ref32 &R, int pending, float o0, float o1, float d0, float d1, float &a0,
                                        float &a1) {
  a0 = o0; a1 = o1;
  if (pending) {
    const float r = rgam32(R, d0, d1);
    a0 = fsub(o0, drift32(R.kh0, R.P0, d0, r));
    a1 = fsub(o1, drift32(R.kh1, R.P1, d1, r));
  }
}

// The FP32-mode bunch seen as FP64 particles: position (with a pending
// trailing half drift applied, exactly as the next push starts from it) and
// full momentum of particle n.
struct Bunch32View {
  Bunch32 b;
  Ref32 R;
  double P0, P1;
  int pending;
  double org0, org1, h0, h1;
  __device__ __forceinline__ void operator()(long long n, double &x, double &y, double &px, double &py) const {
    int ci, cj;
    unpack(b.cell[n], ci, cj);
    const float d0 = b.dpx[n], d1 = b.dpy[n];
    float s0, s1;
    start32(R, pending, b.ox[n], b.oy[n], d0, d1, s0, s1);
    px = __dadd_rn(P0, (double)d0);
    py = __dadd_rn(P1, (double)d1);
    x = __dadd_rn(org0, __dmul_rn(__dadd_rn((double)ci, (double)s0), h0));
    y = __dadd_rn(org1, __dmul_rn(__dadd_rn((double)cj, (double)s1), h1));
  }
};

// Beam moments of the FP32-mode bunch read in place (diag.cu); the same
// out[18] layout and summation order as launch_moments on its FP64 copy.
void launch_moments32(const Bunch32View &v, double *part, double *mean, double *out, cudaStream_t s);

}  // namespace csrst
