// Shared device definitions for the CSRST B200 kernels.
//
// Layout in HBM.  Every field component is its own plane (doubles on the FP64
// path, floats in FP32 mode) with a one-cell guard ring: element (i, j),
// i in [-1, nx], j in [-1, ny], sits at (j + 1) * pitch + (i + 1), x fastest.
// The static mesh pads the pitch so every row starts on a 256-byte boundary;
// the moving window uses pitch = L0 + 2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace csrst {

// Physical constants of the reference (src/Physics.cpp:41-51, src/defs.hh:30-31).
constexpr double kC = 299792458.0;
constexpr double kMu0 = 1.256637061e-06;
constexpr double kEps0 = 8.854187817e-12;
constexpr double kPi = 3.14159265358979323846;
constexpr double kSpaceEps = 1e-10;
constexpr double kMinArea = 1e-20;

// Error codes shared by the kernels and the C ABI (include/csrst.h).
enum : int {
  kOk = 0,
  kErrArg = -1,
  kErrCuda = -2,
  kErrGeometry = -3,
  kErrNoParticles = -4,
  kErrWindowFit = -5,
  kErrWindowMove = -6,
  kErrCrossings = -7,
  kErrWindowWall = -8,
  kErrStaging = -10,
};

template <class T>
struct PlaneT {
  T *p;
  int pitch;
  __host__ __device__ T &at(int i, int j) const { return p[(size_t)(j + 1) * pitch + (i + 1)]; }
};
using Plane = PlaneT<double>;

// Window state that lives on the device so that a whole time step can be
// captured in a CUDA graph: the host never needs the window position.
struct WinState {
  int P0, P1;                 // window position on the static mesh (ddim.first)
  int L0, L1;                 // window size in cells
  double mo0, mo1;            // window origin
  int cur;                    // which bbox slot holds the positions of the next push
  int gb[4];                  // last deposit's particle bounds (incl. old), window cells
  long long bb[2][4];         // ordered-int min x, min y, max x, max y of the next push's positions
  long long bball[4];         // bounds of the current push incl. old positions
  // Gather patch set-up derived from bb[cur] by the prep kernel
  // (PartBunch::getFields, PartBunch.cpp:957-1111).
  int lp[4];                  // particle domain (window cells)
  double ex_o0, ex_o1, ey_o0, ey_o1, hz_o0, hz_o1;  // patch origins
  int ex_I, ex_J, ey_I, ey_J, hz_I, hz_J;           // absolute index of patch (0, 0)
  int err;                    // sticky error code set by kernels
  int moves[2];               // last window move (moveI, moveJ)
};

// One conformal cut cell (BoundaryCell, src/BoundaryCell.hh:28-47) after
// SCBoundaryCondition::limitArea.
struct CutCellDev {
  int i, j;
  double l0, l1, area, n0, n1;
};

// Ordered-integer encoding of a double: a < b  <=>  enc(a) < enc(b).
__host__ __device__ inline long long dbl_ord(double v) {
  long long b;
#ifdef __CUDA_ARCH__
  b = __double_as_longlong(v);
#else
  __builtin_memcpy(&b, &v, 8);
#endif
  return b >= 0 ? b : (b ^ 0x7fffffffffffffffLL);
}
__host__ __device__ inline double ord_dbl(long long b) {
  long long r = b >= 0 ? b : (b ^ 0x7fffffffffffffffLL);
  double v;
#ifdef __CUDA_ARCH__
  v = __longlong_as_double(r);
#else
  __builtin_memcpy(&v, &r, 8);
#endif
  return v;
}

// The reference's float fast inverse square root used for 1/gamma
// (src/utils.hh:491-504).  Every float multiply and subtract rounds
// separately (explicit round-to-nearest operations), as on the host, in
// every translation unit whatever its contraction setting.
__device__ __forceinline__ float q_rsqrt(float x) {
  const float xhalf = __fmul_rn(0.5f, x);
  const float xqhalf = __fmul_rn(0.5010936f, x);
  unsigned int i = __float_as_uint(x);
  i = 0x5f3759dfu - (i >> 1);
  x = __uint_as_float(i);
  x = __fmul_rn(x, __fsub_rn(1.5f, __fmul_rn(__fmul_rn(xhalf, x), x)));
  x = __fmul_rn(x, __fsub_rn(1.5010936f, __fmul_rn(__fmul_rn(xqhalf, x), x)));
  return x;
}

// 1 / gamma for a momentum (beta gamma) vector, as the reference computes it.
__device__ __forceinline__ double inv_gamma(double p0, double p1) {
  return (double)q_rsqrt((float)(1.0 + (p0 * p0 + p1 * p1)));
}

__device__ __forceinline__ void set_err(WinState *ws, int code) { atomicCAS(&ws->err, 0, code); }

}  // namespace csrst
