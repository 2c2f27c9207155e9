// Allocation-free variant of the stand-alone current deposit
// (csrst_deposit_noalloc, declared in include/csrst.h).
//
// csrst_deposit copies its inputs to device memory it allocates and
// accumulates the current in a fixed-point buffer it allocates.  Some callers
// cannot let a library call cudaMalloc/cudaFree: a host framework that owns
// all device memory through its own pool and a fixed budget, or a time loop
// that must not stall the device (cudaMalloc and cudaFree synchronise it).
// Those callers pass device buffers for the inputs and the output; the only
// scratch this deposit needs, the fixed-point accumulator, lives in the
// file-scope array below, which every GPU that loads the library holds until
// the process exits.
#include <mutex>

#include "../../include/csrst.h"
#include "kernels.cuh"
#include "shapes.cuh"

namespace csrst {

// Largest patch (ni * nj cells) this entry point accepts: 2^20 cells, i.e.
// 8 MiB of 64-bit accumulator per device.
constexpr long long kNoAllocMaxCells = 1ll << 20;

static __device__ __align__(256) unsigned long long g_noalloc_acc[kNoAllocMaxCells];
// [0]: crossing overflow, [1]: a non-zero contribution fell outside the patch
static __device__ int g_noalloc_err[2];

__global__ void k_noalloc_clear(unsigned long long *acc, long long m) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x)
    acc[i] = 0ull;
  if (blockIdx.x == 0 && threadIdx.x == 0) { g_noalloc_err[0] = 0; g_noalloc_err[1] = 0; }
}

template <int ORDER>
__global__ void k_noalloc_deposit(int comp, const double *ox, const double *oy, const double *x,
                                  const double *y, const double *q, long long n, double org0, double org1,
                                  double h0, double h1, double dt, int i0, int j0, int ni, int nj,
                                  unsigned long long *acc, double scale) {
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
      g_noalloc_err[0] = kErrCrossings;
    if (dropped) g_noalloc_err[1] = 1;
  }
}

__global__ void k_noalloc_out(const unsigned long long *acc, double *J, long long m, double inv) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x)
    J[i] = (double)(long long)acc[i] * inv;
}

// Device address of the accumulator, looked up once per device.
static int noalloc_scratch(unsigned long long **out) {
  static std::mutex mtx;
  static unsigned long long *addr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return kErrCuda;
  std::lock_guard<std::mutex> lock(mtx);
  if (!addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_acc) != cudaSuccess) return kErrCuda;
    addr[dev] = static_cast<unsigned long long *>(p);
  }
  *out = addr[dev];
  return kOk;
}

}  // namespace csrst

extern "C" int csrst_deposit_noalloc(int order, int comp, const double *ox, const double *oy, const double *x,
                                     const double *y, const double *q, size_t n, const double *o2,
                                     const double *hh2, double dt, int i0, int j0, int ni, int nj, double scale,
                                     double *J, void *stream) {
  using namespace csrst;
  if (order < 0 || order > 2 || (comp != 0 && comp != 1) || ni <= 0 || nj <= 0 || !o2 || !hh2 || !J ||
      !(scale > 0) || (n > 0 && (!ox || !oy || !x || !y || !q)))
    return set_global_error(CSRST_E_ARG, "invalid deposit arguments");
  const long long m = (long long)ni * nj;
  if (m > kNoAllocMaxCells)
    return set_global_error(CSRST_E_ARG, "patch larger than the 2^20-cell accumulator of the allocation-free deposit");
  unsigned long long *acc = nullptr;
  if (noalloc_scratch(&acc) != kOk) return set_global_error(CSRST_E_CUDA, "cudaGetSymbolAddress failed");
  // drop an error left by earlier, unrelated work, so that the checks below
  // see only this call's launches
  (void)cudaGetLastError();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int gm = (int)((m + 255) / 256 < 2048 ? (m + 255) / 256 : 2048);
  k_noalloc_clear<<<gm, 256, 0, s>>>(acc, m);
  if (n > 0) {
    const int gp = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    if (order == 0)
      k_noalloc_deposit<0><<<gp, 256, 0, s>>>(comp, ox, oy, x, y, q, (long long)n, o2[0], o2[1], hh2[0], hh2[1],
                                              dt, i0, j0, ni, nj, acc, scale);
    else if (order == 1)
      k_noalloc_deposit<1><<<gp, 256, 0, s>>>(comp, ox, oy, x, y, q, (long long)n, o2[0], o2[1], hh2[0], hh2[1],
                                              dt, i0, j0, ni, nj, acc, scale);
    else
      k_noalloc_deposit<2><<<gp, 256, 0, s>>>(comp, ox, oy, x, y, q, (long long)n, o2[0], o2[1], hh2[0], hh2[1],
                                              dt, i0, j0, ni, nj, acc, scale);
  }
  k_noalloc_out<<<gm, 256, 0, s>>>(acc, J, m, 1.0 / scale);
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return set_global_error(CSRST_E_CUDA, cudaGetErrorString(ce));
  // the flags come back in stream order, so only this stream is waited for
  int e[2] = {0, 0};
  ce = cudaMemcpyFromSymbolAsync(e, g_noalloc_err, sizeof e, 0, cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess) return set_global_error(CSRST_E_CUDA, cudaGetErrorString(ce));
  if (e[0]) return set_global_error(CSRST_E_CROSSINGS, "too many cell-border crossings");
  if (e[1]) return set_global_error(CSRST_W_OUTSIDE, "contributions outside the patch were dropped");
  return CSRST_OK;
}
