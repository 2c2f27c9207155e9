// Element-wise and reduction kernels of the wake surrogate's training and
// inference (the products are the tensor-core GEMM of gemm.cu).  Reductions
// run in a fixed order, so a training run repeats bit for bit.
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/csrst.h"

namespace csrst {
namespace {

__device__ __forceinline__ long long gtid() { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }
inline unsigned grid_of(long long n) { return (unsigned)((n + 255) / 256 < 65535 * 16 ? (n + 255) / 256 : 65535 * 16); }

// [z][r][c] -> [z][c][r] (dst rows ldd apart) through 32 x 32 shared-memory
// tiles; T is a BF16 value or a 32-bit pair of them.
template <class T>
__global__ void k_transpose(const T *src, T *dst, int rows, int cols, int ldd) {
  __shared__ T t[32][33];
  const long long z = blockIdx.z;
  src += z * (long long)rows * cols;
  dst += z * (long long)ldd * cols;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[k][threadIdx.x] = src[(long long)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) dst[(long long)c * ldd + r] = t[threadIdx.x][k];
  }
}

// d/dx of 0.5 x (1 + erf(x / sqrt 2)) = 0.5 (1 + erf(x / sqrt 2)) + x exp(-x^2 / 2) / sqrt(2 pi)
__global__ void k_gelu_bwd(const float *dy, const float *pre, float *dx32, __nv_bfloat16 *dx16, long long n) {
  for (long long i = gtid(); i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = pre[i];
    const float d = 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * expf(-0.5f * x * x) * 0.3989422804014327f;
    const float v = dy[i] * d;
    if (dx32) dx32[i] = v;
    if (dx16) dx16[i] = __float2bfloat16(v);
  }
}

__global__ void k_cast(const float *x, __nv_bfloat16 *y, long long n) {
  for (long long i = gtid(); i < n; i += (long long)gridDim.x * blockDim.x) y[i] = __float2bfloat16(x[i]);
}

// out[c] (+)= sum_r x[r][c]: each block sums a 256-row slab per column, a
// second pass adds the slabs in order.
__global__ void k_colsum_part(const float *x, int rows, int cols, float *part) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const int r0 = blockIdx.y * 256, r1 = min(rows, r0 + 256);
  float s = 0.0f;
  for (int r = r0; r < r1; ++r) s += x[(long long)r * cols + c];
  part[(long long)blockIdx.y * cols + c] = s;
}
__global__ void k_colsum_final(const float *part, int slabs, int cols, float *out, int accumulate) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int k = 0; k < slabs; ++k) s += part[(long long)k * cols + c];
  out[c] = accumulate ? out[c] + s : s;
}

// Mean squared error, optionally weighted per output (a 0/1 weight leaves
// an output out): grad = 2 w^2 (pred - target) / n (written through gmap:
// index (i / gd) * g0 + (i % gd) * g1, so that the gradient lands in the layout
// of the last product), partial sums per block, then the total in order.
__global__ void k_mse(const float *pred, const float *target, const float *weight, long long n, float *grad, int gd,
                      long long g0, long long g1, double *part) {
  __shared__ double sh[256];
  double s = 0.0;
  for (long long i = gtid(); i < n; i += (long long)gridDim.x * blockDim.x) {
    const float e = weight ? (pred[i] - target[i]) * weight[i] : pred[i] - target[i];
    s += (double)e * e;
    if (grad) grad[(i / gd) * g0 + (i % gd) * g1] = 2.0f * (weight ? weight[i] : 1.0f) * e / (float)n;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_sum_final(const double *part, int np, long long n, double *out) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int k = 0; k < np; ++k) s += part[k];
  *out = s / (double)n;
}

// Adam (Kingma & Ba 2015) with bias correction.  The step counter and the
// schedule live on the device, so a captured training step replays as is:
// k_adam_tick advances t and writes {lr_t, 1 - b1^t, 1 - b2^t}, the learning
// rate following a cosine from lr0 to lr_min over `total` steps.
__global__ void k_adam_tick(int *t, float *coef, float lr0, float lr_min, int total, float b1, float b2) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int k = ++*t;
  const float f = k >= total ? 1.0f : (float)k / (float)total;
  coef[0] = lr_min + 0.5f * (lr0 - lr_min) * (1.0f + cospif(f));
  coef[1] = 1.0f - powf(b1, (float)k);
  coef[2] = 1.0f - powf(b2, (float)k);
}

__global__ void k_adam(float *w, const float *g, float *m, float *v, long long n, const float *coef, float b1,
                       float b2, float eps) {
  const float lr = coef[0], c1 = coef[1], c2 = coef[2];
  for (long long i = gtid(); i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// Complex spectral weights W_k = Wr + i Wi ([modes][cin][cout]) as the real
// block matrices the products take: Mk[2o + p][2c + q] (Z = U Mk^T) and its
// transpose MkT[2c + q][2o + p] (dU = dZ Mk).
__global__ void k_spectral_pack(const float *wr, const float *wi, int modes, int ch, __nv_bfloat16 *mk,
                                __nv_bfloat16 *mkt) {
  const long long n = (long long)modes * ch * ch;
  for (long long i = gtid(); i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / ((long long)ch * ch)), c = (int)((i / ch) % ch), o = (int)(i % ch);
    const float r = wr[i], im = wi[i];
    const long long base = (long long)k * 4 * ch * ch, w2 = 2 * ch;
    const float v[2][2] = {{r, -im}, {im, r}};  // [p][q]
    for (int p = 0; p < 2; ++p)
      for (int q = 0; q < 2; ++q) {
        mk[base + (long long)(2 * o + p) * w2 + 2 * c + q] = __float2bfloat16(v[p][q]);
        mkt[base + (long long)(2 * c + q) * w2 + 2 * o + p] = __float2bfloat16(v[p][q]);
      }
  }
}

// dWr[c][o] = dMk[2o][2c] + dMk[2o+1][2c+1], dWi[c][o] = dMk[2o+1][2c] - dMk[2o][2c+1]
__global__ void k_spectral_unpack(const float *dmk, int modes, int ch, float *dwr, float *dwi) {
  const long long n = (long long)modes * ch * ch;
  for (long long i = gtid(); i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / ((long long)ch * ch)), c = (int)((i / ch) % ch), o = (int)(i % ch);
    const long long base = (long long)k * 4 * ch * ch, w2 = 2 * ch;
    const float *d0 = dmk + base + (long long)(2 * o) * w2, *d1 = d0 + w2;
    dwr[i] = d0[2 * c] + d1[2 * c + 1];
    dwi[i] = d1[2 * c] - d0[2 * c + 1];
  }
}

}  // namespace
}  // namespace csrst

using namespace csrst;

extern "C" {

int csrst_nn_transpose_bf16(const void *src, void *dst, int batch, int rows, int cols, int ldd, void *stream) {
  if (!src || !dst || batch <= 0 || rows <= 0 || cols <= 0 || batch > 65535 || ldd < rows ||
      (rows + 31) / 32 > 65535)
    return CSRST_E_ARG;
  dim3 g((cols + 31) / 32, (rows + 31) / 32, batch);
  k_transpose<__nv_bfloat16><<<g, dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)src,
                                                                         (__nv_bfloat16 *)dst, rows, cols, ldd);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_transpose_b32(const void *src, void *dst, int batch, int rows, int cols, int ldd, void *stream) {
  if (!src || !dst || batch <= 0 || rows <= 0 || cols <= 0 || batch > 65535 || ldd < rows ||
      (rows + 31) / 32 > 65535 || ((uintptr_t)src & 3) || ((uintptr_t)dst & 3))
    return CSRST_E_ARG;
  dim3 g((cols + 31) / 32, (rows + 31) / 32, batch);
  k_transpose<uint32_t><<<g, dim3(32, 8), 0, (cudaStream_t)stream>>>((const uint32_t *)src, (uint32_t *)dst, rows,
                                                                     cols, ldd);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_gelu_bwd(const float *dy, const float *pre, float *dx32, void *dx16, long long n, void *stream) {
  if (!dy || !pre || n <= 0) return CSRST_E_ARG;
  k_gelu_bwd<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(dy, pre, dx32, (__nv_bfloat16 *)dx16, n);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_cast_bf16(const float *x, void *y, long long n, void *stream) {
  if (!x || !y || n <= 0) return CSRST_E_ARG;
  k_cast<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(x, (__nv_bfloat16 *)y, n);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_colsum(const float *x, int rows, int cols, float *part, float *out, int accumulate, void *stream) {
  if (!x || !part || !out || rows <= 0 || cols <= 0) return CSRST_E_ARG;
  const int slabs = (rows + 255) / 256;
  k_colsum_part<<<dim3((cols + 127) / 128, slabs), 128, 0, (cudaStream_t)stream>>>(x, rows, cols, part);
  k_colsum_final<<<(cols + 127) / 128, 128, 0, (cudaStream_t)stream>>>(part, slabs, cols, out, accumulate);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_mse(const float *pred, const float *target, const float *weight, long long n, float *grad, int gd,
                 long long g0, long long g1, double *part, double *loss, void *stream) {
  if (!pred || !target || !part || !loss || n <= 0 || gd <= 0) return CSRST_E_ARG;
  k_mse<<<256, 256, 0, (cudaStream_t)stream>>>(pred, target, weight, n, grad, gd, g0, g1, part);
  k_sum_final<<<1, 32, 0, (cudaStream_t)stream>>>(part, 256, n, loss);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_adam_tick(int *t, float *coef, float lr0, float lr_min, int total, float b1, float b2, void *stream) {
  if (!t || !coef || total <= 0) return CSRST_E_ARG;
  k_adam_tick<<<1, 32, 0, (cudaStream_t)stream>>>(t, coef, lr0, lr_min, total, b1, b2);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_adam(float *w, const float *g, float *m, float *v, long long n, const float *coef, float b1, float b2,
                  float eps, void *stream) {
  if (!w || !g || !m || !v || !coef || n <= 0) return CSRST_E_ARG;
  k_adam<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, coef, b1, b2, eps);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_spectral_pack(const float *wr, const float *wi, int modes, int ch, void *mk, void *mkt, void *stream) {
  if (!wr || !wi || !mk || !mkt || modes <= 0 || ch <= 0) return CSRST_E_ARG;
  k_spectral_pack<<<grid_of((long long)modes * ch * ch), 256, 0, (cudaStream_t)stream>>>(
      wr, wi, modes, ch, (__nv_bfloat16 *)mk, (__nv_bfloat16 *)mkt);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_nn_spectral_unpack(const float *dmk, int modes, int ch, float *dwr, float *dwi, void *stream) {
  if (!dmk || !dwr || !dwi || modes <= 0 || ch <= 0) return CSRST_E_ARG;
  k_spectral_unpack<<<grid_of((long long)modes * ch * ch), 256, 0, (cudaStream_t)stream>>>(dmk, modes, ch, dwr, dwi);
  return cudaGetLastError() == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

}  // extern "C"
