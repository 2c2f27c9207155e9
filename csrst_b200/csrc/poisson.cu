// Initial fields of the bunch: the three boosted electrostatic solves of
// PoissonSolver::computeField (PoissonSolver.cpp:85-201) on the GPU.
//
// The matrix is the reference's (cutoffStencil, PoissonSolver.cpp:678-766): the
// 5-point Laplacian with spacings (gamma hx, hy) on the vertices that are
// inside the pipe or on a cut cell of area > 0.5 and lie before the bend
// (i < L_before / hx, Bend::getLengthStraightSection); every other row is an
// identity row.  Identity rows fix phi = b there, which moves their couplings
// to the right-hand side of the rows next to them; what remains is symmetric
// positive definite and is solved by CG preconditioned with one multigrid
// V-cycle:
//   - x-semicoarsening: the boosted x-spacing is gamma times the y-spacing,
//     so the operator couples along y about gamma^2 times more strongly and
//     only x is coarsened (columns are merged in pairs);
//   - Galerkin coarse operators R A P with P piecewise constant over a pair
//     of columns and R = P^T / 2; they keep the 5-point shape;
//   - zebra y-line Gauss-Seidel smoothing: a column is one tridiagonal system,
//     solved exactly by parallel cyclic reduction in the shared memory of one
//     CTA.  The pre-smoother (red, black) and the post-smoother (black, red)
//     mirror each other, so the V-cycle is a symmetric preconditioner.
// All arithmetic is FP64.  Vectors are stored column-major (i * ny + j), so a
// y-line is contiguous.  Dot products are two-pass block trees with a fixed
// grid, so a solve gives the same bits on every run.
#include <cmath>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "shapes.cuh"

namespace csrst {
namespace {

struct Level {
  int nx, ny;
  double *D, *W, *E, *S, *N;  // stencil; off-diagonals are 0 towards inactive cells
  uint8_t *act;
  double *u, *f, *r;          // correction, right-hand side, residual
};

constexpr int kDotBlocks = 296;
constexpr int kMaxLineLen = 4096;  // y-line length the shared-memory solver takes

__device__ __forceinline__ long long gtid() { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }

// Row classes: good = inside or a cut cell with area > 0.5; active = good and
// before the bend.  Column-major output.
__global__ void k_classes(const uint8_t *mask, const int *cutidx, const CutCellDev *cells, int Nx, int Ny,
                          long long maxX, uint8_t *good, uint8_t *act) {
  const long long k = gtid();
  if (k >= (long long)Nx * Ny) return;
  const int i = (int)(k / Ny), j = (int)(k % Ny);
  const size_t rm = (size_t)j * Nx + i;
  const int c = cutidx[rm];
  const bool g = mask[rm] || (c >= 0 && cells[c].area > 0.5);
  good[k] = g;
  act[k] = g && i < maxX;
}

__global__ void k_coeff0(Level L, double EW, double NS, double Dc) {
  const long long k = gtid();
  if (k >= (long long)L.nx * L.ny) return;
  const int i = (int)(k / L.ny), j = (int)(k % L.ny);
  if (!L.act[k]) {
    L.D[k] = 1.0; L.W[k] = L.E[k] = L.S[k] = L.N[k] = 0.0;
    return;
  }
  L.D[k] = Dc;
  L.W[k] = (i > 0 && L.act[k - L.ny]) ? EW : 0.0;
  L.E[k] = (i + 1 < L.nx && L.act[k + L.ny]) ? EW : 0.0;
  L.S[k] = (j > 0 && L.act[k - 1]) ? NS : 0.0;
  L.N[k] = (j + 1 < L.ny && L.act[k + 1]) ? NS : 0.0;
}

// Galerkin coarse stencil of a pair of columns (2I, 2I+1).
__global__ void k_coarsen(Level F, Level C) {
  const long long k = gtid();
  if (k >= (long long)C.nx * C.ny) return;
  const int I = (int)(k / C.ny), j = (int)(k % C.ny);
  const size_t a = (size_t)(2 * I) * F.ny + j, b = a + F.ny;
  const bool ha = F.act[a], hb = 2 * I + 1 < F.nx && F.act[b];
  if (!ha && !hb) {
    C.act[k] = 0;
    C.D[k] = 1.0; C.W[k] = C.E[k] = C.S[k] = C.N[k] = 0.0;
    return;
  }
  double D = 0.0, W = 0.0, E = 0.0, S = 0.0, N = 0.0;
  if (ha) { D += F.D[a] + F.E[a]; W += F.W[a]; S += F.S[a]; N += F.N[a]; }
  if (hb) { D += F.D[b] + F.W[b]; E += F.E[b]; S += F.S[b]; N += F.N[b]; }
  C.act[k] = 1;
  C.D[k] = 0.5 * D; C.W[k] = 0.5 * W; C.E[k] = 0.5 * E; C.S[k] = 0.5 * S; C.N[k] = 0.5 * N;
}

__device__ __forceinline__ double apply_at(const Level &L, const double *u, long long k) {
  const int i = (int)(k / L.ny), j = (int)(k % L.ny);
  double v = L.D[k] * u[k];
  if (i > 0) v += L.W[k] * u[k - L.ny];
  if (i + 1 < L.nx) v += L.E[k] * u[k + L.ny];
  if (j > 0) v += L.S[k] * u[k - 1];
  if (j + 1 < L.ny) v += L.N[k] * u[k + 1];
  return v;
}

__global__ void k_apply(Level L, const double *u, double *out) {
  const long long k = gtid();
  if (k >= (long long)L.nx * L.ny) return;
  out[k] = L.act[k] ? apply_at(L, u, k) : 0.0;
}

__global__ void k_resid(Level L) {
  const long long k = gtid();
  if (k >= (long long)L.nx * L.ny) return;
  L.r[k] = L.act[k] ? L.f[k] - apply_at(L, L.u, k) : 0.0;
}

__global__ void k_restrict(Level F, Level C) {
  const long long k = gtid();
  if (k >= (long long)C.nx * C.ny) return;
  const int I = (int)(k / C.ny), j = (int)(k % C.ny);
  const size_t a = (size_t)(2 * I) * F.ny + j;
  double v = F.r[a];
  if (2 * I + 1 < F.nx) v += F.r[a + F.ny];
  C.f[k] = C.act[k] ? 0.5 * v : 0.0;
  C.u[k] = 0.0;
}

__global__ void k_prolong(Level F, Level C) {
  const long long k = gtid();
  if (k >= (long long)F.nx * F.ny) return;
  if (!F.act[k]) return;
  const int i = (int)(k / F.ny), j = (int)(k % F.ny);
  F.u[k] += C.u[(size_t)(i / 2) * C.ny + j];
}

// Exact solve of every y-line of one colour (columns colour, colour + 2, ...)
// with the neighbouring columns held fixed, by parallel cyclic reduction.
template <int EPT>
__global__ void __launch_bounds__(1024) k_line(Level L, int colour) {
  extern __shared__ double sm[];
  const int i = 2 * blockIdx.x + colour;
  if (i >= L.nx) return;
  const int ny = L.ny;
  double *sa = sm, *sb = sm + ny, *sc = sm + 2 * ny, *sd = sm + 3 * ny;
  const size_t base = (size_t)i * ny;
  for (int j = threadIdx.x; j < ny; j += blockDim.x) {
    const size_t k = base + j;
    if (L.act[k]) {
      double d = L.f[k];
      if (i > 0) d -= L.W[k] * L.u[k - ny];
      if (i + 1 < L.nx) d -= L.E[k] * L.u[k + ny];
      sa[j] = L.S[k]; sb[j] = L.D[k]; sc[j] = L.N[k]; sd[j] = d;
    } else {
      sa[j] = 0.0; sb[j] = 1.0; sc[j] = 0.0; sd[j] = 0.0;
    }
  }
  __syncthreads();
  for (int s = 1; s < ny; s <<= 1) {
    double na[EPT], nb[EPT], nc[EPT], nd[EPT];
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int j = threadIdx.x + e * blockDim.x;
      if (j >= ny) continue;
      const double a = sa[j], c = sc[j];
      double A = 0.0, B = sb[j], Cc = 0.0, D = sd[j];
      if (j - s >= 0) {
        const double al = -a / sb[j - s];
        A = al * sa[j - s]; B += al * sc[j - s]; D += al * sd[j - s];
      }
      if (j + s < ny) {
        const double ga = -c / sb[j + s];
        Cc = ga * sc[j + s]; B += ga * sa[j + s]; D += ga * sd[j + s];
      }
      na[e] = A; nb[e] = B; nc[e] = Cc; nd[e] = D;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int j = threadIdx.x + e * blockDim.x;
      if (j >= ny) continue;
      sa[j] = na[e]; sb[j] = nb[e]; sc[j] = nc[e]; sd[j] = nd[e];
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < ny; j += blockDim.x) {
    const size_t k = base + j;
    L.u[k] = L.act[k] ? sd[j] / sb[j] : 0.0;
  }
}

// --- CG vector kernels -------------------------------------------------------

__global__ void k_dot_part(const double *a, const double *b, long long n, double *part) {
  __shared__ double sh[256];
  double s = 0.0;
  for (long long k = blockIdx.x * 256ll + threadIdx.x; k < n; k += (long long)gridDim.x * 256)
    s += a[k] * b[k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_parts(const double *part, int np, double *out) {
  __shared__ double sh[512];
  sh[threadIdx.x] = threadIdx.x < np ? part[threadIdx.x] : 0.0;
  __syncthreads();
  for (int w = 256; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_axpy2(double *u, double *r, const double *d, const double *q, double alpha, long long n) {
  const long long k = gtid();
  if (k >= n) return;
  u[k] += alpha * d[k];
  r[k] -= alpha * q[k];
}

__global__ void k_xpby(double *d, const double *z, double beta, long long n) {
  const long long k = gtid();
  if (k < n) d[k] = z[k] + beta * d[k];
}

__global__ void k_sub(double *r, const double *f, const double *q, long long n) {
  const long long k = gtid();
  if (k < n) r[k] = f[k] - q[k];
}

__global__ void k_copy(double *dst, const double *src, long long n) {
  const long long k = gtid();
  if (k < n) dst[k] = src[k];
}

// --- right-hand side, shifts and fields ----------------------------------------

__global__ void k_psum(const double *px, const double *py, const double *q, long long n, double *part) {
  __shared__ double sh[3][256];
  double a = 0.0, b = 0.0, c = 0.0;
  for (long long k = blockIdx.x * 256ll + threadIdx.x; k < n; k += (long long)gridDim.x * 256) {
    a += px[k]; b += py[k]; c += fabs(q[k]);
  }
  sh[0][threadIdx.x] = a; sh[1][threadIdx.x] = b; sh[2][threadIdx.x] = c;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int t = 0; t < 3; ++t) sh[t][threadIdx.x] += sh[t][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int t = 0; t < 3; ++t) part[t * kDotBlocks + blockIdx.x] = sh[t][0];
}

// Charge of the bunch at the positions of one solve (mode 0: R + dt/2 drift;
// 1: that, drifted back and moved by -hx/2 in x; 2: R), accumulated in 64-bit
// fixed point on the row-major Nx x Ny vertices.
template <int ORDER>
__global__ void k_rho(const double *x, const double *y, const double *px, const double *py, const double *q,
                      long long n, int mode, double full, double back, double mv, double org0, double org1,
                      double h0, double h1, int Nx, int Ny, unsigned long long *acc, double scale) {
  for (long long k = gtid(); k < n; k += (long long)gridDim.x * blockDim.x) {
    double X = x[k], Y = y[k];
    if (mode < 2) {
      const double p0 = px[k], p1 = py[k];
      const double r = inv_gamma(p0, p1);
      X = X + full * p0 * r; Y = Y + full * p1 * r;
      if (mode == 1) { X = (X + back * p0 * r) + mv; Y = (Y + back * p1 * r) + 0.0; }
    }
    charge_shape<ORDER>(X, Y, q[k], org0, org1, h0, h1, [&](int i, int j, double v) {
      if (i < 0 || j < 0 || i >= Nx || j >= Ny) return;
      atomicAdd(&acc[(size_t)j * Nx + i], (unsigned long long)__double2ll_rn(v * scale));
    });
  }
}

// b = rho / (eps0 gamma), column-major; rho = (fixed-point sum) / (hx hy).
__global__ void k_rhs(const unsigned long long *acc, double inv, double area, double cc, int Nx, int Ny,
                      double *b) {
  const long long k = gtid();
  if (k >= (long long)Nx * Ny) return;
  const int i = (int)(k / Ny), j = (int)(k % Ny);
  b[k] = ((double)(long long)acc[(size_t)j * Nx + i] * inv / area) * cc;
}

// Right-hand side of the active rows: b minus the couplings to identity rows.
__global__ void k_rhs_eff(Level L, const uint8_t *good, const double *b, double EW, double NS, double *f) {
  const long long k = gtid();
  if (k >= (long long)L.nx * L.ny) return;
  if (!L.act[k]) { f[k] = 0.0; return; }
  const int i = (int)(k / L.ny), j = (int)(k % L.ny);
  double v = b[k];
  if (j > 0 && good[k - 1] && !L.act[k - 1]) v -= NS * b[k - 1];
  if (i > 0 && good[k - L.ny] && !L.act[k - L.ny]) v -= EW * b[k - L.ny];
  if (i + 1 < L.nx && good[k + L.ny] && !L.act[k + L.ny]) v -= EW * b[k + L.ny];
  if (j + 1 < L.ny && good[k + 1] && !L.act[k + 1]) v -= NS * b[k + 1];
  f[k] = v;
}

// Initial guess from the previous solution (shiftLHS, PoissonSolver.cpp:270-303):
// tau = +1 takes the right neighbour, tau = -1/2 mixes in the left one.
__global__ void k_shift(const double *phi, double *out, double tau, int Nx, int Ny) {
  const long long k = gtid();
  if (k >= (long long)Nx * Ny) return;
  const int i = (int)(k / Ny);
  if (tau > 0) {
    const double nb = i + 1 < Nx ? phi[k + Ny] : 0.0;
    out[k] = phi[k] + (tau * nb - tau * phi[k]);
  } else {
    const double t = -tau;
    const double nb = i > 0 ? phi[k - Ny] : 0.0;
    out[k] = phi[k] + (t * nb - t * phi[k]);
  }
}

__global__ void k_finish(const uint8_t *act, const double *u, const double *b, double *phi, long long n) {
  const long long k = gtid();
  if (k < n) phi[k] = act[k] ? u[k] : b[k];
}

__global__ void k_init_u(const uint8_t *act, const double *x0, double *u, long long n) {
  const long long k = gtid();
  if (k < n) u[k] = act[k] ? x0[k] : 0.0;
}

// PoissonSolver::fillFields (PoissonSolver.cpp:441-507): Ey from the first
// potential, Hz (both split halves) from the second, Ex from the third; the
// guard beyond the last row / column holds zero.
__global__ void k_fields(const double *phi1, const double *phi2, const double *phi3, int Nx, int Ny,
                         double gamma, double hr0, double hr1, double bg, double hden, Plane Ex, Plane Ey,
                         Plane Hx, Plane Hy) {
  const long long t = gtid();
  if (t >= (long long)Nx * Ny) return;
  const int i = (int)(t % Nx), j = (int)(t / Nx);
  const size_t k = (size_t)i * Ny + j;
  const double ey0 = gamma * phi1[k] / hr1;
  const double ey1 = j + 1 < Ny ? gamma * phi1[k + 1] / hr1 : 0.0;
  Ey.at(i, j) = ey0 - ey1;
  const double h0v = bg * phi2[k] / hden;
  const double h1v = j + 1 < Ny ? bg * phi2[k + 1] / hden : 0.0;
  Hx.at(i, j) = h0v - h1v;
  Hy.at(i, j) = h0v - h1v;
  const double ex0 = phi3[k] / hr0;
  const double ex1 = i + 1 < Nx ? phi3[k + Ny] / hr0 : 0.0;
  Ex.at(i, j) = ex0 - ex1;
}

inline unsigned blocks_for(long long n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

// Device buffers of one solve, freed together.
struct Pool {
  std::vector<void *> ptrs;
  cudaError_t err = cudaSuccess;
  template <class T>
  T *get(size_t count) {
    void *p = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&p, count * sizeof(T) > 0 ? count * sizeof(T) : 1);
    if (p) ptrs.push_back(p);
    return static_cast<T *>(p);
  }
  ~Pool() {
    for (void *p : ptrs) cudaFree(p);
  }
};

class Solver {
 public:
  Solver(std::vector<Level> &lv, double *part, double *scal, cudaStream_t s) : lv_(lv), part_(part), scal_(scal), s_(s) {}

  cudaError_t dot(const double *a, const double *b, double *out) {
    const long long n = (long long)lv_[0].nx * lv_[0].ny;
    k_dot_part<<<kDotBlocks, 256, 0, s_>>>(a, b, n, part_);
    k_sum_parts<<<1, 512, 0, s_>>>(part_, kDotBlocks, scal_);
    cudaError_t e = cudaMemcpyAsync(out, scal_, sizeof(double), cudaMemcpyDeviceToHost, s_);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s_);
  }

  void line(int l, int colour) {
    const Level &L = lv_[l];
    const int ncol = (L.nx - colour + 1) / 2;
    if (ncol <= 0) return;
    int bs = L.ny < 1024 ? ((L.ny + 31) / 32) * 32 : 1024;
    const int ept = (L.ny + bs - 1) / bs;
    const size_t sm = 4 * (size_t)L.ny * sizeof(double);
    if (ept <= 1) k_line<1><<<ncol, bs, sm, s_>>>(L, colour);
    else if (ept <= 2) k_line<2><<<ncol, bs, sm, s_>>>(L, colour);
    else k_line<4><<<ncol, bs, sm, s_>>>(L, colour);
  }

  // z = V-cycle(r): level 0 right-hand side r, zero initial correction.
  void vcycle(const double *r, double *z) {
    const int nl = (int)lv_.size();
    const long long n0 = (long long)lv_[0].nx * lv_[0].ny;
    k_copy<<<blocks_for(n0), 256, 0, s_>>>(lv_[0].f, r, n0);
    cudaMemsetAsync(lv_[0].u, 0, n0 * sizeof(double), s_);
    for (int l = 0; l + 1 < nl; ++l) {
      line(l, 0); line(l, 1);
      const long long n = (long long)lv_[l].nx * lv_[l].ny, nc = (long long)lv_[l + 1].nx * lv_[l + 1].ny;
      k_resid<<<blocks_for(n), 256, 0, s_>>>(lv_[l]);
      k_restrict<<<blocks_for(nc), 256, 0, s_>>>(lv_[l], lv_[l + 1]);
    }
    for (int k = 0; k < 4; ++k) { line(nl - 1, 0); line(nl - 1, 1); line(nl - 1, 1); line(nl - 1, 0); }
    for (int l = nl - 2; l >= 0; --l) {
      const long long n = (long long)lv_[l].nx * lv_[l].ny;
      k_prolong<<<blocks_for(n), 256, 0, s_>>>(lv_[l], lv_[l + 1]);
      line(l, 1); line(l, 0);
    }
    k_copy<<<blocks_for(n0), 256, 0, s_>>>(z, lv_[0].u, n0);
  }

 private:
  std::vector<Level> &lv_;
  double *part_, *scal_;
  cudaStream_t s_;
};

}  // namespace

int poisson_initial_fields(const PoissonInput &in, PoissonReport *rep, cudaStream_t s, std::string *msg) {
  const int Nx = in.b.Nx, Ny = in.b.Ny;
  const long long m = (long long)Nx * Ny;
  auto fail = [&](const char *what, cudaError_t e) {
    if (msg) *msg = std::string(what) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    return e != cudaSuccess ? kErrCuda : kErrArg;
  };
  if (in.n <= 0) return fail("no particles", cudaSuccess);
  if (Ny > kMaxLineLen) return fail("the multigrid line solver takes at most 4096 rows", cudaSuccess);
  Pool pool;
  // mean momentum and total |q| (Distribution::get_pmean)
  double *part = pool.get<double>(3 * kDotBlocks), *scal = pool.get<double>(4);
  if (pool.err) return fail("cudaMalloc", pool.err);
  k_psum<<<kDotBlocks, 256, 0, s>>>(in.px, in.py, in.q, in.n, part);
  for (int t = 0; t < 3; ++t) k_sum_parts<<<1, 512, 0, s>>>(part + t * kDotBlocks, kDotBlocks, scal + t);
  double sums[3];
  cudaError_t e = cudaMemcpyAsync(sums, scal, sizeof(sums), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail("momentum sum", e);
  const double pm0 = sums[0] / (double)in.n, pm1 = sums[1] / (double)in.n;
  const double gamma = std::sqrt((pm0 * pm0 + pm1 * pm1) + 1);
  const double hr0 = in.b.hr0 * gamma, hr1 = in.b.hr1;
  const double EW = -1 / (hr0 * hr0), NS = -1 / (hr1 * hr1), Dc = -2 * (EW + NS);
  const long long maxX = (long long)(size_t)(in.b.Lb / in.b.hr0);

  // hierarchy
  std::vector<Level> lv;
  {
    int nx = Nx;
    while (true) {
      Level L{};
      L.nx = nx; L.ny = Ny;
      const size_t c = (size_t)nx * Ny;
      L.D = pool.get<double>(c); L.W = pool.get<double>(c); L.E = pool.get<double>(c);
      L.S = pool.get<double>(c); L.N = pool.get<double>(c);
      L.act = pool.get<uint8_t>(c);
      L.u = pool.get<double>(c); L.f = pool.get<double>(c); L.r = pool.get<double>(c);
      lv.push_back(L);
      if (nx <= 2) break;
      nx = (nx + 1) / 2;
    }
  }
  uint8_t *good = pool.get<uint8_t>(m);
  double *b = pool.get<double>(m), *f = pool.get<double>(m), *x = pool.get<double>(m), *r = pool.get<double>(m);
  double *z = pool.get<double>(m), *d = pool.get<double>(m), *q = pool.get<double>(m);
  double *phi[3] = {pool.get<double>(m), pool.get<double>(m), pool.get<double>(m)};
  unsigned long long *acc = pool.get<unsigned long long>(m);
  if (pool.err) return fail("cudaMalloc (multigrid hierarchy)", pool.err);
  // shared memory of the line solver
  {
    const int sm = 4 * Ny * (int)sizeof(double);
    for (cudaError_t ee : {cudaFuncSetAttribute(k_line<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm),
                           cudaFuncSetAttribute(k_line<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm),
                           cudaFuncSetAttribute(k_line<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm)})
      if (ee != cudaSuccess) return fail("line solver shared memory", ee);
  }
  k_classes<<<blocks_for(m), 256, 0, s>>>(in.mask, in.cutidx, in.cells, Nx, Ny, maxX, good, lv[0].act);
  k_coeff0<<<blocks_for(m), 256, 0, s>>>(lv[0], EW, NS, Dc);
  for (size_t l = 1; l < lv.size(); ++l)
    k_coarsen<<<blocks_for((long long)lv[l].nx * Ny), 256, 0, s>>>(lv[l - 1], lv[l]);

  Solver sv(lv, part, scal, s);
  const double area = in.b.hr0 * in.b.hr1, cc = 1 / (kEps0 * gamma);
  const double qsum = sums[2] > 0 ? sums[2] : 1e-300;
  const double scale = std::ldexp(1.0, (int)std::floor(std::log2(std::ldexp(1.0, 62) / qsum)));
  const double full = (in.dt / 2) * kC, back = (-in.dt / 2) * kC, mv = -0.5 * hr0 / gamma;
  const unsigned pg = blocks_for(in.n) < 4096 ? blocks_for(in.n) : 4096;
  const double tols[3] = {in.tol_first, in.tol_rest, in.tol_rest};
  for (int sol = 0; sol < 3; ++sol) {
    // right-hand side of this solve
    cudaMemsetAsync(acc, 0, m * sizeof(unsigned long long), s);
    const int mode = sol;  // 0: R + dt/2 drift, 1: shifted by -hx/2, 2: R
    if (in.order == 0)
      k_rho<0><<<pg, 256, 0, s>>>(in.x, in.y, in.px, in.py, in.q, in.n, mode, full, back, mv, in.b.org0,
                                  in.b.org1, in.b.hr0, in.b.hr1, Nx, Ny, acc, scale);
    else if (in.order == 1)
      k_rho<1><<<pg, 256, 0, s>>>(in.x, in.y, in.px, in.py, in.q, in.n, mode, full, back, mv, in.b.org0,
                                  in.b.org1, in.b.hr0, in.b.hr1, Nx, Ny, acc, scale);
    else
      k_rho<2><<<pg, 256, 0, s>>>(in.x, in.y, in.px, in.py, in.q, in.n, mode, full, back, mv, in.b.org0,
                                  in.b.org1, in.b.hr0, in.b.hr1, Nx, Ny, acc, scale);
    k_rhs<<<blocks_for(m), 256, 0, s>>>(acc, 1.0 / scale, area, cc, Nx, Ny, b);
    k_rhs_eff<<<blocks_for(m), 256, 0, s>>>(lv[0], good, b, EW, NS, f);
    // initial guess: 0, then the shifted previous potential
    if (sol == 0) cudaMemsetAsync(x, 0, m * sizeof(double), s);
    else k_shift<<<blocks_for(m), 256, 0, s>>>(phi[sol - 1], x, sol == 1 ? 1.0 : -0.5, Nx, Ny);
    k_init_u<<<blocks_for(m), 256, 0, s>>>(lv[0].act, x, x, m);
    // preconditioned CG
    k_apply<<<blocks_for(m), 256, 0, s>>>(lv[0], x, q);
    k_sub<<<blocks_for(m), 256, 0, s>>>(r, f, q, m);
    double bn2 = 0, rn2 = 0, rz = 0;
    if ((e = sv.dot(f, f, &bn2)) != cudaSuccess) return fail("dot", e);
    if ((e = sv.dot(r, r, &rn2)) != cudaSuccess) return fail("dot", e);
    const double bn = std::sqrt(bn2);
    double rn = std::sqrt(rn2);
    int it = 0;
    if (bn == 0.0) {
      cudaMemsetAsync(x, 0, m * sizeof(double), s);
      rn = 0.0;
    } else {
      sv.vcycle(r, z);
      k_copy<<<blocks_for(m), 256, 0, s>>>(d, z, m);
      if ((e = sv.dot(r, z, &rz)) != cudaSuccess) return fail("dot", e);
      while (rn / bn > tols[sol] && it < in.maxit) {
        k_apply<<<blocks_for(m), 256, 0, s>>>(lv[0], d, q);
        double dq = 0;
        if ((e = sv.dot(d, q, &dq)) != cudaSuccess) return fail("dot", e);
        const double alpha = rz / dq;
        k_axpy2<<<blocks_for(m), 256, 0, s>>>(x, r, d, q, alpha, m);
        ++it;
        if ((e = sv.dot(r, r, &rn2)) != cudaSuccess) return fail("dot", e);
        rn = std::sqrt(rn2);
        if (rn / bn <= tols[sol]) break;
        sv.vcycle(r, z);
        double rz1 = 0;
        if ((e = sv.dot(r, z, &rz1)) != cudaSuccess) return fail("dot", e);
        const double beta = rz1 / rz;
        rz = rz1;
        k_xpby<<<blocks_for(m), 256, 0, s>>>(d, z, beta, m);
      }
    }
    k_finish<<<blocks_for(m), 256, 0, s>>>(lv[0].act, x, b, phi[sol], m);
    if (rep) { rep->iters[sol] = it; rep->relres[sol] = bn == 0.0 ? 0.0 : rn / bn; }
  }
  const double bg = std::sqrt(gamma * gamma - 1), hden = 2 * kC * kMu0 * hr1;
  k_fields<<<blocks_for(m), 256, 0, s>>>(phi[0], phi[1], phi[2], Nx, Ny, gamma, hr0, hr1, bg, hden, in.Ex, in.Ey,
                                         in.Hx, in.Hy);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail("initial-field kernels", e);
  if (rep) { rep->gamma = gamma; rep->levels = (int)lv.size(); }
  return kOk;
}

}  // namespace csrst
