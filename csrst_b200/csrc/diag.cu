// Diagnostics on the device: beam moments (PartBunch::calcBeamParameters /
// calcMoments, PartBunch.cpp:584-767), the longitudinal field along the bunch
// axis that the CSR wake integrates (IntegrateElongCommand::execute,
// IntegrateElong.cpp:38-89) and the charge difference used by the FP64
// continuity check.  All reductions run in FP64 with a fixed order (per-CTA
// partials reduced by one CTA), so they are reproducible run to run.
#include "bunch32.cuh"
#include "kernels.cuh"
#include "shapes.cuh"

namespace csrst {

constexpr int kDiagBlocks = 296;

// True position when the -dt/2 drift is still pending on the stored R.
__device__ __forceinline__ void true_pos(double &x, double &y, double p0, double p1, double half,
                                         int pending) {
  if (!pending) return;
  const double r = inv_gamma(p0, p1);
  x = x + (-(half * p0 * r));
  y = y + (-(half * p1 * r));
}

template <int NV>
__device__ void block_sum(double (&v)[NV], double *out) {
  __shared__ double sh[NV][32];
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0)
    for (int k = 0; k < NV; ++k) sh[k][w] = v[k];
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int q = 0; q < nw; ++q) s += sh[threadIdx.x][q];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Particle sources of the moment passes: the FP64 arrays (positions with a
// pending trailing half drift undone), or the FP32-mode bunch read in place.
struct Bunch64View {
  const double *x, *y, *px, *py;
  double half;
  int pending;
  __device__ __forceinline__ void operator()(long long i, double &a, double &b, double &p0, double &p1) const {
    a = x[i]; b = y[i]; p0 = px[i]; p1 = py[i];
    true_pos(a, b, p0, p1, half, pending);
  }
};

// pass 1: sum x, px, y, py, gamma; min/max x, y.  part[b * 9 + k]
template <class Src>
__global__ void __launch_bounds__(256) k_mom1(Src src, long long n, double *part) {
  double v[5] = {0, 0, 0, 0, 0};
  double mn0 = INFINITY, mn1 = INFINITY, mx0 = -INFINITY, mx1 = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double a, b, p0, p1;
    src(i, a, b, p0, p1);
    v[0] += a; v[1] += p0; v[2] += b; v[3] += p1;
    v[4] += sqrt(1.0 + (p0 * p0 + p1 * p1));
    mn0 = fmin(mn0, a); mn1 = fmin(mn1, b); mx0 = fmax(mx0, a); mx1 = fmax(mx1, b);
  }
  block_sum<5>(v, part + blockIdx.x * 9);
  double m[4] = {mn0, mn1, -mx0, -mx1};
  __shared__ double sm[4][32];
  for (int k = 0; k < 4; ++k)
    for (int o = 16; o > 0; o >>= 1) m[k] = fmin(m[k], __shfl_down_sync(0xffffffffu, m[k], o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 4; ++k) sm[k][w] = m[k];
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = INFINITY;
    for (int q = 0; q < nw; ++q) s = fmin(s, sm[threadIdx.x][q]);
    part[blockIdx.x * 9 + 5 + threadIdx.x] = s;
  }
}

// pass 2: second moments of (x', px', y', py') in the frame of the mean
// momentum, centred on the mean position (PartBunch.cpp:724-745).  The
// reference forms sum(px'^2) - N |<p>|^2, which cancels to 1e-8 for a beam
// with 1e-4 energy spread; here px' is centred on |<p>| first and the
// identity sum(px'^2) - N m^2 = sum((px'-m)^2) + 2 m sum(px'-m) restores the
// same quantity without the cancellation.  Sums: q0^2, q2^2, (q1-m)^2, q3^2,
// q0 (q1-m), q0, q2 q3, (q1-m), and for the dispersion terms q2 (q1-m), q2,
// q3 (q1-m), q3 (the reference's moments(2,1) and (3,1) pair y' and py' with
// the uncentred px' = (q1-m) + m).
template <class Src>
__global__ void __launch_bounds__(256) k_mom2(Src src, long long n, const double *mean, double *part) {
  const double aR0 = mean[0], aR1 = mean[1], aP0 = mean[2], aP1 = mean[3];
  const double am = sqrt(aP0 * aP0 + aP1 * aP1), cph = aP0 / am, sph = aP1 / am;
  double v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double a, b, p0, p1;
    src(i, a, b, p0, p1);
    const double q1 = cph * p0 + sph * p1 - am;
    const double q3 = -sph * p0 + cph * p1;
    const double d0 = a - aR0, d2 = b - aR1;
    const double q0 = cph * d0 + sph * d2;
    const double q2 = -sph * d0 + cph * d2;
    v[0] += q0 * q0; v[1] += q2 * q2; v[2] += q1 * q1; v[3] += q3 * q3;
    v[4] += q0 * q1; v[5] += q0; v[6] += q2 * q3; v[7] += q1;
    v[8] += q2 * q1; v[9] += q2; v[10] += q3 * q1; v[11] += q3;
  }
  block_sum<12>(v, part + blockIdx.x * 12);
}

// Final reduction and the derived quantities; out[18] as the oracle's layout:
// rmean2 pmean2 rrms2 prms2 eps2 rmin2 rmax2 Ekin dE, pad.
// The final reductions run on one warp in a fixed order: lane t sums the
// block partials t, t + 32, ... in turn, then the lanes combine in a fixed
// shuffle tree, so the result does not depend on scheduling.  (One thread
// walking all partials waited on a dependent chain of a few thousand loads.)
template <int K>
__device__ __forceinline__ void warp_fixed_sums(const double *part, int nb, int stride, int k0, double (&v)[K]) {
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32)
    for (int k = 0; k < K; ++k) v[k] += part[b * stride + k0 + k];
  for (int k = 0; k < K; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
}

__global__ void k_mom_final1(const double *part, int nb, long long n, double *mean, double *out) {
  double s[5], m[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
  warp_fixed_sums<5>(part, nb, 9, 0, s);
  for (int b = threadIdx.x; b < nb; b += 32)
    for (int k = 0; k < 4; ++k) m[k] = fmin(m[k], part[b * 9 + 5 + k]);
  for (int k = 0; k < 4; ++k)
    for (int o = 16; o > 0; o >>= 1) m[k] = fmin(m[k], __shfl_down_sync(0xffffffffu, m[k], o));
  if (threadIdx.x != 0) return;
  const double N = (double)n;
  mean[0] = s[0] / N; mean[1] = s[2] / N; mean[2] = s[1] / N; mean[3] = s[3] / N; mean[4] = s[4] / N;
  out[0] = mean[0]; out[1] = mean[1]; out[2] = mean[2]; out[3] = mean[3];
  out[10] = m[0]; out[11] = m[1]; out[12] = -m[2]; out[13] = -m[3];
}

__global__ void k_mom_final2(const double *part, int nb, long long n, const double *mean, double *out) {
  double M[12];
  warp_fixed_sums<12>(part, nb, 12, 0, M);
  if (threadIdx.x != 0) return;
  const double N = (double)n;
  const double am = sqrt(mean[2] * mean[2] + mean[3] * mean[3]);
  const double rsq[2] = {M[0], M[1]};
  double psq[2] = {M[2] + 2.0 * am * M[7], M[3]};
  const double rp[2] = {M[4] + am * M[5], M[6]};
  for (int i = 0; i < 2; ++i) {
    if (psq[i] < 0) psq[i] = 0;
    const double e2 = (rsq[i] * psq[i] - rp[i] * rp[i]) / (N * N);
    out[4 + i] = sqrt(rsq[i] / N);
    out[6 + i] = sqrt(psq[i] / N);
    out[8 + i] = sqrt(fmax(e2, 0.0));
  }
  const double m0 = 0.51099906e-03 * 1000;
  const double ek = (mean[4] - 1.0) * m0;
  out[14] = ek;
  out[15] = out[6] * sqrt(ek * (ek + 2. * m0) / (1. + ek * (ek + 2. * m0) / (m0 * m0)));
  out[16] = (M[8] + am * M[9]) / N;   // Dy  = moments(2, 1) / N (PartBunch.cpp:643)
  out[17] = (M[10] + am * M[11]) / N;  // DDy = moments(3, 1) / N (PartBunch.cpp:644)
}

// E_s = cos(p) Ex + sin(p) Ey sampled at i = 2 .. L0-3 along the mean
// momentum direction through the centroid; NaN where the sample's cell lies
// outside the window.  The samples use the CIC edge gather of
// ScatterGatherImpl on the window.
template <class T>
struct WakeView {
  const T *base;
  int pitch;
  __device__ __forceinline__ double operator()(int i, int j) const { return (double)base[(ptrdiff_t)j * pitch + i]; }
};

template <class T>
__global__ void k_wake(const WinState *ws, const T *mEx, const T *mEy, int wpitch, double h0, double h1,
                       const double *mean, double *out) {
  const int L0 = ws->L0, L1 = ws->L1;
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i > L0 - 3) return;
  const double r0 = mean[0], r1 = mean[1], p0 = mean[2], p1 = mean[3];
  const double lenP = sqrt(p0 * p0 + p1 * p1);
  const double cP = p0 / lenP, sP = p1 / lenP;
  const double mo0 = ws->mo0, mo1 = ws->mo1;
  const double l0 = mo0 + i * h0 - r0;
  const double a0 = cP * l0 + sP * 0.0 + r0;
  const double a1 = -sP * l0 + cP * 0.0 + r1;
  const int ci = (int)floor((a0 - mo0) / h0), cj = (int)floor((a1 - mo1) / h1);
  if (ci < 0 || cj < 0 || ci >= L0 || cj >= L1) { out[i - 2] = NAN; return; }
  const WakeView<T> pex{mEx + wpitch + 1, wpitch}, pey{mEy + wpitch + 1, wpitch};
  const double pp0 = (a0 - mo0) * (1.0 / h0), pp1 = (a1 - mo1) * (1.0 / h1);
  const double e0 = gather_edge<0>(pex, pp0, pp1, 0), e1 = gather_edge<0>(pey, pp0, pp1, 1);
  out[i - 2] = cP * e0 + sP * e1;
}

// Charge difference rho(R) - rho(oldR) at vertices for the charge shape that
// matches the deposit order (get*ChargeDensityDiffImpl), fixed point.
template <int ORDER>
__global__ void k_charge_diff(const double *ox, const double *oy, const double *x, const double *y,
                              const double *q, long long n, double org0, double org1, double h0,
                              double h1, int i0, int j0, int ni, int nj, unsigned long long *acc,
                              double scale, int *dropped) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const double qq = q[k];
    for (int pass = 0; pass < 2; ++pass) {
      const double sg = pass == 0 ? 1.0 : -1.0;
      const double X = pass == 0 ? x[k] : ox[k], Y = pass == 0 ? y[k] : oy[k];
      auto add = [&](int i, int j, double v) {
        i -= i0; j -= j0;
        const long long iv = __double2ll_rn(sg * v * scale);
        if (i < 0 || j < 0 || i >= ni || j >= nj) {
          if (iv != 0) *dropped = 1;
          return;
        }
        atomicAdd(&acc[(size_t)j * ni + i], (unsigned long long)iv);
      };
      charge_shape<ORDER>(X, Y, qq, org0, org1, h0, h1, add);
    }
  }
}

// Field energy sums (CalcEnergyCommand::execute, CalcEnergy.cpp:41-120): the
// sum of Ex^2 + Ey^2 and of (Hzx + Hzy)^2 over the static mesh's Nx x Ny
// points and, with the window, over the window's L0 x L1 points, which replace
// the static points they cover.  One partial pair per block, summed in order.
template <class T>
__global__ void __launch_bounds__(256) k_energy(const T *Ex, const T *Ey, const T *Hx, const T *Hy, int pitch,
                                                int Nx, int Ny, const T *win, int wpitch, const WinState *ws,
                                                int with_window, double *part) {
  double v[2] = {0.0, 0.0};
  int P0 = 0, P1 = 0, L0 = 0, L1 = 0;
  if (with_window) { P0 = ws->P0; P1 = ws->P1; L0 = ws->L0; L1 = ws->L1; }
  const long long st = (long long)gridDim.x * blockDim.x;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (long long)Nx * Ny; k += st) {
    const int i = (int)(k % Nx), j = (int)(k / Nx);
    if (with_window && i >= P0 && i < P0 + L0 && j >= P1 && j < P1 + L1) continue;
    const size_t o = (size_t)(j + 1) * pitch + (i + 1);
    const double ex = (double)Ex[o], ey = (double)Ey[o], hz = (double)Hx[o] + (double)Hy[o];
    v[0] += ex * ex + ey * ey;
    v[1] += hz * hz;
  }
  if (with_window) {
    const size_t wp = (size_t)wpitch * (L1 + 2);
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (long long)L0 * L1; k += st) {
      const int i = (int)(k % L0), j = (int)(k / L0);
      const size_t o = (size_t)(j + 1) * wpitch + (i + 1);
      const double ex = (double)win[o], ey = (double)win[wp + o];
      const double hz = (double)win[2 * wp + o] + (double)win[3 * wp + o];
      v[0] += ex * ex + ey * ey;
      v[1] += hz * hz;
    }
  }
  block_sum<2>(v, part + blockIdx.x * 2);
}

__global__ void k_energy_final(const double *part, int nb, double area, double *out) {
  double v[2];
  warp_fixed_sums<2>(part, nb, 2, 0, v);
  if (threadIdx.x != 0) return;
  out[0] = v[0] * area;
  out[1] = v[1] * area;
}

// The static mesh with the window's values over the points it covers (the
// state copyFields leaves before SaveEMFieldsCommand, main.cpp:468-476):
// up to two planes summed (the split Hz); outside the static planes' guard
// ring, and for the static current (zero in the loop), the value is 0.
template <class T>
struct OverlayView {
  const T *s1, *s2;           // static planes (NULL: zero), interior (0, 0) at s + pitch + 1
  int pitch, Nx, Ny;
  const T *w1, *w2;           // window planes (NULL: no window)
  int wpitch, P0, P1, L0, L1;
  __device__ __forceinline__ double operator()(int i, int j) const {
    const int a = i - P0, b = j - P1;
    if (w1 && a >= 0 && a < L0 && b >= 0 && b < L1) {
      const ptrdiff_t o = (ptrdiff_t)(b + 1) * wpitch + a + 1;
      return (double)w1[o] + (w2 ? (double)w2[o] : 0.0);
    }
    if (!s1 || i < -1 || j < -1 || i > Nx || j > Ny) return 0.0;
    const ptrdiff_t o = (ptrdiff_t)(j + 1) * pitch + i + 1;
    return (double)s1[o] + (s2 ? (double)s2[o] : 0.0);
  }
};

// SaveEMFieldsCommand::execute (src/Commands/SaveEMFields.cpp:34-189): the
// fields along the line through the centroid in the direction of the mean
// momentum, one sample per static column i0 .. i0 + n - 1, gathered with the
// run's shape order from the overlaid mesh.  out[7 k ..]: signed distance from
// the centroid, E along and across the momentum, Hz, J along it, x, y; samples
// off the static mesh keep their position and zero fields.
template <int ORDER, class T>
__global__ void k_line_fields(const T *Ex, const T *Ey, const T *Hx, const T *Hy, int pitch, int Nx, int Ny,
                              const T *win, int wpitch, const WinState *ws, int with_current, double org0,
                              double org1, double h0, double h1, const double *mean, long long i0, int n,
                              double *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double R0 = mean[0], R1 = mean[1], P0 = mean[2], P1 = mean[3];
  const long long i = i0 + k;
  const double dx = (org0 + (double)i * h0) - R0;
  const double dy = dx / P0 * P1;
  double *o = out + 7 * (size_t)k;
  o[0] = sqrt(dx * dx + dy * dy) * (dx > 0 ? 1.0 : -1.0);
  o[5] = dx + R0;
  o[6] = dy + R1;
  const double x = org0 + (double)i * h0, y = R1 + (x - R0) / P0 * P1;
  const double pp0 = (x - org0) * (1.0 / h0), pp1 = (y - org1) * (1.0 / h1);
  const long long cy = (long long)floor(pp1);
  if (i < 0 || i >= Nx || cy < 0 || cy >= Ny) { o[1] = o[2] = o[3] = o[4] = 0.0; return; }
  const size_t wp = (size_t)wpitch * (ws->L1 + 2);
  const int WP0 = ws->P0, WP1 = ws->P1, L0 = ws->L0, L1 = ws->L1;
  const OverlayView<T> vEx{Ex, nullptr, pitch, Nx, Ny, win, nullptr, wpitch, WP0, WP1, L0, L1};
  const OverlayView<T> vEy{Ey, nullptr, pitch, Nx, Ny, win + wp, nullptr, wpitch, WP0, WP1, L0, L1};
  const OverlayView<T> vH{Hx, Hy, pitch, Nx, Ny, win + 2 * wp, win + 3 * wp, wpitch, WP0, WP1, L0, L1};
  const OverlayView<T> vJx{nullptr, nullptr, pitch, Nx, Ny, with_current ? win + 4 * wp : nullptr, nullptr, wpitch,
                           WP0, WP1, L0, L1};
  const OverlayView<T> vJy{nullptr, nullptr, pitch, Nx, Ny, with_current ? win + 5 * wp : nullptr, nullptr, wpitch,
                           WP0, WP1, L0, L1};
  const double e0 = gather_edge<ORDER>(vEx, pp0, pp1, 0), e1 = gather_edge<ORDER>(vEy, pp0, pp1, 1);
  const double hz = gather_cell<ORDER>(vH, pp0, pp1);
  const double j0 = gather_edge<ORDER>(vJx, pp0, pp1, 0), j1 = gather_edge<ORDER>(vJy, pp0, pp1, 1);
  const double lenP = sqrt(P0 * P0 + P1 * P1), cP = P0 / lenP, sP = P1 / lenP;
  o[1] = cP * e0 + sP * e1;
  o[2] = -sP * e0 + cP * e1;
  o[3] = hz;
  o[4] = cP * j0 + sP * j1;
}

// --- host launchers -----------------------------------------------------------

template <class Src>
static void moments_of(const Src &src, long long n, double *part, double *mean, double *out, cudaStream_t s) {
  k_mom1<<<kDiagBlocks, 256, 0, s>>>(src, n, part);
  k_mom_final1<<<1, 32, 0, s>>>(part, kDiagBlocks, n, mean, out);
  k_mom2<<<kDiagBlocks, 256, 0, s>>>(src, n, mean, part);
  k_mom_final2<<<1, 32, 0, s>>>(part, kDiagBlocks, n, mean, out);
}

void launch_moments(const double *x, const double *y, const double *px, const double *py, long long n,
                    double half, int pending, double *part, double *mean, double *out, cudaStream_t s) {
  moments_of(Bunch64View{x, y, px, py, half, pending}, n, part, mean, out, s);
}

// FP32 mode: the moments of the bunch read in place (the FP64 copy it would
// otherwise be converted into first holds the same values).
void launch_moments32(const Bunch32View &v, double *part, double *mean, double *out, cudaStream_t s) {
  moments_of(v, v.b.n, part, mean, out, s);
}

size_t moments_scratch_doubles() { return (size_t)kDiagBlocks * 12; }

template <class T>
void launch_line_fields(int order, const T *Ex, const T *Ey, const T *Hx, const T *Hy, int pitch, int Nx, int Ny,
                        const T *win, int wpitch, const WinState *ws, int with_current, double org0, double org1,
                        double h0, double h1, const double *mean, long long i0, int n, double *out, cudaStream_t s) {
  const int g = (n + 127) / 128;
  if (order == 0)
    k_line_fields<0, T><<<g, 128, 0, s>>>(Ex, Ey, Hx, Hy, pitch, Nx, Ny, win, wpitch, ws, with_current, org0, org1,
                                          h0, h1, mean, i0, n, out);
  else if (order == 1)
    k_line_fields<1, T><<<g, 128, 0, s>>>(Ex, Ey, Hx, Hy, pitch, Nx, Ny, win, wpitch, ws, with_current, org0, org1,
                                          h0, h1, mean, i0, n, out);
  else
    k_line_fields<2, T><<<g, 128, 0, s>>>(Ex, Ey, Hx, Hy, pitch, Nx, Ny, win, wpitch, ws, with_current, org0, org1,
                                          h0, h1, mean, i0, n, out);
}
template void launch_line_fields<double>(int, const double *, const double *, const double *, const double *, int,
                                         int, int, const double *, int, const WinState *, int, double, double,
                                         double, double, const double *, long long, int, double *, cudaStream_t);
template void launch_line_fields<float>(int, const float *, const float *, const float *, const float *, int, int,
                                        int, const float *, int, const WinState *, int, double, double, double,
                                        double, const double *, long long, int, double *, cudaStream_t);

template <class T>
void launch_field_energy(const T *Ex, const T *Ey, const T *Hx, const T *Hy, int pitch, int Nx, int Ny,
                         const T *win, int wpitch, const WinState *ws, int with_window, double area, double *part,
                         double *out, cudaStream_t s) {
  k_energy<T><<<kDiagBlocks, 256, 0, s>>>(Ex, Ey, Hx, Hy, pitch, Nx, Ny, win, wpitch, ws, with_window, part);
  k_energy_final<<<1, 32, 0, s>>>(part, kDiagBlocks, area, out);
}
template void launch_field_energy<double>(const double *, const double *, const double *, const double *, int, int,
                                          int, const double *, int, const WinState *, int, double, double *,
                                          double *, cudaStream_t);
template void launch_field_energy<float>(const float *, const float *, const float *, const float *, int, int, int,
                                         const float *, int, const WinState *, int, double, double *, double *,
                                         cudaStream_t);

template <class T>
void launch_wake(const WinState *ws, const T *mEx, const T *mEy, int wpitch, int L0, double h0, double h1,
                 const double *mean, double *out, cudaStream_t s) {
  const int n = L0 - 4;
  if (n <= 0) return;
  k_wake<T><<<(n + 127) / 128, 128, 0, s>>>(ws, mEx, mEy, wpitch, h0, h1, mean, out);
}
template void launch_wake<double>(const WinState *, const double *, const double *, int, int, double, double,
                                  const double *, double *, cudaStream_t);
template void launch_wake<float>(const WinState *, const float *, const float *, int, int, double, double,
                                 const double *, double *, cudaStream_t);

void launch_charge_diff(int order, const double *ox, const double *oy, const double *x, const double *y,
                        const double *q, long long n, double org0, double org1, double h0, double h1,
                        int i0, int j0, int ni, int nj, unsigned long long *acc, double scale,
                        int *dropped, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  if (order == 0)
    k_charge_diff<0><<<blocks, 256, 0, s>>>(ox, oy, x, y, q, n, org0, org1, h0, h1, i0, j0, ni, nj, acc, scale, dropped);
  else if (order == 1)
    k_charge_diff<1><<<blocks, 256, 0, s>>>(ox, oy, x, y, q, n, org0, org1, h0, h1, i0, j0, ni, nj, acc, scale, dropped);
  else
    k_charge_diff<2><<<blocks, 256, 0, s>>>(ox, oy, x, y, q, n, org0, org1, h0, h1, i0, j0, ni, nj, acc, scale, dropped);
}

}  // namespace csrst
