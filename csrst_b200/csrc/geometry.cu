// Bend geometry on the GPU: inside test per vertex, edge fractions (lambda)
// and inside mask per cell, cut-cell areas, and the ordered cut-cell list.
// Restates Bend::isInside / crossBoundary / getLambdaField /
// getBoundaryCellAreas (src/Bend.cpp:126-235, :427-545, :664-799) and
// SCBoundaryCondition::limitArea (SCBoundaryCondition.hh:131-137).  The
// dual-grid cut cells (Bend.cpp:547-729) feed nothing in the time step and are
// not built.  cos/sin of the bend angle come from the host so the GPU and a
// host build see the same doubles.
#include <cub/cub.cuh>

#include "kernels.cuh"

namespace csrst {

__device__ bool bend_inside(const BendDev &b, double x0, double x1) {
  const double cosphi = b.cphi, sinphi = b.sphi;
  const double rmin_sq = (b.R - 0.5 * b.w) * (b.R - 0.5 * b.w);
  const double rmax_sq = (b.R + 0.5 * b.w) * (b.R + 0.5 * b.w);
  const double D0 = x0 - b.cen0, D1 = x1 - b.cen1;
  if (D0 < 0.0) {
    if (x0 < kSpaceEps || x1 < kSpaceEps || x1 > b.w - kSpaceEps) return false;
  } else if (D1 * sinphi > D0 * cosphi) {
    const double l = D0 * D0 + D1 * D1;
    if (l <= rmin_sq || l >= rmax_sq) return false;
  } else {
    double p0, p1;
    if (fabs(b.phi) > kSpaceEps) {
      p0 = cosphi * D0 + (-sinphi) * D1 + b.cen0;
      p1 = sinphi * D0 + cosphi * D1 + b.cen1;
    } else {
      p0 = x0; p1 = x1;
    }
    if (p1 < kSpaceEps || p1 > b.w - kSpaceEps || p0 > b.Lb + b.La - kSpaceEps) return false;
  }
  return true;
}

// Fraction of the edge base -> base + dir that is inside the pipe; false
// where the reference asserts.  Note the first straight section's top-wall
// branch returns max(1, min(0, .)) = 1, kept as written.
__device__ bool bend_cross(const BendDev &b, double base0, double base1, double dir0, double dir1,
                           double &out) {
  const double cosphi = b.cphi, sinphi = b.sphi;
  const double x0 = base0 + b.org0, x1 = base1 + b.org1;
  const double D0 = x0 - b.cen0, D1 = x1 - b.cen1;
  if (D0 < 0.0) {
    double t = 99.9;
    if (x1 < b.w + kSpaceEps && x1 + dir1 > b.w - kSpaceEps) t = fmax(1.0, fmin(0.0, (b.w - x1) / dir1));
    if (x1 > -kSpaceEps && x1 + dir1 < kSpaceEps) t = fmin(t, -x1 / dir1);
    if (x0 > -kSpaceEps && x0 + dir0 < kSpaceEps) t = fmin(t, -x0 / dir0);
    out = t;
    return true;
  } else if (D1 * sinphi > D0 * cosphi) {
    const double rmin_sq = (b.R - 0.5 * b.w) * (b.R - 0.5 * b.w);
    const double rmax_sq = (b.R + 0.5 * b.w) * (b.R + 0.5 * b.w);
    const double dist1 = D0 * D0 + D1 * D1;
    const double e0 = D0 + dir0, e1 = D1 + dir1;
    const double dist2 = e0 * e0 + e1 * e1;
    const double aa = dir0 * dir0 + dir1 * dir1;
    const double bb = D0 * dir0 + D1 * dir1;
    double c;
    if (dist1 < rmax_sq && dist2 > rmax_sq) c = (D0 * D0 + D1 * D1) - rmax_sq;
    else if (dist1 > rmin_sq && dist2 < rmin_sq) c = (D0 * D0 + D1 * D1) - rmin_sq;
    else { out = 99.9; return true; }
    double t = 99.9;
    double tau = (-bb + sqrt(bb * bb - aa * c)) / aa;
    if (fabs(tau - 0.5) < 0.5) t = tau;
    tau = -tau - 2 * bb / aa;
    if (fabs(tau - 0.5) < 0.5) t = fmin(t, tau);
    out = t;
    return true;
  } else {
    double xr0, xr1, dr0, dr1;
    if (fabs(b.phi) > kSpaceEps) {
      xr0 = cosphi * D0 - sinphi * D1 + b.cen0;
      xr1 = sinphi * D0 + cosphi * D1 + b.cen1;
      dr0 = cosphi * dir0 - sinphi * dir1;
      dr1 = sinphi * dir0 + cosphi * dir1;
    } else {
      xr0 = x0; xr1 = x1; dr0 = dir0; dr1 = dir1;
    }
    double t0 = 99.9, t1 = 99.9, t2 = 99.9;
    if (fabs(dr1) > kSpaceEps) {
      t0 = -xr1 / dr1; if (t0 < 0.0) t0 = 99.9;
      t1 = (b.w - xr1) / dr1; if (t1 < 0.0) t1 = 99.9;
    }
    if (fabs(dr0) > kSpaceEps) {
      t2 = (b.Lb + b.La - xr0) / dr0; if (t2 < 0.0) t2 = 99.9;
    }
    double t = fmin(t0, fmin(t1, t2));
    if (t > 1 + kSpaceEps && t < 1.001) t = 1.0;
    if (!(t < 1 + kSpaceEps) || !(t >= 0)) return false;
    out = fmin(1.0, fmax(0.0, t));
    return true;
  }
}

// Vertex flags with a guard of 2 (GenericGeometry uses GEOMETRY_GCS = 2).
__global__ void k_vertices(BendDev b, uint8_t *iv) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)b.Nx * b.Ny) return;
  const int cx = (int)(k % b.Nx), cy = (int)(k / b.Nx);
  const double x1 = b.org1 + cy * b.hr1, x0 = b.org0 + cx * b.hr0;
  iv[(size_t)(cy + 2) * (b.Nx + 4) + cx + 2] = bend_inside(b, x0, x1) ? 1 : 0;
}

__device__ __forceinline__ int cell_case(const BendDev &b, const uint8_t *iv, int cx, int cy) {
  const int W = b.Nx + 4;
  const uint8_t *p = iv + (size_t)(cy + 2) * W + cx + 2;
  return p[0] + (p[1] << 1) + (p[W] << 2) + (p[W + 1] << 3);
}

// lambda (2 doubles per cell, guard 2, zero outside), inside mask, candidates.
__global__ void k_lambda(BendDev b, const uint8_t *iv, double *lam, uint8_t *mask, uint8_t *cand,
                         int *err) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)b.Nx * b.Ny) return;
  const int cx = (int)(k % b.Nx), cy = (int)(k / b.Nx);
  const int cc = cell_case(b, iv, cx, cy);
  double l0 = 0.0, l1 = 0.0;
  mask[k] = cc == 15;
  cand[k] = cc != 0 && cc != 15;
  const double h0 = b.hr0, h1 = b.hr1;
  bool ok = true;
  switch (cc) {
    case 15: l0 = 1.0; l1 = 1.0; break;
    case 1: ok &= bend_cross(b, cx * h0, cy * h1, h0, 0.0, l0); ok &= bend_cross(b, cx * h0, cy * h1, 0.0, h1, l1); break;
    case 2: case 10: ok &= bend_cross(b, (cx + 1) * h0, cy * h1, -h0, 0.0, l0); l1 = 0.0; break;
    case 3: case 11: l0 = 1.0; ok &= bend_cross(b, cx * h0, cy * h1, 0.0, h1, l1); break;
    case 4: case 12: l0 = 0.0; ok &= bend_cross(b, cx * h0, (cy + 1) * h1, 0.0, -h1, l1); break;
    case 5: case 13: ok &= bend_cross(b, cx * h0, cy * h1, h0, 0.0, l0); l1 = 1.0; break;
    case 7: l0 = 1.0; l1 = 1.0; break;
    case 8: l0 = 0.0; l1 = 0.0; break;
    case 14: ok &= bend_cross(b, (cx + 1) * h0, cy * h1, -h0, 0.0, l0);
             ok &= bend_cross(b, cx * h0, (cy + 1) * h1, 0.0, -h1, l1); break;
    default: break;
  }
  if (!ok) atomicExch(err, kErrGeometry);
  double *q = lam + ((size_t)(cy + 2) * (b.Nx + 4) + cx + 2) * 2;
  q[0] = l0; q[1] = l1;
}

__device__ double area_cases(int cc, double l0, double l1, double n0, double n1) {
  switch (cc) {
    case 1: return l0 * l1 / 2;
    case 2: return l0 * n1 / 2;
    case 3: return (l1 + n1) / 2;
    case 4: return n0 * l1 / 2;
    case 5: return (l0 + n0) / 2;
    case 7: return 1 - (1 - n0) * (1 - n1) / 2;
    case 8: return n0 * n1 / 2;
    case 10: return (l0 + n0) / 2;
    case 11: return 1 - (1 - l1) * (1 - n0) / 2;
    case 12: return (l1 + n1) / 2;
    case 13: return 1 - (1 - l0) * (1 - n1) / 2;
    case 14: return 1 - (1 - l0) * (1 - l1) / 2;
    default: return 0.0;
  }
}

// Area per candidate; keep[k] = 1 for the cells the reference keeps.
__global__ void k_area(BendDev b, const uint8_t *iv, const double *lam, const uint8_t *cand,
                       uint8_t *keep, double *area, int *err) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)b.Nx * b.Ny) return;
  keep[k] = 0;
  if (!cand[k]) return;
  const int cx = (int)(k % b.Nx), cy = (int)(k / b.Nx);
  const int cc = cell_case(b, iv, cx, cy);
  const size_t W = b.Nx + 4;
  const double *q = lam + ((size_t)(cy + 2) * W + cx + 2) * 2;
  const double l0 = q[0], l1 = q[1];
  const double n0 = q[2 * W], n1 = q[2 + 1];
  double a = area_cases(cc, l0, l1, n0, n1);
  if (!(a < 1.0 + kSpaceEps) || !(a >= 0.0)) { atomicExch(err, kErrGeometry); return; }
  if (a < kSpaceEps) return;
  a = fmax(a, l0 / 2); a = fmax(a, l1 / 2); a = fmax(a, n0 / 2); a = fmax(a, n1 / 2);
  keep[k] = 1;
  area[k] = a;
}

__global__ void k_cells(BendDev b, const long long *sel, int n, const double *lam, const double *area,
                        CutCellDev *cells, int *cutidx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long k = sel[t];
  const int cx = (int)(k % b.Nx), cy = (int)(k / b.Nx);
  const size_t W = b.Nx + 4;
  const double *q = lam + ((size_t)(cy + 2) * W + cx + 2) * 2;
  CutCellDev c;
  c.i = cx; c.j = cy; c.l0 = q[0]; c.l1 = q[1]; c.n0 = q[2 * W]; c.n1 = q[3];
  c.area = area[k];
  cells[t] = c;
  cutidx[k] = t;
}

__global__ void k_fill_int(int *p, long long n, int v) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k < n) p[k] = v;
}

// Builds mask (Nx*Ny bytes), the cut-cell list and the cell -> cut-cell map.
// All temporaries are freed before return.  Returns a csrst error code.
int build_geometry(const BendDev &b, uint8_t *d_mask, CutCellDev **d_cells, int *ncells,
                   int **d_cutidx, cudaStream_t s) {
  const long long nc = (long long)b.Nx * b.Ny;
  const size_t W = (size_t)(b.Nx + 4) * (b.Ny + 4);
  uint8_t *iv = nullptr, *cand = nullptr, *keep = nullptr;
  double *lam = nullptr, *area = nullptr;
  long long *sel = nullptr;
  int *err = nullptr, *nsel = nullptr;
  void *tmp = nullptr;
  size_t tmpb = 0;
  int rc = kOk, h_err = 0, h_n = 0;
  auto ck = [&](cudaError_t e) { if (e != cudaSuccess && rc == kOk) rc = kErrCuda; };
  ck(cudaMalloc(&iv, W));
  ck(cudaMalloc(&lam, W * 2 * sizeof(double)));
  ck(cudaMalloc(&cand, nc));
  ck(cudaMalloc(&keep, nc));
  ck(cudaMalloc(&area, nc * sizeof(double)));
  ck(cudaMalloc(&sel, nc * sizeof(long long)));
  ck(cudaMalloc(&err, sizeof(int)));
  ck(cudaMalloc(&nsel, sizeof(int)));
  if (rc == kOk) {
    ck(cudaMemsetAsync(iv, 0, W, s));
    ck(cudaMemsetAsync(lam, 0, W * 2 * sizeof(double), s));
    ck(cudaMemsetAsync(err, 0, sizeof(int), s));
    const unsigned g = (unsigned)((nc + 255) / 256);
    k_vertices<<<g, 256, 0, s>>>(b, iv);
    k_lambda<<<g, 256, 0, s>>>(b, iv, lam, d_mask, cand, err);
    k_area<<<g, 256, 0, s>>>(b, iv, lam, cand, keep, area, err);
    cub::CountingInputIterator<long long> it(0);
    ck(cub::DeviceSelect::Flagged(nullptr, tmpb, it, keep, sel, nsel, nc, s));
    ck(cudaMalloc(&tmp, tmpb));
    if (rc == kOk) ck(cub::DeviceSelect::Flagged(tmp, tmpb, it, keep, sel, nsel, nc, s));
    ck(cudaMemcpyAsync(&h_n, nsel, sizeof(int), cudaMemcpyDeviceToHost, s));
    ck(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    ck(cudaStreamSynchronize(s));
  }
  if (rc == kOk && h_err) rc = h_err;
  if (rc == kOk) {
    *ncells = h_n;
    ck(cudaMalloc(d_cells, (size_t)(h_n > 0 ? h_n : 1) * sizeof(CutCellDev)));
    ck(cudaMalloc(d_cutidx, nc * sizeof(int)));
    if (rc == kOk) {
      k_fill_int<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(*d_cutidx, nc, -1);
      if (h_n > 0) k_cells<<<(h_n + 255) / 256, 256, 0, s>>>(b, sel, h_n, lam, area, *d_cells, *d_cutidx);
      ck(cudaStreamSynchronize(s));
    }
  }
  cudaFree(iv); cudaFree(lam); cudaFree(cand); cudaFree(keep); cudaFree(area);
  cudaFree(sel); cudaFree(err); cudaFree(nsel); cudaFree(tmp);
  return rc;
}

}  // namespace csrst
