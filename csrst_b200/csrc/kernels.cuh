// Argument blocks and host launchers shared by the kernel files and the C ABI.
#pragma once

#include <string>

#include "common.cuh"

namespace csrst {

// One push (PartBunch::push_particles) over all particles.
struct PushArgs {
  double *x, *y, *px, *py;
  const double *q;
  long long n;
  WinState *ws;
  // window fields (guarded planes, pitch L0 + 2)
  const double *mEx, *mEy, *mHx, *mHy;
  int wpitch;
  unsigned long long *acc;  // L0 * L1 fixed-point current for jcomp
  double acc_scale;
  int jcomp, pending;
  double half;               // 0.5 * dt * c
  double fact1, fact2;       // half * q/m, fact1 * c
  double h0, h1, dt;
  // hard-edge dipole (Bend::getExternalField, Bend.cpp:865-907)
  double bz, Lb, hw, chh, shh, bwidth;
  int use_smem;
};

// One field sub-step over the static mesh, the cut cells and the window.
struct FieldArgs {
  Plane Ex, Ey, Hx, Hy;            // static mesh
  const uint8_t *mask;             // inside mask, Nx * Ny, x fastest
  int Nx, Ny;
  Plane mEx, mEy, mHx, mHy, mJx, mJy;  // window
  int L0, L1;
  const CutCellDev *cells;
  int ncells;
  WinState *ws;
  unsigned long long *acc;         // fixed-point window current of the E sub-step
  double acc_inv;
  // regular-cell coefficients (TETMSolver.hh:121-125)
  double chx, chy;                 // 0.5 * eta_x / Z0, 0.5 * eta_y / Z0
  double kex, key;                 // eta_y * Z0, eta_x * Z0
  double dteps;                    // c dt Z0
  // cut-cell coefficients (TETMSolver.cpp:87-127)
  double mhx, mhy;                 // -0.5 dt / (hx mu0), +0.5 dt / (hy mu0)
  double de;                       // dt / eps0
  double h0, h1;
  int nbS, nbC, tilesX;            // block ranges: static tiles, cut-cell blocks
};

// Bend parameters (Bend ctor and Bend::Init, Bend.cpp:60-124).
struct BendDev {
  int Nx, Ny;
  double Lb, La, w, R, phi, cphi, sphi;
  double hr0, hr1, org0, org1, cen0, cen1;
};

// particles.cu
void launch_bbox_next(const double *x, const double *y, const double *px, const double *py, long long n,
                      double half, int pending, WinState *ws, cudaStream_t s);
void launch_push_prep(WinState *ws, double h0, double h1, int order, cudaStream_t s);
void launch_push(const PushArgs &a, int order, int L0, int L1, int grid, cudaStream_t s);
void launch_global_bounds(WinState *ws, double h0, double h1, cudaStream_t s);
void launch_drift(double *x, double *y, const double *px, const double *py, long long n, double full,
                  cudaStream_t s);
void launch_gather(int order, int comp, const double *patch, int nx, double o0, double o1, double h0,
                   double h1, const double *x, const double *y, long long n, double *out, cudaStream_t s);
void launch_deposit(int order, int comp, const double *ox, const double *oy, const double *x,
                    const double *y, const double *q, long long n, double org0, double org1, double h0,
                    double h1, double dt, int i0, int j0, int ni, int nj, unsigned long long *acc,
                    double scale, int *err, cudaStream_t s);
void launch_fixed_to_double(const unsigned long long *acc, double *out, long long n, double inv,
                            cudaStream_t s);
// fields.cu
void launch_half_h(FieldArgs a, cudaStream_t s);
void launch_update_e(FieldArgs a, int comp, cudaStream_t s);
void launch_exchange(FieldArgs a, int which, cudaStream_t s);
void launch_copy_to_window(FieldArgs a, cudaStream_t s);
void launch_check_window(FieldArgs a, cudaStream_t s);
void launch_move(FieldArgs a, double *scratch, double h0, double h1, cudaStream_t s);
void launch_reset_outside(FieldArgs a, const int *cutidx, cudaStream_t s);
// geometry.cu
int build_geometry(const BendDev &b, uint8_t *d_mask, CutCellDev **d_cells, int *ncells, int **d_cutidx,
                   cudaStream_t s);
// diag.cu
void launch_moments(const double *x, const double *y, const double *px, const double *py, long long n,
                    double half, int pending, double *part, double *mean, double *out, cudaStream_t s);
size_t moments_scratch_doubles();
void launch_wake(const WinState *ws, const double *mEx, const double *mEy, int wpitch, int L0, double h0,
                 double h1, const double *mean, double *out, cudaStream_t s);
void launch_charge_diff(int order, const double *ox, const double *oy, const double *x, const double *y,
                        const double *q, long long n, double org0, double org1, double h0, double h1,
                        int i0, int j0, int ni, int nj, unsigned long long *acc, double scale,
                        cudaStream_t s);

// poisson.cu: initial fields of the bunch (PoissonSolver::computeField)
struct PoissonInput {
  const double *x, *y, *px, *py, *q;  // bunch on the device, positions R
  long long n;
  int order;                          // charge shape
  const uint8_t *mask;                // inside mask, Nx * Ny
  const int *cutidx;                  // cut-cell index per cell or -1
  const CutCellDev *cells;
  BendDev b;
  double dt;
  Plane Ex, Ey, Hx, Hy;               // static planes written
  double tol_first, tol_rest;         // relative residual of solve 1 and of solves 2, 3
  int maxit;
};
struct PoissonReport {
  double gamma;
  int iters[3];
  double relres[3];
  int levels;
};
int poisson_initial_fields(const PoissonInput &in, PoissonReport *rep, cudaStream_t s, std::string *msg);

}  // namespace csrst
