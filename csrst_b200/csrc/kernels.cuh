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
};

// One cell of the absorbing layer at an open end of the pipe (convolutional
// PML with kappa = 1, csrst_set_pml): each component's curl difference d is
// replaced by d + psi, with psi <- b psi + a d updated first, b = exp(-sigma
// dt'/eps0), a = b - 1 over the component's update interval dt' (dt/2 for the
// half H updates, dt for E).  sigma is the layer's conductivity split along
// the pipe axis: sigma_x for Hzx and Ey, sigma_y for Hzy and Ex, each at its
// component's position.  psi lives in its own array, 4 per cell.
template <class T>
struct PmlCellT {
  int i, j;
  T bhx, ahx, bhy, ahy;  // Hzx, Hzy (half step)
  T bex, aex, bey, aey;  // Ex, Ey
};

// One field sub-step over the static mesh, the cut cells and the window.
// T is the field type: double on the FP64 path, float in FP32 mode.
template <class T>
struct FieldArgsT {
  PlaneT<T> Ex, Ey, Hx, Hy;        // static mesh
  const uint8_t *mask;             // inside mask, Nx * Ny, x fastest
  int Nx, Ny;
  PlaneT<T> mEx, mEy, mHx, mHy, mJx, mJy;  // window
  int L0, L1;
  const CutCellDev *cells;
  int ncells;
  WinState *ws;
  unsigned long long *acc;         // fixed-point window current of the E sub-step
  double acc_inv;
  // regular-cell coefficients (TETMSolver.hh:121-125)
  T chx, chy;                      // 0.5 * eta_x / Z0, 0.5 * eta_y / Z0
  T kex, key;                      // eta_y * Z0, eta_x * Z0
  T dteps;                         // c dt Z0
  // cut-cell coefficients (TETMSolver.cpp:87-127)
  T mhx, mhy;                      // -0.5 dt / (hx mu0), +0.5 dt / (hy mu0)
  T de;                            // dt / eps0
  T h0, h1;
  int nbS, nbC, tilesX;            // block ranges: static tiles, cut-cell blocks
  int tx, ty;                      // static-sweep tile (tx * ty = 256; 0 = 32 x 8)
  // absorbing layers (csrst_set_pml; null when off): the cells, and per row
  // the columns [lo, hi) left to the regular sweep
  const PmlCellT<T> *pml;
  T *psi;                          // 4 per layer cell: Hzx, Hzy, Ex, Ey
  int npml, nbP;
  const int2 *pml_rows;
};
using FieldArgs = FieldArgsT<double>;

// Window move of one member (fields.cu).
template <class T>
struct MoveArgs {
  FieldArgsT<T> f;
  T *scratch;           // 6 window planes
  double h0, h1;
};

// Bend parameters (Bend ctor and Bend::Init, Bend.cpp:60-124).
struct BendDev {
  int Nx, Ny;
  double Lb, La, w, R, phi, cphi, sphi;
  double hr0, hr1, org0, org1, cen0, cen1;
};

// Per-member arguments of the small bookkeeping kernels around a push.
struct PrepArgs {
  WinState *ws;
  double h0, h1;
  int em0, em2, cm0;  // gather-patch margins of the shape order
};

// The members of one shape order in a batched push (device arrays of m
// entries; ppre: first particle of each member, m + 1 entries).
struct PushGroup {
  int order, m, jcomp;
  const void *args;                 // PushArgs or Push32Args
  const unsigned char *smem_ok;     // the member's window accumulator fits in shared memory
  const long long *ppre;
  long long total, all;             // particles of the group, of the whole batch
  size_t smem;                      // dynamic shared memory of the group's launch
};

// api.cu: records the message csrst_get_error(NULL) returns and returns code
// (for entry points that take no handle).
int set_global_error(int code, const char *msg);

// particles.cu
PrepArgs prep_args(WinState *ws, double h0, double h1, int order);
size_t push_tile_bytes(int order);
long long push_batch_smem_limit();
// prep + push + post + bounds of a batch of FP64 members: one push launch per
// shape order present, the CTAs (grid in total) shared out by particle count.
// parts: 1 = the per-member preparation, 2 = the per-member bookkeeping after.
void launch_push_batch(const PushGroup *groups, int ngroups, int m, int grid, const PrepArgs *prep, cudaStream_t s,
                       int parts = 3);
void launch_bbox_next(const double *x, const double *y, const double *px, const double *py, long long n,
                      double half, int pending, WinState *ws, cudaStream_t s);
void launch_push_prep(WinState *ws, double h0, double h1, int order, cudaStream_t s);
void launch_push(const PushArgs &a, int order, int grid, cudaStream_t s);
void launch_global_bounds(WinState *ws, double h0, double h1, cudaStream_t s);
void launch_drift(double *x, double *y, const double *px, const double *py, long long n, double full,
                  cudaStream_t s);
void launch_gather(int order, int comp, const double *patch, int nx, double o0, double o1, double h0,
                   double h1, const double *x, const double *y, long long n, double *out, cudaStream_t s);
void launch_deposit(int order, int comp, const double *ox, const double *oy, const double *x,
                    const double *y, const double *q, long long n, double org0, double org1, double h0,
                    double h1, double dt, int i0, int j0, int ni, int nj, unsigned long long *acc,
                    double scale, int *err, cudaStream_t s);  // err: 2 ints (crossings, dropped)
void launch_fixed_to_double(const unsigned long long *acc, double *out, long long n, double inv,
                            cudaStream_t s);
// fields.cu (instantiated for T = double and T = float)
template <class T> void launch_half_h(FieldArgsT<T> a, cudaStream_t s);
template <class T> void launch_update_e(FieldArgsT<T> a, int comp, cudaStream_t s);
template <class T> void launch_exchange(FieldArgsT<T> a, int which, cudaStream_t s);
template <class T> void launch_copy_to_window(FieldArgsT<T> a, cudaStream_t s);
template <class T> void launch_check_window(FieldArgsT<T> a, cudaStream_t s);
template <class T> void launch_move(FieldArgsT<T> a, T *scratch, double h0, double h1, cudaStream_t s);
template <class T> void launch_reset_outside(FieldArgsT<T> a, const int *cutidx, cudaStream_t s);
// sets the block ranges of a sub-step; returns its block count
template <class T> int sub_grid(FieldArgsT<T> &a);
int exchange_count(int L0, int L1, int which);
template <class T>
void launch_half_h_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, cudaStream_t s);
template <class T>
void launch_update_e_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, int comp,
                           cudaStream_t s);
template <class T>
void launch_exchange_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, int which,
                           cudaStream_t s);
template <class T> void launch_move_batch(const MoveArgs<T> *args, int m, cudaStream_t s);
// The fused static sweep of one time step (fields.cu): a's static planes are
// the source set, dst the destination set (Ex, Ey, Hx, Hy); a carries the
// window, its first push's current and that component's acc_inv.  kind: the
// cell-kind map (static storage layout, kpitch bytes per row, a multiple of
// 16); z: 4 scratch planes of zpitch >= L0 + 6 by zrows >= L1 + 7 elements;
// spin: polls of a tile's staging wait.  The window fix-up runs on s2
// between the events fork (recorded on s) and join (s waits for it).
// Returns kOk, or kErrArg / kErrCuda (tensor-map set-up) before anything is
// launched.
template <class T>
int launch_yee_fused(const FieldArgsT<T> &a, const PlaneT<T> *dst, const uint8_t *kind, int kpitch,
                     const int *cutidx, T *z, int zpitch, int zrows, long long spin, cudaStream_t s, cudaStream_t s2,
                     cudaEvent_t fork, cudaEvent_t join);
// The window's Ey sub-step after the second push, with its strip exchange.
template <class T> void launch_window_ey(const FieldArgsT<T> &a, cudaStream_t s);
// The fused sweep of a batch of members as one persistent launch over a work
// queue: yee_batch_bytes(0 / 1) is the size of one member's entry in the tile
// / fix-up table, yee_batch_entry fills a member's entries (host memory; the
// arguments as for launch_yee_fused) and its tile count, launch_yee_batch
// resets the queue counter and launches over the device tables (tpre: first
// tile of every member, m + 1 entries).  Both return kOk, or kErrArg / kErrCuda
// before anything is launched.
template <class T> size_t yee_batch_bytes(int which);
template <class T>
int yee_batch_entry(const FieldArgsT<T> &a, const PlaneT<T> *dst, const uint8_t *kind, int kpitch, const int *cutidx,
                    T *z, int zpitch, int zrows, long long spin, void *tile_out, void *fix_out, int *ntiles);
template <class T>
int launch_yee_batch(const void *targs, const void *fix, const int *tpre, int m, unsigned *queue, cudaStream_t s);
template <class T>
void launch_window_ey_batch(const FieldArgsT<T> *args, const int *bpre, int m, int nblocks, cudaStream_t s);
void launch_build_kind(const uint8_t *mask, const int *cutidx, int Nx, int Ny, uint8_t *kind, int kpitch,
                       cudaStream_t s);
// geometry.cu
int build_geometry(const BendDev &b, uint8_t *d_mask, CutCellDev **d_cells, int *ncells, int **d_cutidx,
                   cudaStream_t s);
// diag.cu
void launch_moments(const double *x, const double *y, const double *px, const double *py, long long n,
                    double half, int pending, double *part, double *mean, double *out, cudaStream_t s);
// Field energy sums over the static mesh (and the window, replacing the points
// it covers): out2 = {sum(Ex^2 + Ey^2), sum((Hzx + Hzy)^2)} x area; part holds
// 2 doubles per block of the moments grid.
// Fields along the centroid line over static columns i0 .. i0 + n - 1 (7 values per sample).
template <class T>
void launch_line_fields(int order, const T *Ex, const T *Ey, const T *Hx, const T *Hy, int pitch, int Nx, int Ny,
                        const T *win, int wpitch, const WinState *ws, int with_current, double org0, double org1,
                        double h0, double h1, const double *mean, long long i0, int n, double *out, cudaStream_t s);
template <class T>
void launch_field_energy(const T *Ex, const T *Ey, const T *Hx, const T *Hy, int pitch, int Nx, int Ny,
                         const T *win, int wpitch, const WinState *ws, int with_window, double area, double *part,
                         double *out, cudaStream_t s);
size_t moments_scratch_doubles();
template <class T>
void launch_wake(const WinState *ws, const T *mEx, const T *mEy, int wpitch, int L0, double h0, double h1,
                 const double *mean, double *out, cudaStream_t s);
void launch_charge_diff(int order, const double *ox, const double *oy, const double *x, const double *y,
                        const double *q, long long n, double org0, double org1, double h0, double h1,
                        int i0, int j0, int ni, int nj, unsigned long long *acc, double scale,
                        int *dropped, cudaStream_t s);

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

// --- FP32 mode (particles32.cu) -------------------------------------------
// Positions are FP32 offsets from an FP64 cell origin: the static-mesh cell
// (i, j) packed as i | j << 16 and the offset inside it in cells, [0, 1).
// Momenta are FP32 deviations from an FP64 reference momentum P (the mean
// at load): at gamma ~ 1000 a bare FP32 momentum has an ulp of 6e-5, above
// the per-step kicks, while the deviations stay below ~1.
struct Bunch32 {
  int *cell;
  float *ox, *oy;
  float *dpx, *dpy;
  float *q;
  long long n;
};

// FP32-mode reference momentum and drift constants, rounded once from FP64:
// P, 1 + |P|^2 and 0.5 c dt / h (cells per half step per unit beta).
struct Ref32 {
  float P0, P1, G2, kh0, kh1;
};

struct Push32Args {
  Bunch32 b;
  WinState *ws;
  const float *mEx, *mEy, *mHx, *mHy;  // window planes, pitch wpitch
  int wpitch;
  unsigned long long *acc;             // L0 * L1 fixed-point flux (flux32.cuh) for jcomp
  double acc_scale;                    // fixed-point units per unit of charge
  int jcomp, pending;
  Ref32 R;
  float f1, f2;                        // 0.5 c dt q/m and f1 c
  double org0, org1, h0, h1;           // static mesh origin and spacing (bend frame)
  double bz, Lb, hw, chh, shh, bwidth; // hard-edge dipole
  // start position of every particle's move (CSRST_FLAG_KEEP_OLD), or null:
  // old cell, offsets from it
  int *old_cell;
  float *old_o0, *old_o1;
};

int launch_push32(const Push32Args &a, int order, cudaStream_t s);
long long push32_batch_smem_limit();
void launch_push32_batch(const PushGroup *groups, int ngroups, int m, int grid, const PrepArgs *prep,
                         cudaStream_t s, int parts = 3);
void launch_prep32(WinState *ws, int order, cudaStream_t s);
// After a push: swap the box sets, the deposit bounds, and the next push's
// gather-patch set-up when prep_next (nothing moves the particles or the
// window before that push).
void launch_after32(WinState *ws, int prep_next, cudaStream_t s);
void launch_bbox32(const Bunch32 &b, const Ref32 &R, int pending, WinState *ws, cudaStream_t s);
// R += dt c v / h: kd = the drift's dt c / h per axis (Ref32.kh replaced)
void launch_drift32(const Bunch32 &b, const Ref32 &R, float kd0, float kd1, cudaStream_t s);
void launch_from64(const double *x, const double *y, const double *px, const double *py, const double *q,
                   long long n, double org0, double org1, double h0, double h1, double P0, double P1,
                   const Bunch32 &b, cudaStream_t s);
// pending > 0: the stored positions still owe the drift by -kh (cells)
void launch_to64(const Bunch32 &b, const Ref32 &R, double P0, double P1, int pending, double org0, double org1,
                 double h0, double h1, double *x, double *y, double *px, double *py, cudaStream_t s);
// Stand-alone FP32-mode deposit (csrst_flux32): n moves from (cell0, a) to
// (cell1, b), integer flux of component comp and (if drho) the integer charge
// change into dense ni x nj patches at static-mesh index (i0, j0); err[0]:
// crossing overflow, err[1]: a non-zero contribution fell outside the patch.
void launch_flux32(int order, int comp, const int *cell0, const float *a0, const float *a1, const int *cell1,
                   const float *b0, const float *b1, const float *q, long long n, double scale, int i0, int j0,
                   int ni, int nj, unsigned long long *F, unsigned long long *drho, int *err, cudaStream_t s);
void launch_psum(const double *px, const double *py, long long n, double *part, double *out2,
                 cudaStream_t s);
// Plane copies between FP64 and FP32 (rows x cols elements, pitches in elements).
void launch_d2f(const double *src, int spitch, float *dst, int dpitch, int rows, int cols, cudaStream_t s);
void launch_f2d(const float *src, int spitch, double *dst, int dpitch, int rows, int cols, cudaStream_t s);

}  // namespace csrst
