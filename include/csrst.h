/* C ABI of the B200 CSRST per-time-step PIC loop (libcsrst_gpu.so).
 *
 * The reference (kreischtauf/CSRST) has no FFI: its boundary is the C++
 * classes TETMSolver, PartBunch and ScatterGatherImpl over IPPL fields.
 * Each entry point below names the reference interface it replaces.  The
 * C++ facades in include/csrst/ keep those class shapes on top of this ABI.
 *
 * Conventions
 *  - Every call returns an int status: 0 on success, a negative CSRST_E_*
 *    code on failure, a positive CSRST_W_* code when the call succeeded with
 *    a warning; csrst_get_error() returns the message of the last failure or
 *    warning.
 *  - Host buffers are copied; device memory is owned by the handle.
 *  - One handle per thread.  A handle is bound to one device and one CUDA
 *    stream; calls are asynchronous on that stream except the ones that
 *    return host data, which synchronise it.
 *  - Arrays of the static mesh are Nx*Ny doubles, x fastest, no guard cells.
 *    Window arrays are (L0+2)*(L1+2) doubles including the one-cell guard ring.
 */
#ifndef CSRST_H
#define CSRST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CSRST_OK 0
#define CSRST_E_ARG (-1)           /* invalid argument */
#define CSRST_E_CUDA (-2)          /* CUDA runtime error or no device */
#define CSRST_E_GEOMETRY (-3)      /* bend geometry where the reference asserts */
#define CSRST_E_NO_PARTICLES (-4)  /* the call needs a loaded bunch */
#define CSRST_E_WINDOW_FIT (-5)    /* bunch no longer fits the window (moveMesh PAssert) */
#define CSRST_E_WINDOW_MOVE (-6)   /* window would move by other than 0/1 cell in x, -1..1 in y */
#define CSRST_E_CROSSINGS (-7)     /* a particle crossed more cell borders than one push allows */
#define CSRST_E_WINDOW_WALL (-8)   /* window or its ring touches a non-inside cell */
#define CSRST_E_IO (-9)            /* checkpoint file could not be written or read */
#define CSRST_E_STAGING (-10)      /* a field tile's staging copy did not arrive (bounded wait gave up) */
#define CSRST_W_OUTSIDE 1          /* warning: contributions outside the caller's patch were dropped */

typedef struct csrst_handle csrst_handle;

/* csrst_config.flags */
#define CSRST_FLAG_KEEP_OLD 1  /* keep oldR of every push for csrst_get_old_positions */
#define CSRST_FLAG_FP32 2      /* FP32 mode: FP32 fields, gather, kick, drifts and positions (FP32
                                * offsets from FP64 cell origins; momenta as FP32 deviations from an
                                * FP64 reference momentum) and FP32 current path integral with exact
                                * integer charge conservation (csrst_flux32).  No reference
                                * counterpart; checked against the FP64 path to a tolerance. */
#define CSRST_FLAG_SUBSTEP_FIELDS 4 /* one launch per field sub-step instead of the fused static
                                * sweep (same results, bit for bit; the sweep is also off while
                                * absorbing layers are set or the handle is in an ensemble) */

/* Run set-up.  Mirrors the command line of src/main.cpp:111-136 for the
 * parts the time step uses.  shape_order: 0 = IntCIC (ZerothOrderShapeFunction),
 * 1 = IntS1 / TSC (FirstOrderShapeFunction), 2 = IntS2 (SecondOrderShapeFunction). */
typedef struct {
  int Nx, Ny;                 /* static mesh vertices per direction (-x, -y) */
  int shape_order;
  int flags;                  /* CSRST_FLAG_* bits, 0 = the FP64 path */
  double length_before;       /* drift before the bend [m] (--lengthbefore) */
  double length_after;        /* drift after the bend [m] (-l) */
  double width;               /* pipe width [m] (-w) */
  double phi_deg;             /* bending angle [deg] (-P) */
  double ekin_mev;            /* kinetic energy [MeV] (-E) */
  double bz;                  /* dipole field [T] (-B) */
  double dt;                  /* time step [s]; <= 0 selects hx / c (main.cpp:187) */
  double charge_mass;         /* charge-to-mass ratio of PartBunch (main.cpp:223: -1e-9 / m_e[GeV]) */
} csrst_config;

/* Creates the handle on the current CUDA device: bend geometry, inside mask
 * and cut-cell list (Bend::Init + SCBoundaryCondition ctor, main.cpp:168-197),
 * zero static fields. */
int csrst_create(const csrst_config *cfg, csrst_handle **out);
int csrst_destroy(csrst_handle *h);
/* Message of the last failed call on this handle (or of csrst_create when h is NULL). */
int csrst_get_error(const csrst_handle *h, char *buf, size_t len);
/* CUDA stream of the handle (a cudaStream_t). */
void *csrst_stream(csrst_handle *h);
int csrst_sync(csrst_handle *h);

/* Geometry: info8 = hx, hy, origin x, origin y, dt, fixed-point scale of the
 * current deposit (FP32 mode: of the flux, csrst_flux32), number of cut cells, window pitch.  Replaces Bend::Init /
 * getInsideMask / SCBoundaryCondition::getBoundaryCells (Bend.cpp:85-124,
 * SCBoundaryCondition.hh:433-441). */
int csrst_get_info(csrst_handle *h, double *info8);
/* inside: Nx*Ny bytes; cells: 7 doubles per cut cell (i, j, lambda0, lambda1,
 * area, lambdaToNeighbours0, lambdaToNeighbours1), at most max_cells. */
int csrst_get_geometry(csrst_handle *h, uint8_t *inside, double *cells, long max_cells, long *ncells);

/* Static mesh fields (EFD components 0/1, HFD components 0/1). */
int csrst_set_static_fields(csrst_handle *h, const double *ex, const double *ey,
                            const double *hzx, const double *hzy);
int csrst_get_static_fields(csrst_handle *h, double *ex, double *ey, double *hzx, double *hzy);
/* SCBoundaryCondition::resetOutsideDomain (SCBoundaryCondition.hh:163-195). */
int csrst_reset_outside(csrst_handle *h);

/* Loads the bunch (PartBunch ctor + sortParticles, PartBunch.cpp:48-150,
 * :1817-1844), opens the moving window around it (main.cpp:198-217) and
 * fills it from the static mesh (copyFields + exchangeBoundaries,
 * main.cpp:335-342).  q: charge per macro-particle [C]. */
int csrst_load_particles(csrst_handle *h, const double *x, const double *y, const double *px,
                         const double *py, const double *q, size_t n);
/* Initial fields of the loaded bunch (main.cpp:232-248): the three boosted
 * electrostatic solves of PoissonSolver::computeField (PoissonSolver.cpp:85-201)
 * on the matrix of cutoffStencil (:678-766) fill Ey, Hz and Ex of the static
 * mesh (fillFields, :441-507), then SCBoundaryCondition::resetOutsideDomain
 * runs and the window is refilled.  Multigrid-preconditioned CG in FP64 on the
 * GPU replaces Trilinos ML + BlockCG.  tol_first / tol_rest: relative residual
 * of the first solve (main.cpp:94, 1e-12) and of the other two (1e-6);
 * max_iter per solve (main.cpp:93, 500).  report8 (may be NULL): gamma,
 * iterations and relative residual of each solve, multigrid levels. */
int csrst_initial_fields(csrst_handle *h, double tol_first, double tol_rest, int max_iter, double *report8);
/* Current bunch in the handle's (cell-sorted) order. */
int csrst_get_particles(csrst_handle *h, double *x, double *y, double *px, double *py);
/* oldR of the last push (PartBunch::oldR). */
int csrst_get_old_positions(csrst_handle *h, double *ox, double *oy);
/* Window: w4 = position (ddim.first) x, y, size L0, L1; origin2; gb4 = last
 * deposit's particle bounds in window cells (PartBunch::getGlobalBounds). */
int csrst_get_window(csrst_handle *h, int *w4, double *origin2, int *gb4);
/* which: 0 Ex, 1 Ey, 2 Hzx, 3 Hzy, 4 Jx, 5 Jy of the window, incl. guards. */
int csrst_get_window_field(csrst_handle *h, int which, double *out);

/* Absorbing layers at the two open ends of the pipe.  The reference computes
 * PML conductivities in Bend::calculatePMLCoefficients (Bend.cpp:355-425)
 * but zeroes them in TETMSolver::initMaps (TETMSolver.cpp:59-63) and never
 * uses them: its domain ends are PEC walls.  Off by default here too, so
 * that the loop matches the reference; csrst_set_pml turns on a
 * convolutional PML (kappa = 1) over `width` cells before the entry plane of
 * the first straight section and the end plane of the second, each layer
 * ending 2 cells before its end wall (conformal cut cells of a slanted wall
 * next to a strongly damped cell made the update unstable).  Graded
 * sigma = smax (depth / width)^order along the pipe axis, split into its x
 * and y parts, with smax = -(order + 1) eps0 c ln(reflection) / (2 width hx)
 * (the reflection of a normally incident plane wave in the continuum).  The
 * reference's defaults are width 10, order 4, reflection exp(-16)
 * (Bend.cpp:28-32).  width 0 turns the layers off.  Inside cells only (the
 * cut cells at the pipe walls keep their conformal update); a window that
 * touches a layer is an error (CSRST_E_WINDOW_WALL).  Call it before
 * stepping (it drops the captured step) and before creating an ensemble of
 * the handle; the layers' convolution state starts at zero and is not part
 * of a checkpoint (call it again after a restart). */
int csrst_set_pml(csrst_handle *h, int width, int order, double reflection);
/* Number of layer cells, and per static-mesh row the columns [lo, hi) that
 * the regular update keeps (rows2: 2 * Ny ints, may be NULL). */
int csrst_get_pml(csrst_handle *h, int *ncells, int *rows2);

/* PartBunch::push_particles(mmE, mmH, mmJ, dt, Jcomp) (PartBunch.cpp:215-519). */
int csrst_push(csrst_handle *h, int jcomp);
/* PartBunch::drift_particles(dt) (PartBunch.cpp:179-187). */
int csrst_drift(csrst_handle *h, double dt);
/* Field sub-steps of TETMSolver::updateField_firstStep/secondStep, each with
 * its strip exchange and cut-cell correction (TETMSolver.hh:142-206, :241-261). */
int csrst_half_h(csrst_handle *h);
int csrst_update_e(csrst_handle *h, int comp);
/* moveMesh (main.cpp:562-652). */
int csrst_move_window(csrst_handle *h);
/* TETMSolver::updateField_firstStep / updateField_secondStep (TETMSolver.hh:110-266). */
int csrst_step_first(csrst_handle *h);
int csrst_step_second(csrst_handle *h);
/* nsteps iterations of the main loop body (main.cpp:390-506): first step,
 * second step, window move.  Captured as a CUDA graph and replayed.  The
 * static mesh's four sub-steps run as one fused sweep from one plane set into
 * another (the sets swap every step; every read and write of the fields goes
 * to the current set), bit for bit what the sub-step calls above give. */
int csrst_step(csrst_handle *h, int nsteps);
/* One step as csrst_step takes it (same kernels, launched eagerly) with CUDA
 * events between its kernel groups; waits for it and returns the device
 * times in ms4 [ms]: both pushes, the field work (the fused sweep, or the
 * four sub-steps with their exchanges, and the window's Ey), the window move,
 * and the whole step. */
int csrst_step_timed(csrst_handle *h, double *ms4);
/* Polls a fused-sweep tile makes in its staging wait (the TMA copies of its
 * fields) before it gives up, writes nothing and reports CSRST_E_STAGING at
 * the next synchronising call; for sweeps recorded or tabled after this call
 * (a new handle's first steps, an ensemble built after it).  polls == 0
 * restores the default, 2^22.  polls < 0 exercises that path: every staging
 * wait is then on a barrier that nothing completes, and gives up after
 * -polls polls (the tile still waits for its real copies before it ends). */
int csrst_set_staging_wait_limit(long long polls);
/* A handle's bunch arrays and the temporaries of csrst_load_particles come
 * from a stream-ordered memory pool the library keeps per device: memory a
 * destroyed handle or a reload frees stays in the pool for the next load
 * (no device-wide waits for cudaMalloc / cudaFree).  This returns the
 * pool's unused memory of the current device to the driver. */
int csrst_release_memory(void);

/* Batched ensemble (no reference counterpart: the reference runs one bunch
 * per job).  Independent members, each a loaded handle with its own mesh,
 * window, shape order and bunch size, all in the same precision mode, are
 * stepped together: every phase of the time step is one launch over all
 * members and the whole step is one CUDA graph.  Each member's state after a
 * batched step is bitwise the state its own csrst_step would give.  The
 * member handles stay valid for reads between ensemble steps; reloading a
 * member invalidates the ensemble.  Destroy the ensemble before its members;
 * while it exists their own steps use the sub-step kernels. */
typedef struct csrst_ensemble csrst_ensemble;
int csrst_ensemble_create(csrst_handle *const *members, int m, csrst_ensemble **out);
int csrst_ensemble_destroy(csrst_ensemble *e);
int csrst_ensemble_get_error(const csrst_ensemble *e, char *buf, size_t len);
/* CUDA stream of the ensemble (a cudaStream_t). */
void *csrst_ensemble_stream(csrst_ensemble *e);
int csrst_ensemble_step(csrst_ensemble *e, int nsteps);
/* Waits for the ensemble; returns the first member's sticky error (its index in *bad_member). */
int csrst_ensemble_sync(csrst_ensemble *e, int *bad_member);
/* Launch shapes: CTAs of the batched push (0 = two per SM), the field path
 * (tx = ty = 0: the fused static sweep, all members' tiles and window
 * fix-ups from one work queue in one persistent launch per step, the
 * default; else one launch per sub-step with static-sweep tiles of tx x ty,
 * tx * ty = 256) and the number of parts the members are split into, which
 * step side by side on their own streams.  Results do not depend on them. */
int csrst_ensemble_set_shape(csrst_ensemble *e, int push_ctas, int tx, int ty, int parts);
/* Autotuner: times `steps` steps for each candidate shape and keeps the
 * fastest; the timed steps are real steps of the members.  Candidates: push
 * CTAs {4, 16, 32} per SM x field path {fused, 32 x 8, 128 x 2} x parts
 * {1, 2, 4}.  report: rows of (push_ctas, tx, ty, parts, ms per step). */
int csrst_ensemble_tune(csrst_ensemble *e, int steps, double *report, int max_rows, int *nrows);

/* BF16 tensor-core GEMM of the wake surrogate (no reference counterpart):
 * C[M, N] = alpha * A[M, K] . B[N, K]^T with FP32 accumulation, A and B
 * K-major BF16 device matrices (leading dimensions lda, ldb in elements,
 * multiples of 8; K a multiple of 64; N a multiple of 16), `batch` of them
 * stride_a / stride_b apart.  The epilogue adds bias[n] and the residual,
 * keeps the pre-activation, applies GELU and writes FP32 and/or BF16 through
 * the index map below.  *err (device int) is set if a tensor-core wait gave up. */
typedef struct {
  float alpha;
  int act;                            /* 0 none, 1 GELU (erf form), after bias and residual */
  int accumulate;                     /* out32 += value */
  int md, nd;                         /* index-map divisors */
  long long sb, sm0, sm1, sn0, sn1;   /* index = z*sb + (m/md)*sm0 + (m%md)*sm1 + (n/nd)*sn0 + (n%nd)*sn1 */
  const float *bias;                  /* per column n, or NULL */
  const float *res;                   /* residual under the index map, or NULL */
  float *pre;                         /* pre-activation (FP32) under the index map, or NULL */
  float *out32;                       /* FP32 output, or NULL */
  void *out16;                        /* BF16 output, or NULL */
  void *out16t;                       /* second BF16 output under its own map, or NULL */
  int tmd, tnd;
  long long tb, tm0, tm1, tn0, tn1;
  const float *bias_m;                /* per row m, or NULL (added after bias[n]) */
} csrst_gemm_epilogue;
int csrst_gemm_bf16(const void *A, long long lda, long long stride_a, const void *B, long long ldb,
                    long long stride_b, int M, int N, int K, int batch, const csrst_gemm_epilogue *ep, int *err,
                    void *stream);
/* The same with an MN-major A when a_mn_major: element (m, k) of batch z at
 * A[z * stride_a + k * lda + m] (K rows of M contiguous elements; lda >= M, a
 * multiple of 8); a_mn_major == 0 is csrst_gemm_bf16. */
int csrst_gemm_bf16_ex(const void *A, long long lda, long long stride_a, int a_mn_major, const void *B,
                       long long ldb, long long stride_b, int M, int N, int K, int batch,
                       const csrst_gemm_epilogue *ep, int *err, void *stream);
/* Polls each mbarrier wait of the GEMM makes before it gives up and sets *err = 1 (for all later
 * GEMM launches of the process; polls == 0 restores the default, 2^24).  A wait that gives up
 * ends every role of its CTA at its next wait; the kernel still waits, with the default bound,
 * for the copies and tensor-core work it issued, frees its TMEM and returns (*err = 2 if even
 * that wait gave up).  polls < 0 exercises that path: the epilogue's first wait of every GEMM
 * is then on a barrier that nothing completes, and gives up after -polls polls, before any
 * output is written. */
int csrst_gemm_set_wait_limit(long long polls);
/* The same over two K segments into one accumulator: C = A1 B1^T + A2 B2^T (K1, K2 multiples of 64), each
 * segment with its own pointers, leading dimensions and batch strides (a stride may be 0: shared operand). */
int csrst_gemm_bf16_dual(const void *A1, long long lda1, long long stride_a1, const void *B1, long long ldb1,
                         long long stride_b1, int K1, const void *A2, long long lda2, long long stride_a2,
                         const void *B2, long long ldb2, long long stride_b2, int K2, int M, int N, int batch,
                         const csrst_gemm_epilogue *ep, int *err, void *stream);

/* Checkpoint and restart (the restart dump read by LoadH5Part, src/Commands/LoadH5Part.cpp:60-321:
 * run attributes, fields, bunch R / oldR / P / Q), as a dependency-free binary file that holds
 * everything a time step reads: the configuration, step and time, the static-mesh planes, the
 * moving window (position, size, bookkeeping, its fields and fixed-point current) and the bunch in
 * the handle's own form (FP64 arrays, or the FP32 mode's offsets and momentum deviations).  A run
 * restored into a handle created with the same configuration continues bit for bit.  Files are
 * host-endian; the layout is versioned. */
int csrst_checkpoint_write(csrst_handle *h, const char *path, long long step, double time);
/* Particles of the loaded (or restored) bunch. */
int csrst_get_num_particles(csrst_handle *h, long long *n);
int csrst_checkpoint_read(csrst_handle *h, const char *path, long long *step, double *time);

/* Element-wise and reduction kernels of the surrogate's training and inference
 * (device pointers; BF16 arrays as void *).  No reference counterpart. */
/* [batch][rows][cols] -> [batch][cols][ldd] (ldd >= rows; columns rows .. ldd - 1 untouched) */
int csrst_nn_transpose_bf16(const void *src, void *dst, int batch, int rows, int cols, int ldd, void *stream);
/* the same for 32-bit elements (pairs of BF16 values kept together); 4-byte aligned pointers */
int csrst_nn_transpose_b32(const void *src, void *dst, int batch, int rows, int cols, int ldd, void *stream);
/* dx = dy * GELU'(pre) (erf form); dx32 and/or dx16 */
int csrst_nn_gelu_bwd(const float *dy, const float *pre, float *dx32, void *dx16, long long n, void *stream);
int csrst_nn_cast_bf16(const float *x, void *y, long long n, void *stream);
/* out[c] (+)= sum over rows of x[r][c] in a fixed order; part: ceil(rows/256)*cols floats of scratch */
int csrst_nn_colsum(const float *x, int rows, int cols, float *part, float *out, int accumulate, void *stream);
/* loss = mean (w_i (pred_i - target_i))^2 (w = 1 when weight is NULL); grad[(i/gd)*g0 + (i%gd)*g1] =
 * 2 w_i^2 (pred_i - target_i) / n (grad may be NULL); part: 256 doubles of scratch; loss: one device double */
int csrst_nn_mse(const float *pred, const float *target, const float *weight, long long n, float *grad, int gd,
                 long long g0, long long g1, double *part, double *loss, void *stream);
/* Adam with bias correction; the step counter *t and coef = {lr_t, 1 - b1^t, 1 - b2^t} live on the device:
 * adam_tick advances t and writes coef (cosine schedule from lr0 to lr_min over `total` steps) */
int csrst_nn_adam_tick(int *t, float *coef, float lr0, float lr_min, int total, float b1, float b2, void *stream);
int csrst_nn_adam(float *w, const float *g, float *m, float *v, long long n, const float *coef, float b1, float b2,
                  float eps, void *stream);
/* complex spectral weights Wr + i Wi [modes][ch][ch] -> real blocks Mk [modes][2ch][2ch] and their transposes */
int csrst_nn_spectral_pack(const float *wr, const float *wi, int modes, int ch, void *mk, void *mkt, void *stream);
int csrst_nn_spectral_unpack(const float *dmk, int modes, int ch, float *dwr, float *dwi, void *stream);

/* Beam moments (PartBunch::calcBeamParameters, PartBunch.cpp:584-657):
 * out18 = rmean2, pmean2, rrms2, prms2, eps_norm2, rmin2, rmax2, Ekin[MeV], dE, Dy, DDy. */
int csrst_diag_moments(csrst_handle *h, double *out18);
/* Field energy sums (CalcEnergyCommand, src/Commands/CalcEnergy.cpp:41-120): out2 = {sum of
 * Ex^2 + Ey^2, sum of (Hzx + Hzy)^2} over the static mesh's points times the cell area, with the
 * window's points replacing the ones they cover when with_window is set (needs a loaded bunch).
 * The reference's energy is 0.25 eps0 (E_now + E_last) + 0.5 mu0 H (csrst_b200.diagnostics). */
int csrst_diag_field_energy(csrst_handle *h, int with_window, double *out2);
/* Fields along the line through the bunch centroid in the direction of its mean momentum
 * (SaveEMFieldsCommand, src/Commands/SaveEMFields.cpp:34-189): one sample per static column from
 * 1.5 g0 - 0.5 g1 to 2 g1 - g0 (g0, g1 the columns holding the bunch's extremes), gathered with the
 * run's shape order from the static mesh with the window's values over the points it covers.
 * out[7 k ..] = signed distance from the centroid, E along and across the momentum, Hz, J along
 * the momentum, x, y.  with_current: J from the window (the reference copies it on plot steps
 * only; otherwise its static J, zero in the loop, gives 0).  *count receives the number of
 * samples; out = NULL returns only the count; cap < count is an error. */
int csrst_diag_line_fields(csrst_handle *h, int with_current, double *out, int cap, int *count);
/* Longitudinal field along the bunch axis at window columns 2 .. L0-3
 * (IntegrateElongCommand::execute, IntegrateElong.cpp:38-89); NaN where the
 * sample lies outside the window.  n must be L0 - 4. */
int csrst_diag_wake(csrst_handle *h, double *out, int n);
/* The same into device memory, enqueued on the handle's stream without
 * waiting (for many members read at once): out_dev receives the L0 - 4
 * samples, meta_dev the window origin (x, y) and the bunch centroid (x, y). */
int csrst_diag_wake_async(csrst_handle *h, double *out_dev, int n, double *meta_dev);

/* ScatterGatherImpl<IntOp>::gather (ScatterGatherImpl.hh:27-47) on a dense
 * host patch (nx * ny, x fastest) with origin o and spacing hh; comp 0/1 =
 * edge component, 2 = cell-centred.  Runs on the current device. */
int csrst_gather(int order, int comp, const double *patch, int nx, int ny, const double *o2,
                 const double *hh2, const double *x, const double *y, size_t n, double *out);
/* ShapeFunction<IntOp>::getCurrentDensityBase{X,Y} (ShapeFunction.hh:173-204):
 * current of particles moving old -> new on a mesh with origin o2, spacing
 * hh2, into a dense (ni x nj) patch whose element (0,0) is mesh index
 * (i0, j0).  Accumulated in 64-bit fixed point with the given scale.  The
 * reference sizes its patch to hold every contribution (the particle box plus
 * getExtraMarginCurrent); here the caller chooses the patch, and a non-zero
 * contribution that falls outside it is dropped and reported by the return
 * value CSRST_W_OUTSIDE (J is still written).  csrst_charge_diff does the same. */
int csrst_deposit(int order, int comp, const double *ox, const double *oy, const double *x,
                  const double *y, const double *q, size_t n, const double *o2, const double *hh2,
                  double dt, int i0, int j0, int ni, int nj, double scale, double *J);
/* Charge difference rho(new) - rho(old) at vertices for the charge shape of
 * the same order (get*ChargeDensityDiffImpl), divided by the cell area.  The
 * fixed-point scale applies to the charge before the division: pick it from
 * the total |q| (e.g. the largest power of two with 4 sum|q| * scale < 2^62). */
int csrst_charge_diff(int order, const double *ox, const double *oy, const double *x,
                      const double *y, const double *q, size_t n, const double *o2,
                      const double *hh2, int i0, int j0, int ni, int nj, double scale, double *rho);

/* FP32 mode's charge-conserving deposit (no reference counterpart; the
 * push of a CSRST_FLAG_FP32 handle deposits with it).  n moves from start
 * cell0 + offset (a0, a1) (cells, any value) to end cell1 + offset (b0, b1)
 * (in [0, 1)), cells packed as i | j << 16 like the FP32 bunch, charge q.
 * F receives the integer flux of component comp (Fx = Jx dt hy / q, Fy =
 * Jy dt hx / q, times scale * q) in a dense (ni x nj) patch at mesh index
 * (i0, j0), at the elements of Jx(i, j) / Jy(i, j); drho (may be NULL) the
 * integer charge change rho(end) - rho(start) in the same units at the
 * vertices.  drho + div F = 0 holds exactly in integers:
 *   drho(i,j) + Fx(i,j) - Fx(i-1,j) + Fy(i,j) - Fy(i,j-1) = 0.
 * The path integral of the reference's current (Zeroth/First/Second-
 * OrderShapeFunction) runs in FP32, the end points' charge weights in FP64.
 * Host arrays.  Returns CSRST_E_CROSSINGS for a move of more than one cell
 * on an axis, CSRST_W_OUTSIDE when contributions fell outside the patch. */
int csrst_flux32(int order, int comp, const int *cell0, const float *a0, const float *a1, const int *cell1,
                 const float *b0, const float *b1, const float *q, size_t n, double scale, int i0, int j0, int ni,
                 int nj, long long *F, long long *drho);
/* Raw FP32-mode bunch of a CSRST_FLAG_FP32 handle (host arrays, NULL to skip):
 * which = 0: packed cells, offsets, momentum deviations and charges of the
 * bunch as stored; which = 1: the packed cell and offsets of the start of
 * each particle's last move (CSRST_FLAG_KEEP_OLD; d0, d1, q must be NULL).
 * The reference momentum is csrst_get_particles' momentum minus d. */
int csrst_get_bunch32(csrst_handle *h, int which, int *cell, float *o0, float *o1, float *d0, float *d1, float *q);

/* Allocation-free csrst_deposit, for callers that cannot let a library
 * allocate device memory: a host framework that owns all device memory
 * through its own pool and budget, or a time loop that must not stall the
 * device (cudaMalloc and cudaFree synchronise it).  No counterpart in the
 * reference, which deposits on the CPU.
 *  - ox, oy, x, y, q and J are DEVICE pointers owned by the caller; o2 and
 *    hh2 are host arrays of 2 doubles.  Same result as csrst_deposit.
 *  - The fixed-point accumulator is a file-scope __device__ array of 2^20
 *    cells (8 MiB) that every GPU which loads the library holds until exit;
 *    ni * nj above 2^20 is rejected with CSRST_E_ARG.  Nothing is allocated
 *    or freed (no cudaMalloc, cudaFree or allocating library call).
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) and keeps it for the life of the process.  After
 *    cudaDeviceReset the kept address is stale: calls after a reset are not
 *    supported.
 *  - Runs on `stream` (a cudaStream_t, NULL = default stream) and waits for
 *    that stream before it returns, because it reads the crossing and
 *    dropped-contribution flags back; so it cannot be called while a stream
 *    is being captured into a graph.  All calls share the one array per
 *    device, so calls that overlap on the GPU (other threads or streams) race.
 *  - Same return values as csrst_deposit (CSRST_E_CROSSINGS, CSRST_W_OUTSIDE);
 *    csrst_get_error(NULL) gives the message of a failure or warning. */
int csrst_deposit_noalloc(int order, int comp, const double *ox, const double *oy, const double *x,
                          const double *y, const double *q, size_t n, const double *o2,
                          const double *hh2, double dt, int i0, int j0, int ni, int nj, double scale,
                          double *J, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CSRST_H */
