// C ABI of libcsrst_gpu.so (declared in include/csrst.h): the handle, device
// memory, the order of kernel launches for one time step and its CUDA graph.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/csrst.h"
#include "bunch32.cuh"
#include "kernels.cuh"

namespace csrst {

__global__ void k_gather_perm(const long long *perm, long long n, const double *a, double *b) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[perm[i]];
}
__global__ void k_sort_keys(const double *x, const double *y, long long n, const WinState *ws,
                            double h1, unsigned long long *kx, long long *idx) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  kx[i] = (unsigned long long)dbl_ord(x[i]) ^ 0x8000000000000000ull;
  idx[i] = i;
}
// y slice of the window (PartBunch::sortParticles, PartBunch.cpp:1826-1829)
__global__ void k_slice_keys(const double *y, const long long *idx, long long n, const WinState *ws,
                             double h1, unsigned int *ks) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double mn1 = ord_dbl(ws->bb[ws->cur][1]);
  const int lp2 = (int)floor((mn1 - ws->mo1) / h1);
  ks[i] = (unsigned int)((int)floor((y[idx[i]] - ws->mo1) / h1) - lp2);
}
inline double bits_to_double(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}
// Input check of a bunch on the device: out[0] = the first index whose
// values are not all finite or (in FP32 mode, whose cells are 16-bit static
// mesh indices) whose position lies off the static mesh, ~0 if none; out[1] =
// max |q| as the bits of a non-negative double.  out starts as {~0, 0}.
__global__ void k_check_bunch(const double *x, const double *y, const double *px, const double *py,
                              const double *q, long long n, int on_mesh, double org0, double org1, double h0,
                              double h1, int Nx, int Ny, unsigned long long *out) {
  unsigned long long bad = ~0ull, qm = 0ull;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    bool ok = isfinite(x[i]) && isfinite(y[i]) && isfinite(px[i]) && isfinite(py[i]) && isfinite(q[i]);
    if (ok) {
      const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(q[i]));
      qm = b > qm ? b : qm;
      if (on_mesh) {
        const double a = (x[i] - org0) / h0, c = (y[i] - org1) / h1;
        ok = a >= 0 && a < Nx && c >= 0 && c < Ny;
      }
    }
    if (!ok && (unsigned long long)i < bad) bad = (unsigned long long)i;
  }
  if (bad != ~0ull) atomicMin(&out[0], bad);
  if (qm) atomicMax(&out[1], qm);
}
// FP32-mode positions (cell + offset) as FP64 positions.
__global__ void k_old32_to64(const int *cell, const float *o0, const float *o1, long long n, double org0, double org1,
                             double h0, double h1, double *x, double *y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cell[i];
  const int ci = c & 0xffff, cj = (int)((unsigned)c >> 16);
  x[i] = __dadd_rn(org0, __dmul_rn(__dadd_rn((double)ci, (double)o0[i]), h0));
  y[i] = __dadd_rn(org1, __dmul_rn(__dadd_rn((double)cj, (double)o1[i]), h1));
}
__global__ void k_acc_to_plane(const unsigned long long *acc, Plane p, int L0, int L1, double inv) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L0 * L1) return;
  p.at(k % L0, k / L0) = (double)(long long)acc[k] * inv;
}
__global__ void k_set_pending_old(const double *x, const double *y, const double *px, const double *py,
                                  long long n, double half, int pending, double *ox, double *oy) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = x[i], b = y[i];
  if (pending) {
    const double r = inv_gamma(px[i], py[i]);
    a = a + (-(half * px[i] * r));
    b = b + (-(half * py[i] * r));
  }
  ox[i] = a; oy[i] = b;
}

}  // namespace csrst

using namespace csrst;

namespace {

enum BBoxState { kBBInvalid, kBBValid, kBBValidIfPending };

static std::string g_create_error;

}  // namespace

struct csrst_handle {
  csrst_config cfg{};
  int order = 0;
  cudaStream_t s = nullptr;
  BendDev b{};
  double dt = 0, half = 0, chh = 0, shh = 0, bwidth = 0;
  int pitch = 0;
  double *Ex = nullptr, *Ey = nullptr, *Hx = nullptr, *Hy = nullptr;
  uint8_t *mask = nullptr;
  CutCellDev *cells = nullptr;
  int ncells = 0;
  int *cutidx = nullptr;
  // window
  int L0 = 0, L1 = 0, wpitch = 0;
  double *win = nullptr;  // 6 planes
  double *scratch = nullptr;
  unsigned long long *acc = nullptr;  // 2 * L0 * L1
  double acc_scale = 0;
  bool acc_fresh[2] = {false, false};
  WinState *ws = nullptr;
  // particles
  long long n = 0;
  double *x = nullptr, *y = nullptr, *px = nullptr, *py = nullptr, *q = nullptr;
  double *ox = nullptr, *oy = nullptr;
  bool pending = false;
  bool fresh = false;  // loaded, no push yet
  // FP32 mode: the last push's closing kernel set up the next push's gather
  // patch (prepped); the next push is to do so (prep_after)
  bool prepped = false, prep_after = false;
  BBoxState bb = kBBInvalid;
  int push_grid = 0;
  // diagnostics scratch
  double *dscratch = nullptr, *dmean = nullptr, *dout = nullptr;
  // graphs of one step: the fused sweep swaps the static plane sets every
  // step, so there is one graph per set that is current when it starts
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  bool graph_fused = false;   // the sweep the graphs were recorded with
  std::string err;
  // FP32 mode (CSRST_FLAG_FP32): FP32 static and window planes, FP32 bunch
  bool fp32 = false;
  Ref32 R32{};                // reference momentum and drift constants in FP32
  int *old_cell = nullptr;    // CSRST_FLAG_KEEP_OLD in FP32 mode: start of each particle's last move
  float *old_o0 = nullptr, *old_o1 = nullptr;
  int pitch32 = 0;
  float *Exf = nullptr, *Eyf = nullptr, *Hxf = nullptr, *Hyf = nullptr;
  float *winf = nullptr, *scratchf = nullptr;
  Bunch32 b32{};
  double P0 = 0, P1 = 0;      // reference momentum
  double kh0 = 0, kh1 = 0;    // 0.5 c dt / h
  double *d64 = nullptr;      // 4 n doubles: the bunch in FP64 for diagnostics and reads
  // absorbing layers at the open ends (csrst_set_pml), null when off
  PmlCellT<double> *pml = nullptr;
  PmlCellT<float> *pml32 = nullptr;
  int npml = 0;
  int2 *pml_rows = nullptr;
  void *psi = nullptr;        // the layers' convolution state, 4 per cell, field type
  // the fused field sweep: the other static plane set (a fused step reads the
  // current set and writes this one, then the two swap), the cell kinds in
  // the static storage layout, and the scratch of the fix-up around the window
  double *ExB = nullptr, *EyB = nullptr, *HxB = nullptr, *HyB = nullptr;
  float *ExfB = nullptr, *EyfB = nullptr, *HxfB = nullptr, *HyfB = nullptr;
  uint8_t *kind = nullptr;
  int kpitch = 0;
  void *zfix = nullptr;
  int zpitch = 0, zrows = 0;
  int par = 0;                // plane-set swaps so far, mod 2
  int ens_refs = 0;           // ensembles whose argument tables hold this handle's planes
  cudaEvent_t *tev = nullptr; // csrst_step_timed: 8 events around the step's kernel groups
  cudaStream_t s2 = nullptr;  // the fused sweep's window fix-up, beside its tiles
  cudaEvent_t fork = nullptr, join = nullptr;
};

// One part of a batch: its members' argument tables in device memory and the
// streams its launches go to (the two shape-order groups of a push run side
// by side on s and s2).
struct EnsPart {
  std::vector<csrst_handle *> mem;
  int m = 0;
  long long particles = 0;
  cudaStream_t s = nullptr, s2 = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr, end = nullptr;
  std::vector<PushGroup> groups[2];  // [jcomp], one per shape order
  std::vector<void *> blocks;        // device allocations of the push groups
  FieldArgs *f64[2] = {nullptr, nullptr};
  FieldArgsT<float> *f32[2] = {nullptr, nullptr};
  MoveArgs<double> *mv64 = nullptr;
  MoveArgs<float> *mv32 = nullptr;
  PrepArgs *prep = nullptr;
  int *bpre_sub = nullptr, *bpre_ex[3] = {nullptr, nullptr, nullptr};
  int nsub = 0, nex[3] = {0, 0, 0};
  int push_grid = 0;
  // the fused sweep (csrst_ensemble::fused): per plane-set parity p (p = 0:
  // the members' sets as current at build time), the tile and fix-up tables
  // reading the current set, the window-Ey (comp 1) and move arguments over
  // the set current after the sweep; the members' first tiles; the blocks of
  // the window-Ey launch; the work-queue counter
  void *ytile[2] = {nullptr, nullptr}, *yfix[2] = {nullptr, nullptr};
  void *fey[2] = {nullptr, nullptr}, *fmv[2] = {nullptr, nullptr};
  int *tpre = nullptr, *bpre_ey = nullptr;
  int ney = 0;
  unsigned *queue = nullptr;
};

// A batch of members stepped together: every phase of the time step is one
// launch per part for all its members; the parts run side by side on their
// own streams (so that one part's pushes overlap another's field sweeps),
// and the whole step is captured as one CUDA graph.
struct csrst_ensemble {
  std::vector<csrst_handle *> mem;
  int m = 0;
  bool fp32 = false;
  cudaStream_t s = nullptr;  // the ensemble's stream (graph launches, ordering with the members)
  cudaEvent_t done = nullptr, fork = nullptr;
  std::vector<EnsPart> parts;
  // launch shapes (set by csrst_ensemble_set_shape / csrst_ensemble_tune);
  // tx = ty = 0: the fused static sweep (one persistent launch per step)
  int push_grid = 0, tx = 0, ty = 0, nparts = 1;
  bool fused = false;        // the fused sweep is in use (shape and members allow it)
  int epar = 0;              // plane-set swaps of the fused sweep since the tables were built, mod 2
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // one step, per parity
  bool holds = false;        // the members' ens_refs count this ensemble
  std::string err;
};

namespace {

int fail(csrst_handle *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  else g_create_error = msg;
  return code;
}

}  // namespace

int csrst::set_global_error(int code, const char *msg) { return fail(nullptr, code, msg); }

namespace {

int cuda_fail(csrst_handle *h, cudaError_t e, const char *where) {
  return fail(h, CSRST_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call);    \
  } while (0)

Plane plane(double *p, int pitch) { return Plane{p, pitch}; }

Plane wplane(const csrst_handle *h, int k) {
  return Plane{h->win + (size_t)k * h->wpitch * (h->L1 + 2), h->wpitch};
}

FieldArgs field_args(csrst_handle *h, int comp) {
  FieldArgs a{};
  const size_t ps = (size_t)h->pitch * (h->b.Ny + 2);
  a.Ex = plane(h->Ex, h->pitch); a.Ey = plane(h->Ey, h->pitch);
  a.Hx = plane(h->Hx, h->pitch); a.Hy = plane(h->Hy, h->pitch);
  (void)ps;
  a.mask = h->mask;
  a.Nx = h->b.Nx; a.Ny = h->b.Ny;
  a.mEx = wplane(h, 0); a.mEy = wplane(h, 1); a.mHx = wplane(h, 2); a.mHy = wplane(h, 3);
  a.mJx = wplane(h, 4); a.mJy = wplane(h, 5);
  a.L0 = h->L0; a.L1 = h->L1;
  a.cells = h->cells; a.ncells = h->ncells;
  a.ws = h->ws;
  a.acc = h->acc ? h->acc + (size_t)(comp == 1 ? 1 : 0) * h->L0 * h->L1 : nullptr;
  const double h0 = h->b.hr0, h1 = h->b.hr1, dt = h->dt;
  // FP64 path: the accumulator holds J * scale; FP32 mode: the flux
  // F = J dt h_other / q in units of 1 / scale per unit charge (flux32.cuh)
  a.acc_inv = h->acc_scale > 0 ? (h->fp32 ? 1.0 / (h->acc_scale * dt * (comp == 1 ? h0 : h1)) : 1.0 / h->acc_scale)
                               : 0.0;
  // TETMSolver.hh:121-125 and TETMSolver.cpp:87-127
  const double etax = kC * dt / h0, etay = kC * dt / h1;
  const double Z0 = std::sqrt(kMu0 / kEps0);
  a.chx = 0.5 * etax / Z0; a.chy = 0.5 * etay / Z0;
  a.kex = etay * Z0; a.key = etax * Z0;
  a.dteps = kC * dt * Z0;
  a.mhx = -0.5 * (dt / (h0 * kMu0)); a.mhy = +0.5 * (dt / (h1 * kMu0));
  a.de = dt / kEps0;
  a.h0 = h0; a.h1 = h1;
  a.pml = h->pml; a.npml = h->npml; a.pml_rows = h->pml_rows;
  a.psi = static_cast<double *>(h->psi);
  return a;
}

PlaneT<float> wplane32(const csrst_handle *h, int k) {
  return PlaneT<float>{h->winf + (size_t)k * h->wpitch * (h->L1 + 2), h->wpitch};
}

// The same sub-step arguments for FP32 mode: FP32 planes, coefficients
// computed in FP64 and rounded once.
FieldArgsT<float> field_args32(csrst_handle *h, int comp) {
  const FieldArgs d = field_args(h, comp);
  FieldArgsT<float> a{};
  a.Ex = PlaneT<float>{h->Exf, h->pitch32}; a.Ey = PlaneT<float>{h->Eyf, h->pitch32};
  a.Hx = PlaneT<float>{h->Hxf, h->pitch32}; a.Hy = PlaneT<float>{h->Hyf, h->pitch32};
  a.mask = d.mask; a.Nx = d.Nx; a.Ny = d.Ny;
  if (h->winf) {
    a.mEx = wplane32(h, 0); a.mEy = wplane32(h, 1); a.mHx = wplane32(h, 2); a.mHy = wplane32(h, 3);
    a.mJx = wplane32(h, 4); a.mJy = wplane32(h, 5);
  }
  a.L0 = d.L0; a.L1 = d.L1; a.cells = d.cells; a.ncells = d.ncells; a.ws = d.ws; a.acc = d.acc;
  a.acc_inv = d.acc_inv;
  a.chx = (float)d.chx; a.chy = (float)d.chy; a.kex = (float)d.kex; a.key = (float)d.key;
  a.dteps = (float)d.dteps; a.mhx = (float)d.mhx; a.mhy = (float)d.mhy; a.de = (float)d.de;
  a.h0 = (float)d.h0; a.h1 = (float)d.h1;
  a.pml = h->pml32; a.npml = d.npml; a.pml_rows = d.pml_rows;
  a.psi = static_cast<float *>(h->psi);
  return a;
}

// Host copy of the Bend set-up (Bend ctor and Bend::Init, Bend.cpp:60-124).
void bend_setup(csrst_handle *h) {
  const csrst_config &c = h->cfg;
  BendDev &b = h->b;
  const double mass = 0.511e6, ekin = c.ekin_mev * 1e6;
  b.Nx = c.Nx; b.Ny = c.Ny; b.Lb = c.length_before; b.La = c.length_after; b.w = c.width;
  if (std::abs(c.bz) > 1e-8) {
    b.R = std::sqrt(ekin * ekin + 2. * ekin * mass) / (kC * std::abs(c.bz));
    b.phi = -c.bz / std::abs(c.bz) * std::abs(c.phi_deg) * kPi / 180.;
  } else {
    b.R = 9999999.9;
    b.phi = 0.0;
  }
  const double cosphi = std::cos(b.phi), sinphi = std::abs(std::sin(b.phi));
  double dl, dw;
  if (std::abs(c.bz) > 1e-8) {
    dl = (c.length_before + c.length_after * cosphi + (b.R + 0.5 * c.width) * sinphi);
    dw = ((b.R - 0.5 * c.width) * (1 - cosphi) + c.width + c.length_after * sinphi);
  } else {
    dl = c.length_after + c.length_before;
    dw = c.width;
  }
  b.hr0 = dl / (c.Nx - 2);
  b.hr1 = dw / (c.Ny - 2);
  if (c.bz <= 0.0) {
    b.org0 = 0 - b.hr0; b.org1 = (c.width - dw) - b.hr1;
    b.cen0 = c.length_before; b.cen1 = 0.5 * c.width - b.R;
  } else {
    b.org0 = -b.hr0; b.org1 = -b.hr1;
    b.cen0 = c.length_before; b.cen1 = 0.5 * c.width + b.R;
  }
  b.cphi = std::cos(b.phi);
  b.sphi = std::sin(b.phi);
  h->dt = c.dt > 0 ? c.dt : b.hr0 / kC;
  h->half = 0.5 * h->dt * kC;
  h->chh = std::cos(0.5 * b.phi);
  h->shh = std::sin(0.5 * b.phi);
  h->bwidth = 2 * b.R * std::abs(h->shh);
}

// Stream-ordered allocations from the library's own memory pool (one per
// device; memory freed into it stays there for the next allocation instead
// of going back to the driver at every synchronisation): the bunch arrays of
// a handle and the temporaries of a bunch upload, so that a reload, or a new
// handle after an old one, allocates and frees without device-wide waits.
cudaMemPool_t lib_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps p{};
    p.allocType = cudaMemAllocationTypePinned;
    p.location.type = cudaMemLocationTypeDevice;
    p.location.id = dev;
    cudaMemPool_t m = nullptr;
    if (cudaMemPoolCreate(&m, &p) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(m, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = m;
  }
  return pools[dev];
}

template <class P>
cudaError_t palloc(P **p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t m = lib_pool();
  if (!m) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, m, s);
}

void pfree(void *p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

void drop_graphs(csrst_handle *h) {
  for (cudaGraphExec_t &g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

void free_particles(csrst_handle *h) {
  // the bunch arrays come from the pool (palloc), freed in the handle's stream order
  for (double *p : {h->x, h->y, h->px, h->py, h->q, h->ox, h->oy}) pfree(p, h->s);
  h->x = h->y = h->px = h->py = h->q = h->ox = h->oy = nullptr;
  cudaFree(h->win); cudaFree(h->scratch); cudaFree(h->acc);
  h->win = h->scratch = nullptr; h->acc = nullptr;
  pfree(h->b32.cell, h->s); pfree(h->b32.ox, h->s); pfree(h->b32.oy, h->s); pfree(h->b32.dpx, h->s);
  pfree(h->b32.dpy, h->s); pfree(h->b32.q, h->s); pfree(h->d64, h->s);
  cudaFree(h->winf); cudaFree(h->scratchf);
  cudaFree(h->old_cell); cudaFree(h->old_o0); cudaFree(h->old_o1);
  h->old_cell = nullptr; h->old_o0 = h->old_o1 = nullptr;
  h->b32 = Bunch32{};
  h->winf = h->scratchf = nullptr;
  h->d64 = nullptr;
  cudaFree(h->zfix);
  h->zfix = nullptr;
  drop_graphs(h);
  h->n = 0;
}

int check_err(csrst_handle *h) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, &h->ws->err, sizeof(int), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  if (e) {
    const char *m = e == kErrWindowFit ? "bunch no longer fits the window"
                  : e == kErrWindowMove ? "window move out of range"
                  : e == kErrCrossings ? "too many cell-border crossings in one push"
                  : e == kErrWindowWall ? "window touches a non-inside cell"
                  : "device error";
    return fail(h, e, m);
  }
  return CSRST_OK;
}

PushArgs push_args(csrst_handle *h, int jcomp) {
  PushArgs a{};
  a.x = h->x; a.y = h->y; a.px = h->px; a.py = h->py; a.q = h->q; a.n = h->n;
  a.ws = h->ws;
  a.mEx = wplane(h, 0).p; a.mEy = wplane(h, 1).p; a.mHx = wplane(h, 2).p; a.mHy = wplane(h, 3).p;
  a.wpitch = h->wpitch;
  a.acc = h->acc + (size_t)jcomp * h->L0 * h->L1;
  a.acc_scale = h->acc_scale;
  a.jcomp = jcomp;
  a.pending = h->pending ? 1 : 0;
  a.half = h->half;
  a.fact1 = h->half * h->cfg.charge_mass;
  a.fact2 = a.fact1 * kC;
  a.h0 = h->b.hr0; a.h1 = h->b.hr1; a.dt = h->dt;
  a.bz = h->cfg.bz; a.Lb = h->b.Lb; a.hw = 0.5 * h->b.w;
  a.chh = h->chh; a.shh = h->shh; a.bwidth = h->bwidth;
  return a;
}

Push32Args push_args32(csrst_handle *h, int jcomp) {
  Push32Args a{};
  a.b = h->b32;
  a.ws = h->ws;
  a.mEx = wplane32(h, 0).p; a.mEy = wplane32(h, 1).p; a.mHx = wplane32(h, 2).p; a.mHy = wplane32(h, 3).p;
  a.wpitch = h->wpitch;
  a.acc = h->acc + (size_t)jcomp * h->L0 * h->L1;
  a.acc_scale = h->acc_scale;
  a.jcomp = jcomp;
  a.pending = h->pending ? 1 : 0;
  a.R = h->R32;
  const double fact1 = h->half * h->cfg.charge_mass;
  a.f1 = (float)fact1; a.f2 = (float)(fact1 * kC);
  a.org0 = h->b.org0; a.org1 = h->b.org1; a.h0 = h->b.hr0; a.h1 = h->b.hr1;
  a.bz = h->cfg.bz; a.Lb = h->b.Lb; a.hw = 0.5 * h->b.w;
  a.chh = h->chh; a.shh = h->shh; a.bwidth = h->bwidth;
  a.old_cell = h->old_cell; a.old_o0 = h->old_o0; a.old_o1 = h->old_o1;
  return a;
}

// PartBunch::push_particles on the device (no host synchronisation).
int push_async(csrst_handle *h, int jcomp) {
  const bool bb_ok = h->bb == kBBValid || (h->bb == kBBValidIfPending && h->pending);
  if (h->fp32) {
    if (!bb_ok) {
      launch_bbox32(h->b32, h->R32, h->pending ? 1 : 0, h->ws, h->s);
      h->prepped = false;
    }
    if (!h->prepped) launch_prep32(h->ws, h->order, h->s);
    launch_push32(push_args32(h, jcomp), h->order, h->s);
    launch_after32(h->ws, h->prep_after ? 1 : 0, h->s);
    h->prepped = h->prep_after;
    h->prep_after = false;
    h->pending = false;
    h->fresh = false;
    h->bb = kBBValidIfPending;
    h->acc_fresh[jcomp] = true;
    return CSRST_OK;
  }
  if (h->cfg.flags & CSRST_FLAG_KEEP_OLD) {  // keep oldR for inspection
    k_set_pending_old<<<(unsigned)((h->n + 255) / 256), 256, 0, h->s>>>(h->x, h->y, h->px, h->py, h->n,
                                                                       h->half, h->pending, h->ox, h->oy);
  }
  if (!bb_ok) launch_bbox_next(h->x, h->y, h->px, h->py, h->n, h->half, h->pending, h->ws, h->s);
  launch_push_prep(h->ws, h->b.hr0, h->b.hr1, h->order, h->s);
  launch_push(push_args(h, jcomp), h->order, h->push_grid, h->s);
  launch_global_bounds(h->ws, h->b.hr0, h->b.hr1, h->s);
  h->pending = false;
  h->fresh = false;
  h->bb = kBBValidIfPending;
  h->acc_fresh[jcomp] = true;
  return CSRST_OK;
}

void drift_now(csrst_handle *h, double dt) {
  if (h->fp32)
    launch_drift32(h->b32, h->R32, (float)(dt * kC / h->b.hr0), (float)(dt * kC / h->b.hr1), h->s);
  else
    launch_drift(h->x, h->y, h->px, h->py, h->n, dt * kC, h->s);
}

// drift(-dt/2) right after a push: defer it into the next push.
void drift_back(csrst_handle *h) {
  if (h->pending) {  // materialise the older one first
    drift_now(h, -0.5 * h->dt);
    h->bb = kBBInvalid;
    h->prepped = false;
  }
  h->pending = true;
  if (h->bb == kBBValidIfPending) h->bb = kBBValid;
}

void materialise(csrst_handle *h) {
  if (!h->pending) return;
  drift_now(h, -0.5 * h->dt);
  h->prepped = false;
  h->pending = false;
  if (h->fp32) h->bb = kBBInvalid;
  // the stored box of the next gather positions stays exact: R_true + h v(P)
  // has the same bits whether the drift was deferred or applied
}

void half_h_async(csrst_handle *h) {
  if (h->fp32) {
    FieldArgsT<float> a = field_args32(h, 0);
    launch_half_h(a, h->s);
    launch_exchange(a, 0, h->s);
    return;
  }
  FieldArgs a = field_args(h, 0);
  launch_half_h(a, h->s);
  launch_exchange(a, 0, h->s);
}

void update_e_async(csrst_handle *h, int comp) {
  if (h->fp32) {
    FieldArgsT<float> a = field_args32(h, comp);
    launch_update_e(a, comp, h->s);
    launch_exchange(a, comp == 0 ? 1 : 2, h->s);
  } else {
    FieldArgs a = field_args(h, comp);
    launch_update_e(a, comp, h->s);
    launch_exchange(a, comp == 0 ? 1 : 2, h->s);
  }
  h->acc_fresh[comp] = false;
}

void move_async(csrst_handle *h) {
  if (h->fp32) launch_move(field_args32(h, 0), h->scratchf, h->b.hr0, h->b.hr1, h->s);
  else launch_move(field_args(h, 0), h->scratch, h->b.hr0, h->b.hr1, h->s);
}

// Window fill from the static mesh (copyFields + exchangeBoundaries,
// main.cpp:335-342) and the window-wall check.
void fill_window(csrst_handle *h) {
  if (h->fp32) {
    FieldArgsT<float> fa = field_args32(h, 0);
    launch_copy_to_window(fa, h->s);
    launch_exchange(fa, 0, h->s);
    launch_exchange(fa, 1, h->s);
    launch_exchange(fa, 2, h->s);
    launch_check_window(fa, h->s);
  } else {
    FieldArgs fa = field_args(h, 0);
    launch_copy_to_window(fa, h->s);
    launch_exchange(fa, 0, h->s);
    launch_exchange(fa, 1, h->s);
    launch_exchange(fa, 2, h->s);
    launch_check_window(fa, h->s);
  }
}

// The bunch as FP64 arrays (positions with any pending drift applied):
// the FP64 path's own arrays, or FP32 mode's converted into d64.
void bunch64(csrst_handle *h, const double **x, const double **y, const double **px, const double **py,
             int *pending) {
  if (!h->fp32) {
    *x = h->x; *y = h->y; *px = h->px; *py = h->py; *pending = h->pending ? 1 : 0;
    return;
  }
  const size_t n = (size_t)h->n;
  launch_to64(h->b32, h->R32, h->P0, h->P1, h->pending ? 1 : 0, h->b.org0, h->b.org1, h->b.hr0,
              h->b.hr1, h->d64, h->d64 + n, h->d64 + 2 * n, h->d64 + 3 * n, h->s);
  *x = h->d64; *y = h->d64 + n; *px = h->d64 + 2 * n; *py = h->d64 + 3 * n; *pending = 0;
}

// Beam moments of the current bunch into dout (out[18]) and dmean, without a
// host synchronisation; FP32 mode reads its bunch in place.
void moments_async(csrst_handle *h) {
  if (h->fp32) {
    launch_moments32(Bunch32View{h->b32, h->R32, h->P0, h->P1, h->pending ? 1 : 0, h->b.org0, h->b.org1,
                                 h->b.hr0, h->b.hr1},
                     h->dscratch, h->dmean, h->dout, h->s);
    return;
  }
  launch_moments(h->x, h->y, h->px, h->py, h->n, h->half, h->pending ? 1 : 0, h->dscratch, h->dmean, h->dout,
                 h->s);
}

// Polls of a fused-sweep tile's staging wait before it gives up
// (csrst_set_staging_wait_limit; negative: the stuck-wait hook).
constexpr long long kStagingDefault = 1ll << 22;
long long g_staging_polls = kStagingDefault;

// The fused static sweep runs unless something needs the sub-step kernels:
// absorbing layers, an ensemble whose tables hold this handle's planes, or
// CSRST_FLAG_SUBSTEP_FIELDS.
bool fused_ok(const csrst_handle *h) {
  return h->zfix && h->kind && !h->pml && h->ens_refs == 0 && !(h->cfg.flags & CSRST_FLAG_SUBSTEP_FIELDS);
}

void swap_sets(csrst_handle *h) {
  std::swap(h->Ex, h->ExB); std::swap(h->Ey, h->EyB); std::swap(h->Hx, h->HxB); std::swap(h->Hy, h->HyB);
  std::swap(h->Exf, h->ExfB); std::swap(h->Eyf, h->EyfB); std::swap(h->Hxf, h->HxfB); std::swap(h->Hyf, h->HyfB);
  h->par ^= 1;
}

// Half H, Ex and half H of the static mesh and the window with their strip
// exchanges, and the static Ey, as one sweep into the other plane set
// (fields.cu); the sets then swap.
int fused_fields_async(csrst_handle *h) {
  int rc;
  if (h->fp32) {
    const PlaneT<float> dst[4] = {{h->ExfB, h->pitch32}, {h->EyfB, h->pitch32}, {h->HxfB, h->pitch32},
                                  {h->HyfB, h->pitch32}};
    rc = launch_yee_fused(field_args32(h, 0), dst, h->kind, h->kpitch, h->cutidx, static_cast<float *>(h->zfix),
                          h->zpitch, h->zrows, g_staging_polls, h->s, h->s2, h->fork, h->join);
  } else {
    const Plane dst[4] = {{h->ExB, h->pitch}, {h->EyB, h->pitch}, {h->HxB, h->pitch}, {h->HyB, h->pitch}};
    rc = launch_yee_fused(field_args(h, 0), dst, h->kind, h->kpitch, h->cutidx, static_cast<double *>(h->zfix),
                          h->zpitch, h->zrows, g_staging_polls, h->s, h->s2, h->fork, h->join);
  }
  if (rc != kOk) return fail(h, rc == kErrArg ? CSRST_E_ARG : CSRST_E_CUDA, "fused field sweep: tensor-map set-up");
  h->acc_fresh[0] = false;
  swap_sets(h);
  return CSRST_OK;
}

// The window's Ey sub-step and Ey exchange after the second push.
void window_ey_async(csrst_handle *h) {
  if (h->fp32) launch_window_ey(field_args32(h, 1), h->s);
  else launch_window_ey(field_args(h, 1), h->s);
  h->acc_fresh[1] = false;
}

void mark(csrst_handle *h, int k) {
  if (h->tev) cudaEventRecord(h->tev[k], h->s);
}

// TETMSolver::updateField_firstStep + updateField_secondStep + moveMesh.
// Events 0..7 (csrst_step_timed) bracket the pushes, the field work of each
// half and the move.
int step_async(csrst_handle *h) {
  mark(h, 0);
  // in the fused step nothing moves the particles or the window between the
  // two pushes: the first push's closing kernel also sets up the second
  h->prepped = false;
  h->prep_after = h->fp32 && fused_ok(h);
  push_async(h, 0);
  mark(h, 1);
  if (fused_ok(h)) {
    const int rc = fused_fields_async(h);
    if (rc) {
      h->prepped = false;
      return rc;
    }
    mark(h, 2);
    drift_back(h);
    mark(h, 3);
    push_async(h, 1);
    mark(h, 4);
    window_ey_async(h);
  } else {
    half_h_async(h);
    update_e_async(h, 0);
    half_h_async(h);
    mark(h, 2);
    drift_back(h);
    mark(h, 3);
    push_async(h, 1);
    mark(h, 4);
    update_e_async(h, 1);
  }
  mark(h, 5);
  drift_back(h);
  mark(h, 6);
  move_async(h);
  mark(h, 7);
  return CSRST_OK;
}

// FP32 mode's reference momentum and drift constants, rounded once.
void set_ref32(csrst_handle *h) {
  h->R32.P0 = (float)h->P0;
  h->R32.P1 = (float)h->P1;
  h->R32.G2 = (float)(1.0 + (h->P0 * h->P0 + h->P1 * h->P1));
  h->R32.kh0 = (float)h->kh0;
  h->R32.kh1 = (float)h->kh1;
}

// Start positions of the last move (CSRST_FLAG_KEEP_OLD in FP32 mode).
cudaError_t alloc_old32(csrst_handle *h) {
  if (!(h->cfg.flags & CSRST_FLAG_KEEP_OLD) || !h->fp32) return cudaSuccess;
  const size_t n = (size_t)h->n;
  cudaError_t e = cudaMalloc(&h->old_cell, n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&h->old_o0, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&h->old_o1, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMemsetAsync(h->old_cell, 0, n * sizeof(int), h->s);
  return e;
}

int need_bunch(csrst_handle *h) {
  if (!h) return CSRST_E_ARG;
  if (h->n <= 0 || !(h->win || h->winf)) return fail(h, CSRST_E_NO_PARTICLES, "no bunch loaded");
  return CSRST_OK;
}

}  // namespace

extern "C" {

int csrst_create(const csrst_config *cfg, csrst_handle **out) {
  if (!cfg || !out) return fail(nullptr, CSRST_E_ARG, "null argument");
  *out = nullptr;
  if (cfg->Nx < 8 || cfg->Ny < 8 || cfg->shape_order < 0 || cfg->shape_order > 2 || !(cfg->width > 0))
    return fail(nullptr, CSRST_E_ARG, "invalid configuration");
  if (cfg->flags & ~(CSRST_FLAG_KEEP_OLD | CSRST_FLAG_FP32 | CSRST_FLAG_SUBSTEP_FIELDS))
    return fail(nullptr, CSRST_E_ARG, "unknown flags");
  if ((cfg->flags & CSRST_FLAG_FP32) && (cfg->Nx > 32767 || cfg->Ny > 32767))
    return fail(nullptr, CSRST_E_ARG, "FP32 mode packs cell indices in 16 bits: Nx, Ny <= 32767");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, CSRST_E_CUDA, "no CUDA device");
  csrst_handle *h = new csrst_handle;
  h->cfg = *cfg;
  h->order = cfg->shape_order;
  h->fp32 = (cfg->flags & CSRST_FLAG_FP32) != 0;
  bend_setup(h);
  h->kh0 = h->half / h->b.hr0;
  h->kh1 = h->half / h->b.hr1;
  auto bad = [&](cudaError_t e, const char *w) {
    g_create_error = std::string(w) + ": " + cudaGetErrorString(e);
    csrst_destroy(h);
    return CSRST_E_CUDA;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking)) != cudaSuccess) return bad(e, "stream");
  {  // the window fix-up's stream at the highest priority: its cluster starts ahead of the sweep's tiles
    int least = 0, greatest = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess) return bad(e, "stream");
    if ((e = cudaStreamCreateWithPriority(&h->s2, cudaStreamNonBlocking, greatest)) != cudaSuccess)
      return bad(e, "stream");
  }
  if ((e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming)) != cudaSuccess) return bad(e, "event");
  if ((e = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming)) != cudaSuccess) return bad(e, "event");
  const int Nx = cfg->Nx, Ny = cfg->Ny;
  h->pitch = ((Nx + 2 + 31) / 32) * 32;
  const size_t ps = (size_t)h->pitch * (Ny + 2);
  if (h->fp32) {  // FP32 static planes only; FP64 copies are made on demand
    h->pitch32 = ((Nx + 2 + 63) / 64) * 64;
    const size_t ps32 = (size_t)h->pitch32 * (Ny + 2);
    float **planes[8] = {&h->Exf, &h->Eyf, &h->Hxf, &h->Hyf, &h->ExfB, &h->EyfB, &h->HxfB, &h->HyfB};
    for (float **p : planes) {
      if ((e = cudaMalloc(p, ps32 * sizeof(float))) != cudaSuccess) return bad(e, "static fields");
      if ((e = cudaMemsetAsync(*p, 0, ps32 * sizeof(float), h->s)) != cudaSuccess) return bad(e, "memset");
    }
  } else {
    double **planes[8] = {&h->Ex, &h->Ey, &h->Hx, &h->Hy, &h->ExB, &h->EyB, &h->HxB, &h->HyB};
    for (double **p : planes) {
      if ((e = cudaMalloc(p, ps * sizeof(double))) != cudaSuccess) return bad(e, "static fields");
      if ((e = cudaMemsetAsync(*p, 0, ps * sizeof(double), h->s)) != cudaSuccess) return bad(e, "memset");
    }
  }
  if ((e = cudaMalloc(&h->mask, (size_t)Nx * Ny)) != cudaSuccess) return bad(e, "mask");
  if ((e = cudaMalloc(&h->ws, sizeof(WinState))) != cudaSuccess) return bad(e, "window state");
  if ((e = cudaMemsetAsync(h->ws, 0, sizeof(WinState), h->s)) != cudaSuccess) return bad(e, "memset");
  const size_t nd = moments_scratch_doubles();
  if ((e = cudaMalloc(&h->dscratch, nd * sizeof(double))) != cudaSuccess) return bad(e, "diag");
  if ((e = cudaMalloc(&h->dmean, 8 * sizeof(double))) != cudaSuccess) return bad(e, "diag");
  if ((e = cudaMalloc(&h->dout, 32 * sizeof(double))) != cudaSuccess) return bad(e, "diag");
  int rc = build_geometry(h->b, h->mask, &h->cells, &h->ncells, &h->cutidx, h->s);
  if (rc != kOk) {
    g_create_error = rc == kErrGeometry ? "bend geometry: the reference asserts for this configuration"
                                        : "geometry build failed";
    csrst_destroy(h);
    return rc;
  }
  // cell kinds of the fused sweep, in the static storage layout
  h->kpitch = ((Nx + 2 + 15) / 16) * 16;
  const size_t kb = (size_t)h->kpitch * (Ny + 2);
  if ((e = cudaMalloc(&h->kind, kb)) != cudaSuccess) return bad(e, "cell kinds");
  if ((e = cudaMemsetAsync(h->kind, 0, kb, h->s)) != cudaSuccess) return bad(e, "memset");
  launch_build_kind(h->mask, h->cutidx, Nx, Ny, h->kind, h->kpitch, h->s);
  if ((e = cudaGetLastError()) != cudaSuccess) return bad(e, "cell kinds");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  h->push_grid = 3 * sms;  // single-member FP64 push: three CTAs per SM
  *out = h;
  return CSRST_OK;
}

int csrst_destroy(csrst_handle *h) {
  if (!h) return CSRST_OK;
  if (h->s) cudaStreamSynchronize(h->s);
  free_particles(h);
  drop_graphs(h);
  cudaFree(h->Ex); cudaFree(h->Ey); cudaFree(h->Hx); cudaFree(h->Hy);
  cudaFree(h->Exf); cudaFree(h->Eyf); cudaFree(h->Hxf); cudaFree(h->Hyf);
  cudaFree(h->ExB); cudaFree(h->EyB); cudaFree(h->HxB); cudaFree(h->HyB);
  cudaFree(h->ExfB); cudaFree(h->EyfB); cudaFree(h->HxfB); cudaFree(h->HyfB);
  cudaFree(h->kind);
  cudaFree(h->mask); cudaFree(h->cells); cudaFree(h->cutidx); cudaFree(h->ws);
  cudaFree(h->dscratch); cudaFree(h->dmean); cudaFree(h->dout);
  cudaFree(h->pml); cudaFree(h->pml32); cudaFree(h->pml_rows); cudaFree(h->psi);
  if (h->s2) cudaStreamSynchronize(h->s2);
  if (h->fork) cudaEventDestroy(h->fork);
  if (h->join) cudaEventDestroy(h->join);
  if (h->s2) cudaStreamDestroy(h->s2);
  if (h->s) cudaStreamDestroy(h->s);
  delete h;
  return CSRST_OK;
}

int csrst_get_error(const csrst_handle *h, char *buf, size_t len) {
  if (!buf || len == 0) return CSRST_E_ARG;
  const std::string &m = h ? h->err : g_create_error;
  std::snprintf(buf, len, "%s", m.c_str());
  return CSRST_OK;
}

void *csrst_stream(csrst_handle *h) { return h ? (void *)h->s : nullptr; }

int csrst_sync(csrst_handle *h) {
  if (!h) return CSRST_E_ARG;
  CK(cudaStreamSynchronize(h->s));
  CK(cudaGetLastError());
  return check_err(h);
}

int csrst_get_info(csrst_handle *h, double *info8) {
  if (!h || !info8) return CSRST_E_ARG;
  double v[8] = {h->b.hr0, h->b.hr1, h->b.org0, h->b.org1, h->dt, h->acc_scale, (double)h->ncells,
                 (double)h->wpitch};
  std::memcpy(info8, v, sizeof(v));
  return CSRST_OK;
}

int csrst_get_geometry(csrst_handle *h, uint8_t *inside, double *cells, long max_cells, long *ncells) {
  if (!h) return CSRST_E_ARG;
  if (inside) CK(cudaMemcpyAsync(inside, h->mask, (size_t)h->b.Nx * h->b.Ny, cudaMemcpyDeviceToHost, h->s));
  if (ncells) *ncells = h->ncells;
  if (cells && max_cells > 0 && h->ncells > 0) {
    std::vector<CutCellDev> c(h->ncells);
    CK(cudaMemcpyAsync(c.data(), h->cells, c.size() * sizeof(CutCellDev), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    for (long k = 0; k < (long)c.size() && k < max_cells; ++k) {
      double v[7] = {(double)c[k].i, (double)c[k].j, c[k].l0, c[k].l1, c[k].area, c[k].n0, c[k].n1};
      std::memcpy(cells + 7 * k, v, sizeof(v));
    }
  }
  CK(cudaStreamSynchronize(h->s));
  return CSRST_OK;
}

int csrst_set_static_fields(csrst_handle *h, const double *ex, const double *ey, const double *hzx,
                            const double *hzy) {
  if (!h) return CSRST_E_ARG;
  if (h->fp32) {  // through an FP64 staging buffer, rounded once on the device
    const double *src[4] = {ex, ey, hzx, hzy};
    float *dst[4] = {h->Exf, h->Eyf, h->Hxf, h->Hyf};
    double *tmp = nullptr;
    CK(cudaMalloc(&tmp, (size_t)h->b.Nx * h->b.Ny * sizeof(double)));
    for (int k = 0; k < 4; ++k) {
      if (!src[k]) continue;
      CK(cudaMemcpyAsync(tmp, src[k], (size_t)h->b.Nx * h->b.Ny * sizeof(double), cudaMemcpyHostToDevice, h->s));
      launch_d2f(tmp, h->b.Nx, dst[k] + h->pitch32 + 1, h->pitch32, h->b.Ny, h->b.Nx, h->s);
    }
    CK(cudaStreamSynchronize(h->s));
    cudaFree(tmp);
    CK(cudaGetLastError());
    return CSRST_OK;
  }
  const double *src[4] = {ex, ey, hzx, hzy};
  double *dst[4] = {h->Ex, h->Ey, h->Hx, h->Hy};
  for (int k = 0; k < 4; ++k) {
    if (!src[k]) continue;
    CK(cudaMemcpy2DAsync(dst[k] + h->pitch + 1, h->pitch * sizeof(double), src[k], h->b.Nx * sizeof(double),
                         h->b.Nx * sizeof(double), h->b.Ny, cudaMemcpyHostToDevice, h->s));
  }
  CK(cudaStreamSynchronize(h->s));
  return CSRST_OK;
}

int csrst_get_static_fields(csrst_handle *h, double *ex, double *ey, double *hzx, double *hzy) {
  if (!h) return CSRST_E_ARG;
  if (h->fp32) {
    double *dst[4] = {ex, ey, hzx, hzy};
    const float *src[4] = {h->Exf, h->Eyf, h->Hxf, h->Hyf};
    double *tmp = nullptr;
    CK(cudaMalloc(&tmp, (size_t)h->b.Nx * h->b.Ny * sizeof(double)));
    for (int k = 0; k < 4; ++k) {
      if (!dst[k]) continue;
      launch_f2d(src[k] + h->pitch32 + 1, h->pitch32, tmp, h->b.Nx, h->b.Ny, h->b.Nx, h->s);
      CK(cudaMemcpyAsync(dst[k], tmp, (size_t)h->b.Nx * h->b.Ny * sizeof(double), cudaMemcpyDeviceToHost, h->s));
      CK(cudaStreamSynchronize(h->s));
    }
    cudaFree(tmp);
    CK(cudaGetLastError());
    return CSRST_OK;
  }
  double *dst[4] = {ex, ey, hzx, hzy};
  const double *src[4] = {h->Ex, h->Ey, h->Hx, h->Hy};
  for (int k = 0; k < 4; ++k) {
    if (!dst[k]) continue;
    CK(cudaMemcpy2DAsync(dst[k], h->b.Nx * sizeof(double), src[k] + h->pitch + 1, h->pitch * sizeof(double),
                         h->b.Nx * sizeof(double), h->b.Ny, cudaMemcpyDeviceToHost, h->s));
  }
  CK(cudaStreamSynchronize(h->s));
  return CSRST_OK;
}

int csrst_reset_outside(csrst_handle *h) {
  if (!h) return CSRST_E_ARG;
  if (h->fp32) launch_reset_outside(field_args32(h, 0), h->cutidx, h->s);
  else launch_reset_outside(field_args(h, 0), h->cutidx, h->s);
  CK(cudaStreamSynchronize(h->s));
  return CSRST_OK;
}

int csrst_load_particles(csrst_handle *h, const double *x, const double *y, const double *px,
                         const double *py, const double *q, size_t n) {
  if (!h || (n > 0 && (!x || !y || !px || !py || !q))) return CSRST_E_ARG;
  if (n == 0) return fail(h, CSRST_E_NO_PARTICLES, "empty bunch");
  CK(cudaStreamSynchronize(h->s));
  const long long N = (long long)n;
  const size_t nb = n * sizeof(double);
  // the bunch goes up and is checked on the device before the handle's
  // current bunch is released, so that a rejected bunch leaves it intact
  double *tmp[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  unsigned long long *chk = nullptr;
  auto drop = [&]() {
    for (int k = 0; k < 5; ++k) pfree(tmp[k], h->s);
    pfree(chk, h->s);
  };
  for (int k = 0; k < 5; ++k)
    if (palloc(&tmp[k], nb, h->s) != cudaSuccess) { drop(); return fail(h, CSRST_E_CUDA, "bunch upload: out of memory"); }
  if (palloc(&chk, 2 * sizeof(unsigned long long), h->s) != cudaSuccess) {
    drop();
    return fail(h, CSRST_E_CUDA, "bunch upload: out of memory");
  }
  const double *src[5] = {x, y, px, py, q};
  for (int k = 0; k < 5; ++k) CK(cudaMemcpyAsync(tmp[k], src[k], nb, cudaMemcpyHostToDevice, h->s));
  unsigned long long hchk[2] = {~0ull, 0ull};
  CK(cudaMemcpyAsync(chk, hchk, sizeof(hchk), cudaMemcpyHostToDevice, h->s));
  {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (N + 255) / 256, cap = 8LL * sms;
    k_check_bunch<<<(unsigned)(want < cap ? want : cap), 256, 0, h->s>>>(
        tmp[0], tmp[1], tmp[2], tmp[3], tmp[4], N, h->fp32 ? 1 : 0, h->b.org0, h->b.org1, h->b.hr0, h->b.hr1,
        h->b.Nx, h->b.Ny, chk);
  }
  CK(cudaMemcpyAsync(hchk, chk, sizeof(hchk), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  if (hchk[0] < (unsigned long long)n) {  // the first rejected particle, with its reason
    const size_t i = (size_t)hchk[0];
    drop();
    if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(px[i]) || !std::isfinite(py[i]) ||
        !std::isfinite(q[i]))
      return fail(h, CSRST_E_ARG, "non-finite particle data at index " + std::to_string(i));
    // FP32 mode stores 16-bit cell indices of the static mesh
    return fail(h, CSRST_E_ARG, "particle outside the static mesh at index " + std::to_string(i));
  }
  const double qmax = bits_to_double(hchk[1]);
  pfree(chk, h->s);
  chk = nullptr;
  free_particles(h);
  h->n = N;
  for (double **p : {&h->x, &h->y, &h->px, &h->py, &h->q, &h->ox, &h->oy}) CK(palloc(p, nb, h->s));
  // particle box on the static mesh -> window +-5 cells (main.cpp:198-217)
  WinState w0{};
  w0.cur = 0;
  CK(cudaMemcpyAsync(h->ws, &w0, sizeof(WinState), cudaMemcpyHostToDevice, h->s));
  launch_bbox_next(tmp[0], tmp[1], tmp[2], tmp[3], N, 0.0, 0, h->ws, h->s);
  long long bb[4];
  CK(cudaMemcpyAsync(bb, h->ws->bb[0], sizeof(bb), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  const double mn0 = ord_dbl(bb[0]), mn1 = ord_dbl(bb[1]), mx0 = ord_dbl(bb[2]), mx1 = ord_dbl(bb[3]);
  int d[4] = {(int)std::floor((mn0 - h->b.org0) / h->b.hr0), (int)std::floor((mx0 - h->b.org0) / h->b.hr0),
              (int)std::floor((mn1 - h->b.org1) / h->b.hr1), (int)std::floor((mx1 - h->b.org1) / h->b.hr1)};
  d[0] -= 5; d[1] += 5; d[2] -= 5; d[3] += 5;
  h->L0 = d[1] - d[0] + 1; h->L1 = d[3] - d[2] + 1;
  h->wpitch = h->L0 + 2;
  w0.P0 = d[0]; w0.P1 = d[2]; w0.L0 = h->L0; w0.L1 = h->L1;
  w0.mo0 = h->b.org0 + d[0] * h->b.hr0;
  w0.mo1 = h->b.org1 + d[2] * h->b.hr1;
  w0.bb[0][0] = bb[0]; w0.bb[0][1] = bb[1]; w0.bb[0][2] = bb[2]; w0.bb[0][3] = bb[3];
  CK(cudaMemcpyAsync(h->ws, &w0, sizeof(WinState), cudaMemcpyHostToDevice, h->s));
  const size_t wp = (size_t)h->wpitch * (h->L1 + 2);
  if (h->fp32) {
    CK(cudaMalloc(&h->winf, 6 * wp * sizeof(float)));
    CK(cudaMemsetAsync(h->winf, 0, 6 * wp * sizeof(float), h->s));
    CK(cudaMalloc(&h->scratchf, 6 * wp * sizeof(float)));
  } else {
    CK(cudaMalloc(&h->win, 6 * wp * sizeof(double)));
    CK(cudaMemsetAsync(h->win, 0, 6 * wp * sizeof(double), h->s));
    CK(cudaMalloc(&h->scratch, 6 * wp * sizeof(double)));
  }
  CK(cudaMalloc(&h->acc, 2 * (size_t)h->L0 * h->L1 * sizeof(unsigned long long)));
  CK(cudaMemsetAsync(h->acc, 0, 2 * (size_t)h->L0 * h->L1 * sizeof(unsigned long long), h->s));
  // scratch of the fused sweep's fix-up: the window's footprint widened by
  // two cells and the cells its sub-steps read (launch_yee_fused)
  h->zpitch = h->L0 + 6;
  h->zrows = h->L1 + 7;
  CK(cudaMalloc(&h->zfix, 4 * (size_t)h->zpitch * h->zrows * (h->fp32 ? sizeof(float) : sizeof(double))));
  // PartBunch::sortParticles: y slice of the window, then x (stable radix sorts)
  {
    unsigned long long *kx = nullptr, *kx2 = nullptr;
    unsigned int *ks = nullptr, *ks2 = nullptr;
    long long *i1 = nullptr, *i2 = nullptr;
    void *ct = nullptr;
    size_t ctb = 0, ctb2 = 0;
    CK(palloc(&kx, n * 8, h->s)); CK(palloc(&kx2, n * 8, h->s));
    CK(palloc(&ks, n * 4, h->s)); CK(palloc(&ks2, n * 4, h->s));
    CK(palloc(&i1, n * 8, h->s)); CK(palloc(&i2, n * 8, h->s));
    const unsigned g = (unsigned)((n + 255) / 256);
    k_sort_keys<<<g, 256, 0, h->s>>>(tmp[0], tmp[1], N, h->ws, h->b.hr1, kx, i1);
    CK(cub::DeviceRadixSort::SortPairs(nullptr, ctb, kx, kx2, i1, i2, (int)n, 0, 64, h->s));
    CK(cub::DeviceRadixSort::SortPairs(nullptr, ctb2, ks, ks2, i2, i1, (int)n, 0, 32, h->s));
    CK(palloc(&ct, ctb > ctb2 ? ctb : ctb2, h->s));
    CK(cub::DeviceRadixSort::SortPairs(ct, ctb, kx, kx2, i1, i2, (int)n, 0, 64, h->s));
    k_slice_keys<<<g, 256, 0, h->s>>>(tmp[1], i2, N, h->ws, h->b.hr1, ks);
    CK(cub::DeviceRadixSort::SortPairs(ct, ctb2, ks, ks2, i2, i1, (int)n, 0, 32, h->s));
    double *dst[5] = {h->x, h->y, h->px, h->py, h->q};
    for (int k = 0; k < 5; ++k) k_gather_perm<<<g, 256, 0, h->s>>>(i1, N, tmp[k], dst[k]);
    for (void *p : {(void *)kx, (void *)kx2, (void *)ks, (void *)ks2, (void *)i1, (void *)i2, ct}) pfree(p, h->s);
  }
  for (int k = 0; k < 5; ++k) pfree(tmp[k], h->s);
  CK(cudaMemcpyAsync(h->ox, h->x, nb, cudaMemcpyDeviceToDevice, h->s));
  CK(cudaMemcpyAsync(h->oy, h->y, nb, cudaMemcpyDeviceToDevice, h->s));
  // 64-bit fixed-point scale of the current: a power of two with the
  // largest possible per-cell sum (every particle, 4x margin) below 2^62.
  const double bound = 4.0 * (double)n * (qmax > 0 ? qmax : 1e-30) * kC / (h->b.hr0 * h->b.hr1);
  h->acc_scale = std::ldexp(1.0, (int)std::floor(std::log2(std::ldexp(1.0, 62) / bound)));
  // window fill (copyFields + exchangeBoundaries, main.cpp:335-342)
  fill_window(h);
  h->pending = false;
  h->bb = kBBInvalid;
  h->acc_fresh[0] = h->acc_fresh[1] = false;
  if (h->fp32) {
    // reference momentum = mean momentum; then the FP32 bunch replaces the FP64 arrays
    double *part = nullptr, sums[2];
    CK(palloc(&part, (2 * 296 + 2) * sizeof(double), h->s));
    launch_psum(h->px, h->py, N, part, part + 2 * 296, h->s);
    CK(cudaMemcpyAsync(sums, part + 2 * 296, sizeof(sums), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    pfree(part, h->s);
    h->P0 = sums[0] / (double)N;
    h->P1 = sums[1] / (double)N;
    set_ref32(h);
    // FP32 mode accumulates the flux q-units of flux32.cuh: every particle
    // carries K = q scale, and a cell's flux stays below 4 N max|q| scale
    const double fbound = 4.0 * (double)n * (qmax > 0 ? qmax : 1e-30) * (1.0 + 1e-6);
    h->acc_scale = std::ldexp(1.0, (int)std::floor(std::log2(std::ldexp(1.0, 62) / fbound)));
    Bunch32 &b = h->b32;
    b.n = N;
    CK(palloc(&b.cell, n * sizeof(int), h->s));
    for (float **p : {&b.ox, &b.oy, &b.dpx, &b.dpy, &b.q}) CK(palloc(p, n * sizeof(float), h->s));
    CK(palloc(&h->d64, 4 * nb, h->s));
    launch_from64(h->x, h->y, h->px, h->py, h->q, N, h->b.org0, h->b.org1, h->b.hr0, h->b.hr1, h->P0, h->P1, b,
                  h->s);
    for (double **p : {&h->x, &h->y, &h->px, &h->py, &h->q, &h->ox, &h->oy}) { pfree(*p, h->s); *p = nullptr; }
    CK(alloc_old32(h));
    launch_bbox32(b, h->R32, 0, h->ws, h->s);
  } else {
    launch_bbox_next(h->x, h->y, h->px, h->py, N, h->half, 0, h->ws, h->s);
  }
  h->bb = kBBValid;
  h->fresh = true;
  CK(cudaStreamSynchronize(h->s));
  CK(cudaGetLastError());
  return check_err(h);
}

int csrst_initial_fields(csrst_handle *h, double tol_first, double tol_rest, int max_iter, double *report8) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!h->fresh) return fail(h, CSRST_E_ARG, "initial fields need a freshly loaded bunch (before the first push)");
  if (!(tol_first > 0) || !(tol_rest > 0) || max_iter < 1) return fail(h, CSRST_E_ARG, "invalid tolerance");
  PoissonInput in{};
  in.n = h->n;
  in.order = h->order;
  in.mask = h->mask; in.cutidx = h->cutidx; in.cells = h->cells;
  in.b = h->b; in.dt = h->dt;
  in.tol_first = tol_first; in.tol_rest = tol_rest; in.maxit = max_iter;
  // FP32 mode solves in FP64 (the bunch converted, the planes staged) and
  // rounds the fields once
  double *qd = nullptr, *stage = nullptr;
  const size_t ps = (size_t)h->pitch * (h->b.Ny + 2);
  if (h->fp32) {
    int pend = 0;
    bunch64(h, &in.x, &in.y, &in.px, &in.py, &pend);
    CK(cudaMalloc(&qd, (size_t)h->n * sizeof(double)));
    launch_f2d(h->b32.q, (int)h->n, qd, (int)h->n, 1, (int)h->n, h->s);
    in.q = qd;
    CK(cudaMalloc(&stage, 4 * ps * sizeof(double)));
    CK(cudaMemsetAsync(stage, 0, 4 * ps * sizeof(double), h->s));
    in.Ex = plane(stage, h->pitch); in.Ey = plane(stage + ps, h->pitch);
    in.Hx = plane(stage + 2 * ps, h->pitch); in.Hy = plane(stage + 3 * ps, h->pitch);
  } else {
    in.x = h->x; in.y = h->y; in.px = h->px; in.py = h->py; in.q = h->q;
    in.Ex = plane(h->Ex, h->pitch); in.Ey = plane(h->Ey, h->pitch);
    in.Hx = plane(h->Hx, h->pitch); in.Hy = plane(h->Hy, h->pitch);
  }
  PoissonReport rep{};
  std::string msg;
  rc = poisson_initial_fields(in, &rep, h->s, &msg);
  if (h->fp32 && rc == kOk) {
    float *dst[4] = {h->Exf, h->Eyf, h->Hxf, h->Hyf};
    for (int k = 0; k < 4; ++k)
      launch_d2f(stage + k * ps, h->pitch, dst[k], h->pitch32, h->b.Ny + 2, h->b.Nx + 2, h->s);
    cudaStreamSynchronize(h->s);
  }
  cudaFree(qd);
  cudaFree(stage);
  if (rc) return fail(h, rc == kErrCuda ? CSRST_E_CUDA : CSRST_E_ARG, "initial fields: " + msg);
  // resetOutsideDomain, then copyFields + exchangeBoundaries (main.cpp:248, :335-342)
  if (h->fp32) launch_reset_outside(field_args32(h, 0), h->cutidx, h->s);
  else launch_reset_outside(field_args(h, 0), h->cutidx, h->s);
  fill_window(h);
  CK(cudaStreamSynchronize(h->s));
  CK(cudaGetLastError());
  if (report8) {
    report8[0] = rep.gamma;
    for (int k = 0; k < 3; ++k) { report8[1 + 2 * k] = rep.iters[k]; report8[2 + 2 * k] = rep.relres[k]; }
    report8[7] = rep.levels;
  }
  return check_err(h);
}

int csrst_get_particles(csrst_handle *h, double *x, double *y, double *px, double *py) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (h->fp32) {  // cell origin + offset and P + deviation, formed in FP64
    const double *src[4];
    int pend = 0;
    bunch64(h, &src[0], &src[1], &src[2], &src[3], &pend);
    double *dst[4] = {x, y, px, py};
    for (int k = 0; k < 4; ++k)
      if (dst[k]) CK(cudaMemcpyAsync(dst[k], src[k], (size_t)h->n * sizeof(double), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    return check_err(h);
  }
  materialise(h);
  const size_t nb = (size_t)h->n * sizeof(double);
  if (x) CK(cudaMemcpyAsync(x, h->x, nb, cudaMemcpyDeviceToHost, h->s));
  if (y) CK(cudaMemcpyAsync(y, h->y, nb, cudaMemcpyDeviceToHost, h->s));
  if (px) CK(cudaMemcpyAsync(px, h->px, nb, cudaMemcpyDeviceToHost, h->s));
  if (py) CK(cudaMemcpyAsync(py, h->py, nb, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return check_err(h);
}

int csrst_get_old_positions(csrst_handle *h, double *ox, double *oy) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!(h->cfg.flags & CSRST_FLAG_KEEP_OLD))
    return fail(h, CSRST_E_ARG, "create the handle with CSRST_FLAG_KEEP_OLD to keep oldR");
  const size_t nb = (size_t)h->n * sizeof(double);
  if (h->fp32) {  // the start of each particle's last move, as FP64 positions
    k_old32_to64<<<(unsigned)((h->n + 255) / 256), 256, 0, h->s>>>(h->old_cell, h->old_o0, h->old_o1, h->n, h->b.org0,
                                                                     h->b.org1, h->b.hr0, h->b.hr1, h->d64,
                                                                     h->d64 + h->n);
    if (ox) CK(cudaMemcpyAsync(ox, h->d64, nb, cudaMemcpyDeviceToHost, h->s));
    if (oy) CK(cudaMemcpyAsync(oy, h->d64 + h->n, nb, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    return CSRST_OK;
  }
  if (ox) CK(cudaMemcpyAsync(ox, h->ox, nb, cudaMemcpyDeviceToHost, h->s));
  if (oy) CK(cudaMemcpyAsync(oy, h->oy, nb, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CSRST_OK;
}

int csrst_get_window(csrst_handle *h, int *w4, double *origin2, int *gb4) {
  int rc = need_bunch(h);
  if (rc) return rc;
  WinState w;
  CK(cudaMemcpyAsync(&w, h->ws, sizeof(WinState), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  if (w4) { w4[0] = w.P0; w4[1] = w.P1; w4[2] = w.L0; w4[3] = w.L1; }
  if (origin2) { origin2[0] = w.mo0; origin2[1] = w.mo1; }
  if (gb4) std::memcpy(gb4, w.gb, sizeof(w.gb));
  return CSRST_OK;
}

int csrst_get_window_field(csrst_handle *h, int which, double *out) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (which < 0 || which > 5 || !out) return fail(h, CSRST_E_ARG, "which must be 0..5");
  if (h->fp32) {
    const size_t wp = (size_t)h->wpitch * (h->L1 + 2);
    double *tmp = nullptr;
    CK(cudaMalloc(&tmp, wp * sizeof(double)));
    if (which >= 4 && h->acc_fresh[which - 4]) {  // the current before its FP32 rounding
      CK(cudaMemsetAsync(tmp, 0, wp * sizeof(double), h->s));
      const int c = which - 4;
      k_acc_to_plane<<<(h->L0 * h->L1 + 255) / 256, 256, 0, h->s>>>(h->acc + (size_t)c * h->L0 * h->L1,
                                                                  Plane{tmp, h->wpitch}, h->L0, h->L1,
                                                                  field_args(h, c).acc_inv);
    } else {
      launch_f2d(h->winf + (size_t)which * wp, (int)wp, tmp, (int)wp, 1, (int)wp, h->s);
    }
    CK(cudaMemcpyAsync(out, tmp, wp * sizeof(double), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    cudaFree(tmp);
    return CSRST_OK;
  }
  if (which >= 4 && h->acc_fresh[which - 4]) {
    const int c = which - 4;
    k_acc_to_plane<<<(h->L0 * h->L1 + 255) / 256, 256, 0, h->s>>>(h->acc + (size_t)c * h->L0 * h->L1,
                                                                wplane(h, which), h->L0, h->L1,
                                                                1.0 / h->acc_scale);
  }
  const size_t wp = (size_t)h->wpitch * (h->L1 + 2);
  CK(cudaMemcpyAsync(out, h->win + (size_t)which * wp, wp * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CSRST_OK;
}

int csrst_push(csrst_handle *h, int jcomp) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (jcomp != 0 && jcomp != 1) return fail(h, CSRST_E_ARG, "jcomp must be 0 or 1");
  push_async(h, jcomp);
  return CSRST_OK;
}

int csrst_drift(csrst_handle *h, double dt) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!h->pending && dt == -0.5 * h->dt) {
    drift_back(h);
    return CSRST_OK;
  }
  materialise(h);
  drift_now(h, dt);
  h->bb = kBBInvalid;
  return CSRST_OK;
}

int csrst_half_h(csrst_handle *h) {
  int rc = need_bunch(h);
  if (rc) return rc;
  half_h_async(h);
  return CSRST_OK;
}

int csrst_update_e(csrst_handle *h, int comp) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (comp != 0 && comp != 1) return fail(h, CSRST_E_ARG, "comp must be 0 or 1");
  update_e_async(h, comp);
  return CSRST_OK;
}

int csrst_move_window(csrst_handle *h) {
  int rc = need_bunch(h);
  if (rc) return rc;
  move_async(h);
  return CSRST_OK;
}

int csrst_step_first(csrst_handle *h) {
  int rc = need_bunch(h);
  if (rc) return rc;
  push_async(h, 0);
  half_h_async(h);
  update_e_async(h, 0);
  half_h_async(h);
  drift_back(h);
  return CSRST_OK;
}

int csrst_step_second(csrst_handle *h) {
  int rc = need_bunch(h);
  if (rc) return rc;
  push_async(h, 1);
  update_e_async(h, 1);
  drift_back(h);
  return CSRST_OK;
}

int csrst_step(csrst_handle *h, int nsteps) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (nsteps < 0) return fail(h, CSRST_E_ARG, "nsteps < 0");
  // The graph is recorded in the steady state of the loop: the stored
  // positions owe the trailing -dt/2 drift and the box of the next gather
  // positions is current.  Anything else runs one step eagerly first.
  while (nsteps > 0 && !(h->pending && h->bb == kBBValid)) {
    if ((rc = step_async(h))) return rc;
    --nsteps;
  }
  if (nsteps == 0) return CSRST_OK;
  const bool fused = fused_ok(h);
  if (fused != h->graph_fused) {
    drop_graphs(h);
    h->graph_fused = fused;
  }
  for (; nsteps > 0; --nsteps) {
    const int p = h->par;
    if (!h->graph[p]) {  // recorded on the first step that starts from this plane set
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
      rc = step_async(h);
      const cudaError_t ce = cudaStreamEndCapture(h->s, &g);
      if (rc) {
        if (ce == cudaSuccess) cudaGraphDestroy(g);
        return rc;
      }
      if (ce != cudaSuccess) return cuda_fail(h, ce, "cudaStreamEndCapture");
      cudaError_t e = cudaGraphInstantiate(&h->graph[p], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    } else if (fused) {
      swap_sets(h);  // what the recorded step does to the host's view of the planes
    }
    CK(cudaGraphLaunch(h->graph[p], h->s));
  }
  return CSRST_OK;
}

int csrst_release_memory(void) {
  cudaMemPool_t m = lib_pool();
  if (!m) return CSRST_E_CUDA;
  return cudaMemPoolTrimTo(m, 0) == cudaSuccess ? CSRST_OK : CSRST_E_CUDA;
}

int csrst_set_staging_wait_limit(long long polls) {
  g_staging_polls = polls != 0 ? polls : kStagingDefault;
  return CSRST_OK;
}

int csrst_step_timed(csrst_handle *h, double *ms4) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!ms4) return fail(h, CSRST_E_ARG, "ms4 is NULL");
  cudaEvent_t ev[8] = {};
  for (cudaEvent_t &e : ev) CK(cudaEventCreate(&e));
  h->tev = ev;
  rc = step_async(h);
  h->tev = nullptr;
  cudaError_t e = cudaStreamSynchronize(h->s);
  float t[4] = {0, 0, 0, 0};
  if (!rc && e == cudaSuccess) {
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&b, ev[3], ev[4]);
    t[0] = a + b;
    cudaEventElapsedTime(&a, ev[1], ev[2]);
    cudaEventElapsedTime(&b, ev[4], ev[5]);
    t[1] = a + b;
    cudaEventElapsedTime(&t[2], ev[6], ev[7]);
    cudaEventElapsedTime(&t[3], ev[0], ev[7]);
  }
  for (cudaEvent_t &v : ev) cudaEventDestroy(v);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(h, e, "csrst_step_timed");
  for (int k = 0; k < 4; ++k) ms4[k] = t[k];
  return check_err(h);
}

int csrst_diag_moments(csrst_handle *h, double *out18) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!out18) return CSRST_E_ARG;
  moments_async(h);
  CK(cudaMemcpyAsync(out18, h->dout, 18 * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  return check_err(h);  // one synchronisation for both copies
}

int csrst_diag_wake(csrst_handle *h, double *out, int n) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!out || n != h->L0 - 4) return fail(h, CSRST_E_ARG, "wake buffer must hold L0 - 4 values");
  moments_async(h);
  double *d = nullptr;
  CK(cudaMallocAsync(&d, (size_t)n * sizeof(double), h->s));
  if (h->fp32)
    launch_wake(h->ws, wplane32(h, 0).p, wplane32(h, 1).p, h->wpitch, h->L0, h->b.hr0, h->b.hr1, h->dmean, d,
                h->s);
  else
    launch_wake(h->ws, wplane(h, 0).p, wplane(h, 1).p, h->wpitch, h->L0, h->b.hr0, h->b.hr1, h->dmean, d, h->s);
  CK(cudaMemcpyAsync(out, d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  CK(cudaFreeAsync(d, h->s));
  CK(cudaStreamSynchronize(h->s));
  return check_err(h);
}

int csrst_diag_line_fields(csrst_handle *h, int with_current, double *out, int cap, int *count) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!count) return fail(h, CSRST_E_ARG, "line fields: count pointer missing");
  moments_async(h);
  double m[18];
  CK(cudaMemcpyAsync(m, h->dout, sizeof(m), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  // samples from 1.5 g0 - 0.5 g1 to 2 g1 - g0, g0 / g1 the static cells holding rmin / rmax
  // (SaveEMFields.cpp:59-76)
  const double g0 = std::floor((m[10] - h->b.org0) / h->b.hr0), g1 = std::floor((m[12] - h->b.org0) / h->b.hr0);
  const double l0 = std::floor(1.5 * g0 - 0.5 * g1), u0 = 2 * g1 - g0;
  const long long i0 = (long long)l0;
  const int n = (int)std::floor(u0 - l0 + 0.5) + 1;
  *count = n;
  if (!out) return CSRST_OK;
  if (cap < n) return fail(h, CSRST_E_ARG, "line fields: output holds fewer than count samples");
  double *d = nullptr;
  CK(cudaMallocAsync(&d, (size_t)n * 7 * sizeof(double), h->s));
  if (h->fp32)
    launch_line_fields(h->order, h->Exf, h->Eyf, h->Hxf, h->Hyf, h->pitch32, h->cfg.Nx, h->cfg.Ny, h->winf,
                       h->wpitch, h->ws, with_current, h->b.org0, h->b.org1, h->b.hr0, h->b.hr1, h->dmean, i0, n, d,
                       h->s);
  else
    launch_line_fields(h->order, h->Ex, h->Ey, h->Hx, h->Hy, h->pitch, h->cfg.Nx, h->cfg.Ny, h->win, h->wpitch,
                       h->ws, with_current, h->b.org0, h->b.org1, h->b.hr0, h->b.hr1, h->dmean, i0, n, d, h->s);
  CK(cudaMemcpyAsync(out, d, (size_t)n * 7 * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  CK(cudaFreeAsync(d, h->s));
  CK(cudaStreamSynchronize(h->s));
  return check_err(h);
}

int csrst_diag_field_energy(csrst_handle *h, int with_window, double *out2) {
  if (!h || !out2) return CSRST_E_ARG;
  if (with_window) {
    const int rc = need_bunch(h);
    if (rc) return rc;
  }
  const double area = h->b.hr0 * h->b.hr1;
  if (h->fp32)
    launch_field_energy(h->Exf, h->Eyf, h->Hxf, h->Hyf, h->pitch32, h->cfg.Nx, h->cfg.Ny, h->winf, h->wpitch, h->ws,
                        with_window, area, h->dscratch, h->dout, h->s);
  else
    launch_field_energy(h->Ex, h->Ey, h->Hx, h->Hy, h->pitch, h->cfg.Nx, h->cfg.Ny, h->win, h->wpitch, h->ws,
                        with_window, area, h->dscratch, h->dout, h->s);
  CK(cudaMemcpyAsync(out2, h->dout, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  CK(cudaGetLastError());
  return CSRST_OK;
}

int csrst_diag_wake_async(csrst_handle *h, double *out_dev, int n, double *meta_dev) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!out_dev || !meta_dev || n != h->L0 - 4) return fail(h, CSRST_E_ARG, "wake buffer must hold L0 - 4 values");
  moments_async(h);
  if (h->fp32)
    launch_wake(h->ws, wplane32(h, 0).p, wplane32(h, 1).p, h->wpitch, h->L0, h->b.hr0, h->b.hr1, h->dmean, out_dev,
                h->s);
  else
    launch_wake(h->ws, wplane(h, 0).p, wplane(h, 1).p, h->wpitch, h->L0, h->b.hr0, h->b.hr1, h->dmean, out_dev, h->s);
  CK(cudaMemcpyAsync(meta_dev, &h->ws->mo0, 2 * sizeof(double), cudaMemcpyDeviceToDevice, h->s));
  CK(cudaMemcpyAsync(meta_dev + 2, h->dmean, 2 * sizeof(double), cudaMemcpyDeviceToDevice, h->s));
  return CSRST_OK;
}

// ---- batched ensemble ----

}  // extern "C"

namespace {

template <class T>
T *dev_copy(const std::vector<T> &v, cudaError_t &e) {
  T *p = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&p, (v.empty() ? 1 : v.size()) * sizeof(T));
  if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return p;
}

void part_free(EnsPart &P) {
  for (int k = 0; k < 2; ++k) {
    cudaFree(P.f64[k]); cudaFree(P.f32[k]);
    P.f64[k] = nullptr; P.f32[k] = nullptr;
    P.groups[k].clear();
  }
  for (void *p : P.blocks) cudaFree(p);
  P.blocks.clear();
  cudaFree(P.mv64); cudaFree(P.mv32); cudaFree(P.prep); cudaFree(P.bpre_sub);
  for (int k = 0; k < 2; ++k) {
    cudaFree(P.ytile[k]); cudaFree(P.yfix[k]); cudaFree(P.fey[k]); cudaFree(P.fmv[k]);
    P.ytile[k] = P.yfix[k] = P.fey[k] = P.fmv[k] = nullptr;
  }
  cudaFree(P.tpre); cudaFree(P.bpre_ey); cudaFree(P.queue);
  P.tpre = P.bpre_ey = nullptr;
  P.queue = nullptr;
  for (int k = 0; k < 3; ++k) { cudaFree(P.bpre_ex[k]); P.bpre_ex[k] = nullptr; }
  P.mv64 = nullptr; P.mv32 = nullptr; P.prep = nullptr; P.bpre_sub = nullptr;
  if (P.fork) cudaEventDestroy(P.fork);
  if (P.join) cudaEventDestroy(P.join);
  if (P.end) cudaEventDestroy(P.end);
  if (P.s2) cudaStreamDestroy(P.s2);
  if (P.s) cudaStreamDestroy(P.s);
  P.fork = P.join = P.end = nullptr;
  P.s = P.s2 = nullptr;
}

void ensemble_free_tables(csrst_ensemble *e) {
  if (e->s) cudaStreamSynchronize(e->s);
  for (EnsPart &P : e->parts) part_free(P);
  e->parts.clear();
  for (cudaGraphExec_t &g : e->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

int efail(csrst_ensemble *e, int code, const std::string &msg) {
  if (e) e->err = msg;
  else g_create_error = msg;
  return code;
}

// The fused sweep's tables of one part, for both plane-set parities: parity
// 0 reads the sets current now and writes the others, parity 1 the reverse;
// the window-Ey and move arguments are those of the set written.
template <class T>
cudaError_t part_build_fused_t(csrst_ensemble *e, EnsPart &P) {
  const int m = P.m;
  const size_t tb = yee_batch_bytes<T>(0), fb = yee_batch_bytes<T>(1);
  std::vector<uint8_t> tile[2], fix[2];
  std::vector<FieldArgsT<T>> fey[2];
  std::vector<MoveArgs<T>> fmv[2];
  std::vector<int> tpre(1, 0), bey(1, 0);
  for (int p = 0; p < 2; ++p) { tile[p].resize(tb * m); fix[p].resize(fb * m); }
  cudaError_t err = cudaSuccess;
  for (int k = 0; k < m && err == cudaSuccess; ++k) {
    csrst_handle *h = P.mem[k];
    for (int p = 0; p < 2; ++p) {  // each pass ends with the sets swapped: two passes restore them
      FieldArgsT<T> a;
      PlaneT<T> dst[4];
      if constexpr (sizeof(T) == 4) {
        a = field_args32(h, 0);
        dst[0] = {h->ExfB, h->pitch32}; dst[1] = {h->EyfB, h->pitch32};
        dst[2] = {h->HxfB, h->pitch32}; dst[3] = {h->HyfB, h->pitch32};
      } else {
        a = field_args(h, 0);
        dst[0] = {h->ExB, h->pitch}; dst[1] = {h->EyB, h->pitch}; dst[2] = {h->HxB, h->pitch}; dst[3] = {h->HyB, h->pitch};
      }
      int nt = 0;
      const int rc = yee_batch_entry<T>(a, dst, h->kind, h->kpitch, h->cutidx, static_cast<T *>(h->zfix), h->zpitch,
                                        h->zrows, g_staging_polls, tile[p].data() + tb * k, fix[p].data() + fb * k,
                                        &nt);
      if (rc != kOk) err = cudaErrorInvalidValue;
      if (p == 0) tpre.push_back(tpre.back() + nt);
      swap_sets(h);
      if constexpr (sizeof(T) == 4) {
        fey[p].push_back(field_args32(h, 1));
        fmv[p].push_back(MoveArgs<float>{field_args32(h, 0), h->scratchf, h->b.hr0, h->b.hr1});
      } else {
        fey[p].push_back(field_args(h, 1));
        fmv[p].push_back(MoveArgs<double>{field_args(h, 0), h->scratch, h->b.hr0, h->b.hr1});
      }
    }
    bey.push_back(bey.back() + (h->L0 * h->L1 + h->L1 + 2 + 255) / 256);
  }
  for (int p = 0; p < 2; ++p) {
    P.ytile[p] = dev_copy(tile[p], err);
    P.yfix[p] = dev_copy(fix[p], err);
    P.fey[p] = dev_copy(fey[p], err);
    P.fmv[p] = dev_copy(fmv[p], err);
  }
  P.tpre = dev_copy(tpre, err);
  P.bpre_ey = dev_copy(bey, err);
  P.ney = bey.back();
  if (err == cudaSuccess) err = cudaMalloc(&P.queue, sizeof(unsigned));
  return err;
}

cudaError_t part_build_fused(csrst_ensemble *e, EnsPart &P) {
  return e->fp32 ? part_build_fused_t<float>(e, P) : part_build_fused_t<double>(e, P);
}

// Argument tables of the steady-state step (pending drift, current boxes) of
// one part.
cudaError_t part_build(csrst_ensemble *e, EnsPart &P) {
  std::vector<FieldArgs> a64[2];
  std::vector<FieldArgsT<float>> a32[2];
  std::vector<MoveArgs<double>> mv64;
  std::vector<MoveArgs<float>> mv32;
  std::vector<PrepArgs> prep;
  std::vector<int> bsub(1, 0), bex[3];
  for (int k = 0; k < 3; ++k) bex[k].assign(1, 0);
  const long long cap = e->fp32 ? push32_batch_smem_limit() : push_batch_smem_limit();
  // per shape order: members, their push arguments, shared-memory fit, particle prefix
  struct Group {
    std::vector<PushArgs> p64[2];
    std::vector<Push32Args> p32[2];
    std::vector<unsigned char> ok;
    std::vector<long long> ppre{0};
    size_t smem = 0;
  } grp[3];
  P.particles = 0;
  for (csrst_handle *h : P.mem) {
    prep.push_back(prep_args(h->ws, h->b.hr0, h->b.hr1, h->order));
    Group &G = grp[h->order];
    G.ppre.push_back(G.ppre.back() + h->n);
    P.particles += h->n;
    const size_t tiles = push_tile_bytes(h->order);
    const size_t need = (size_t)h->L0 * h->L1 * sizeof(unsigned long long) + tiles;
    const bool fits = (long long)need <= cap;
    G.ok.push_back(fits ? 1 : 0);
    G.smem = std::max(G.smem, fits ? need : tiles);
    int nb = 0;
    for (int c = 0; c < 2; ++c) {
      if (e->fp32) {
        FieldArgsT<float> a = field_args32(h, c);
        a.tx = e->tx; a.ty = e->ty;
        nb = sub_grid(a);
        a32[c].push_back(a);
        Push32Args pa = push_args32(h, c);
        pa.pending = 1;
        G.p32[c].push_back(pa);
      } else {
        FieldArgs a = field_args(h, c);
        a.tx = e->tx; a.ty = e->ty;
        nb = sub_grid(a);
        a64[c].push_back(a);
        PushArgs pa = push_args(h, c);
        pa.pending = 1;
        G.p64[c].push_back(pa);
      }
    }
    if (e->fp32) mv32.push_back(MoveArgs<float>{a32[0].back(), h->scratchf, h->b.hr0, h->b.hr1});
    else mv64.push_back(MoveArgs<double>{a64[0].back(), h->scratch, h->b.hr0, h->b.hr1});
    bsub.push_back(bsub.back() + nb);
    for (int k = 0; k < 3; ++k) bex[k].push_back(bex[k].back() + (exchange_count(h->L0, h->L1, k) + 127) / 128);
  }
  cudaError_t err = cudaSuccess;
  for (int o = 0; o < 3; ++o) {
    Group &G = grp[o];
    const int gm = (int)G.ok.size();
    if (gm == 0) continue;
    unsigned char *ok = dev_copy(G.ok, err);
    long long *pp = dev_copy(G.ppre, err);
    P.blocks.push_back(ok);
    P.blocks.push_back(pp);
    for (int c = 0; c < 2; ++c) {
      void *args = e->fp32 ? (void *)dev_copy(G.p32[c], err) : (void *)dev_copy(G.p64[c], err);
      P.blocks.push_back(args);
      P.groups[c].push_back(PushGroup{o, gm, c, args, ok, pp, G.ppre.back(), 0, G.smem});
    }
  }
  for (int c = 0; c < 2; ++c) {
    if (e->fp32) P.f32[c] = dev_copy(a32[c], err);
    else P.f64[c] = dev_copy(a64[c], err);
  }
  if (e->fp32) P.mv32 = dev_copy(mv32, err);
  else P.mv64 = dev_copy(mv64, err);
  P.prep = dev_copy(prep, err);
  P.bpre_sub = dev_copy(bsub, err);
  for (int k = 0; k < 3; ++k) { P.bpre_ex[k] = dev_copy(bex[k], err); P.nex[k] = bex[k].back(); }
  P.nsub = bsub.back();
  if (e->fused && err == cudaSuccess) err = part_build_fused(e, P);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&P.s, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&P.s2, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&P.fork, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&P.join, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&P.end, cudaEventDisableTiming);
  return err;
}

// Splits the members into parts of about equal particle counts (largest
// first, each to the lightest part) and builds their tables.
int ensemble_build(csrst_ensemble *e) {
  ensemble_free_tables(e);
  // the fused sweep when the shape asks for it and every member allows it
  e->fused = e->tx == 0 && e->ty == 0;
  for (csrst_handle *h : e->mem)
    e->fused = e->fused && h->zfix && h->kind && !h->pml && !(h->cfg.flags & CSRST_FLAG_SUBSTEP_FIELDS);
  e->epar = 0;
  if (e->push_grid <= 0) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e->push_grid = 2 * sms;
  }
  const int np = std::max(1, std::min(e->nparts, e->m));
  e->parts.resize(np);
  std::vector<int> idx(e->m);
  for (int k = 0; k < e->m; ++k) idx[k] = k;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return e->mem[a]->n > e->mem[b]->n; });
  std::vector<long long> load(np, 0);
  std::vector<std::vector<int>> pick(np);
  for (int k : idx) {
    const int p = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    pick[p].push_back(k);
    load[p] += e->mem[k]->n;
  }
  long long all = 0;
  for (int p = 0; p < np; ++p) {
    std::sort(pick[p].begin(), pick[p].end());  // members in their given order
    for (int k : pick[p]) e->parts[p].mem.push_back(e->mem[k]);
    e->parts[p].m = (int)pick[p].size();
    all += load[p];
  }
  for (EnsPart &P : e->parts) {
    const cudaError_t c = part_build(e, P);
    if (c != cudaSuccess) return efail(e, CSRST_E_CUDA, std::string("ensemble tables: ") + cudaGetErrorString(c));
    P.push_grid = std::max(1, (int)((long long)e->push_grid * P.particles / (all > 0 ? all : 1)));
    for (int c = 0; c < 2; ++c)
      for (PushGroup &G : P.groups[c]) G.all = P.particles;
  }
  return CSRST_OK;
}

// The push of every member of a part: the shape-order groups run side by side
// on two streams, after the per-member preparation and before the bounds.
void part_push(csrst_ensemble *e, EnsPart &P, int jcomp) {
  const std::vector<PushGroup> &G = P.groups[jcomp];
  const int ng = (int)G.size();
  auto batch = [&](const PushGroup *g, int n, int grid, const PrepArgs *prep, cudaStream_t st, int parts) {
    if (e->fp32) launch_push32_batch(g, n, P.m, grid, prep, st, parts);
    else launch_push_batch(g, n, P.m, grid, prep, st, parts);
  };
  if (ng <= 1) {
    batch(G.data(), ng, P.push_grid, P.prep, P.s, 3);
    return;
  }
  batch(nullptr, 0, 0, P.prep, P.s, 1);
  cudaEventRecord(P.fork, P.s);
  cudaStreamWaitEvent(P.s2, P.fork, 0);
  for (int g = 0; g < ng; ++g) batch(&G[g], 1, P.push_grid, nullptr, (g & 1) ? P.s2 : P.s, 0);
  cudaEventRecord(P.join, P.s2);
  cudaStreamWaitEvent(P.s, P.join, 0);
  batch(nullptr, 0, 0, P.prep, P.s, 2);
}

template <class T>
void part_fields_fused(const csrst_ensemble *e, EnsPart &P, int half) {
  const int p = e->epar;
  if (half == 0) {  // the static sweep of the whole step and the window's half H, Ex, half H
    launch_yee_batch<T>(P.ytile[p], P.yfix[p], P.tpre, P.m, P.queue, P.s);
  } else {          // the window's Ey (after the second push), then the window move
    launch_window_ey_batch<T>(static_cast<const FieldArgsT<T> *>(P.fey[p]), P.bpre_ey, P.m, P.ney, P.s);
    launch_move_batch<T>(static_cast<const MoveArgs<T> *>(P.fmv[p]), P.m, P.s);
  }
}

template <class T>
void part_fields(EnsPart &P, const FieldArgsT<T> *a0, const FieldArgsT<T> *a1, const MoveArgs<T> *mv, int half) {
  if (half == 0) {  // half H, Ex, half H (after the first push)
    launch_half_h_batch(a0, P.bpre_sub, P.m, P.nsub, P.s);
    launch_exchange_batch(a0, P.bpre_ex[0], P.m, P.nex[0], 0, P.s);
    launch_update_e_batch(a0, P.bpre_sub, P.m, P.nsub, 0, P.s);
    launch_exchange_batch(a0, P.bpre_ex[1], P.m, P.nex[1], 1, P.s);
    launch_half_h_batch(a0, P.bpre_sub, P.m, P.nsub, P.s);
    launch_exchange_batch(a0, P.bpre_ex[0], P.m, P.nex[0], 0, P.s);
  } else {          // Ey (after the second push), then the window move
    launch_update_e_batch(a1, P.bpre_sub, P.m, P.nsub, 1, P.s);
    launch_exchange_batch(a1, P.bpre_ex[2], P.m, P.nex[2], 2, P.s);
    launch_move_batch(mv, P.m, P.s);
  }
}

// The host's view of a fused step: every member's plane sets swap.
void ensemble_swap(csrst_ensemble *e) {
  for (csrst_handle *h : e->mem) swap_sets(h);
  e->epar ^= 1;
}

// One steady-state time step of every member (main.cpp:390-506), all parts
// side by side, joined back on the ensemble stream.
void ensemble_step_async(csrst_ensemble *e) {
  cudaEventRecord(e->fork, e->s);
  for (EnsPart &P : e->parts) {
    cudaStreamWaitEvent(P.s, e->fork, 0);
    for (int half = 0; half < 2; ++half) {
      part_push(e, P, half);
      if (e->fused) {
        if (e->fp32) part_fields_fused<float>(e, P, half);
        else part_fields_fused<double>(e, P, half);
      } else if (e->fp32) {
        part_fields(P, P.f32[0], P.f32[1], P.mv32, half);
      } else {
        part_fields(P, P.f64[0], P.f64[1], P.mv64, half);
      }
    }
    cudaEventRecord(P.end, P.s);
    cudaStreamWaitEvent(e->s, P.end, 0);
  }
  if (e->fused) ensemble_swap(e);
}

// Brings every member to the steady state of the loop (the stored positions
// owe the trailing drift, the box of the next gather positions is current)
// with single-member steps, then hands the members to the ensemble stream.
int ensemble_steady(csrst_ensemble *e, int &nsteps) {
  while (nsteps > 0) {
    bool all = true;
    for (csrst_handle *h : e->mem) all = all && h->pending && h->bb == kBBValid;
    if (all) break;
    for (csrst_handle *h : e->mem) step_async(h);
    --nsteps;
  }
  for (csrst_handle *h : e->mem) {
    cudaError_t c = cudaStreamSynchronize(h->s);
    if (c != cudaSuccess) return efail(e, CSRST_E_CUDA, std::string("member stream: ") + cudaGetErrorString(c));
  }
  return CSRST_OK;
}

void ensemble_mark(csrst_ensemble *e) {
  for (csrst_handle *h : e->mem) {
    h->pending = true;
    h->bb = kBBValid;
    h->fresh = false;
    h->acc_fresh[0] = h->acc_fresh[1] = false;
  }
}

// Member streams wait for the ensemble's work before anything else.
int ensemble_release(csrst_ensemble *e) {
  cudaError_t c = cudaEventRecord(e->done, e->s);
  for (csrst_handle *h : e->mem)
    if (c == cudaSuccess) c = cudaStreamWaitEvent(h->s, e->done, 0);
  if (c != cudaSuccess) return efail(e, CSRST_E_CUDA, std::string("ensemble release: ") + cudaGetErrorString(c));
  return CSRST_OK;
}

}  // namespace

extern "C" {

int csrst_ensemble_create(csrst_handle *const *members, int m, csrst_ensemble **out) {
  if (!out || !members || m <= 0) return efail(nullptr, CSRST_E_ARG, "ensemble: no members");
  *out = nullptr;
  csrst_ensemble *e = new csrst_ensemble;
  e->m = m;
  for (int k = 0; k < m; ++k) {
    csrst_handle *h = members[k];
    if (!h || h->n <= 0 || !(h->win || h->winf)) {
      delete e;
      return efail(nullptr, CSRST_E_NO_PARTICLES, "ensemble: member " + std::to_string(k) + " has no bunch");
    }
    if (k > 0 && h->fp32 != e->fp32) {
      delete e;
      return efail(nullptr, CSRST_E_ARG, "ensemble: members must share one precision mode");
    }
    if (h->cfg.flags & CSRST_FLAG_KEEP_OLD) {
      delete e;
      return efail(nullptr, CSRST_E_ARG, "ensemble: CSRST_FLAG_KEEP_OLD members cannot be batched");
    }
    e->fp32 = h->fp32;
    e->mem.push_back(h);
  }
  if (cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
    csrst_ensemble_destroy(e);
    return efail(nullptr, CSRST_E_CUDA, "ensemble: stream");
  }
  // the argument tables hold the members' plane pointers: their single
  // steps keep to the sub-step kernels (no plane-set swap) from here on
  for (csrst_handle *h : e->mem) ++h->ens_refs;
  e->holds = true;
  const int rc = ensemble_build(e);
  if (rc) {
    g_create_error = e->err;
    csrst_ensemble_destroy(e);
    return rc;
  }
  *out = e;
  return CSRST_OK;
}

int csrst_ensemble_destroy(csrst_ensemble *e) {
  if (!e) return CSRST_OK;
  if (e->holds)
    for (csrst_handle *h : e->mem) --h->ens_refs;
  ensemble_free_tables(e);
  if (e->done) cudaEventDestroy(e->done);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->s) cudaStreamDestroy(e->s);
  delete e;
  return CSRST_OK;
}

int csrst_ensemble_get_error(const csrst_ensemble *e, char *buf, size_t len) {
  if (!buf || len == 0) return CSRST_E_ARG;
  std::snprintf(buf, len, "%s", (e ? e->err : g_create_error).c_str());
  return CSRST_OK;
}

void *csrst_ensemble_stream(csrst_ensemble *e) { return e ? (void *)e->s : nullptr; }

int csrst_ensemble_step(csrst_ensemble *e, int nsteps) {
  if (!e || nsteps < 0) return efail(e, CSRST_E_ARG, "ensemble step: invalid arguments");
  int rc = ensemble_steady(e, nsteps);
  if (rc) return rc;
  if (nsteps > 0) {
    for (int k = 0; k < nsteps; ++k) {
      const int p = e->epar;
      if (!e->graph[p]) {  // recorded on the first step from this parity (the recording swaps the host's view)
        cudaGraph_t g;
        if (cudaStreamBeginCapture(e->s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
          return efail(e, CSRST_E_CUDA, "ensemble graph capture");
        ensemble_step_async(e);
        if (cudaStreamEndCapture(e->s, &g) != cudaSuccess) return efail(e, CSRST_E_CUDA, "ensemble graph capture");
        const cudaError_t c = cudaGraphInstantiate(&e->graph[p], g, 0);
        cudaGraphDestroy(g);
        if (c != cudaSuccess) return efail(e, CSRST_E_CUDA, std::string("ensemble graph: ") + cudaGetErrorString(c));
      } else if (e->fused) {
        ensemble_swap(e);
      }
      if (cudaGraphLaunch(e->graph[p], e->s) != cudaSuccess) return efail(e, CSRST_E_CUDA, "ensemble graph launch");
    }
    ensemble_mark(e);
  }
  return ensemble_release(e);
}

// Sticky device errors of all members: the first member with one, or 0.
int csrst_ensemble_sync(csrst_ensemble *e, int *bad_member) {
  if (!e) return CSRST_E_ARG;
  if (bad_member) *bad_member = -1;
  if (cudaStreamSynchronize(e->s) != cudaSuccess) return efail(e, CSRST_E_CUDA, "ensemble stream");
  for (int k = 0; k < e->m; ++k) {
    const int rc = csrst_sync(e->mem[k]);
    if (rc) {
      if (bad_member) *bad_member = k;
      return efail(e, rc, "member " + std::to_string(k) + ": " + e->mem[k]->err);
    }
  }
  return CSRST_OK;
}

// Launch shapes: CTAs of the batched push over all parts (0 = two per SM),
// the static-sweep tile (tx * ty = 256) and the number of parts that run side
// by side.  Results do not depend on them.
int csrst_ensemble_set_shape(csrst_ensemble *e, int push_ctas, int tx, int ty, int parts) {
  if (!e || push_ctas < 0 || parts < 1 || !((tx == 0 && ty == 0) || (tx > 0 && ty > 0 && tx * ty == 256)))
    return efail(e, CSRST_E_ARG, "invalid shape");
  if (cudaStreamSynchronize(e->s) != cudaSuccess) return efail(e, CSRST_E_CUDA, "ensemble stream");
  e->push_grid = push_ctas;
  e->tx = tx; e->ty = ty;
  e->nparts = parts;
  return ensemble_build(e);
}

// The autotuner: times `steps` steady-state steps (events on the ensemble
// stream, launched eagerly) for each candidate shape and keeps the fastest.
// The timed steps are real steps of the members.  report: rows of
// (push_ctas, tx, ty, parts, ms per step); *nrows receives the row count.
int csrst_ensemble_tune(csrst_ensemble *e, int steps, double *report, int max_rows, int *nrows) {
  if (!e || steps < 1) return efail(e, CSRST_E_ARG, "tune: invalid arguments");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int warm = 1;
  int rc = ensemble_steady(e, warm);
  if (rc) return rc;
  const int ctas[3] = {4 * sms, 16 * sms, 32 * sms};
  const int tiles[3][2] = {{0, 0}, {32, 8}, {128, 2}};  // the fused sweep, the sub-step tiles
  const int parts[3] = {1, 2, 4};
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  float best = 1e30f;
  int bc = 2 * sms, bt = 0, bp = 1, rows = 0;
  for (int pa = 0; pa < 3; ++pa)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        e->push_grid = ctas[a];
        e->tx = tiles[b][0]; e->ty = tiles[b][1];
        e->nparts = parts[pa];
        if ((rc = ensemble_build(e))) return rc;
        ensemble_step_async(e);  // untimed warm-up of this shape
        cudaEventRecord(t0, e->s);
        for (int k = 0; k < steps; ++k) ensemble_step_async(e);
        cudaEventRecord(t1, e->s);
        if (cudaEventSynchronize(t1) != cudaSuccess) return efail(e, CSRST_E_CUDA, "tune: timing");
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        ms /= steps;
        if (report && rows < max_rows) {
          double *r = report + 5 * rows;
          r[0] = ctas[a]; r[1] = tiles[b][0]; r[2] = tiles[b][1]; r[3] = parts[pa]; r[4] = ms;
        }
        ++rows;
        if (ms < best) { best = ms; bc = ctas[a]; bt = b; bp = parts[pa]; }
      }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  ensemble_mark(e);
  e->push_grid = bc;
  e->tx = tiles[bt][0]; e->ty = tiles[bt][1];
  e->nparts = bp;
  if (nrows) *nrows = rows < max_rows ? rows : max_rows;
  if ((rc = ensemble_build(e))) return rc;
  return ensemble_release(e);
}

// ---- absorbing layers at the open ends ----

}  // extern "C"

namespace {

// Conductivity of the absorbing layers of thickness W at the point (x, y),
// split along the pipe axis into sx, sy: the layers at the entry plane x = 0
// of the first straight section (axis +x) and at the end plane of the second
// (the centreline's end: the arc of radius R and angle |phi| about the bend
// centre of Bend::Init, then length_after along the outgoing axis).  Each
// layer stops kPmlGap cells before its end plane: a slanted end wall is made
// of conformal cut cells, and a strongly damped layer cell next to them made
// the coupled update grow without bound, while a regular strip in between
// keeps it stable.  sigma(depth) = smax (depth / W)^m.
constexpr double kPmlGap = 2.0;
void pml_sigma(const BendDev &b, double W, int m, double smax, double x, double y, double *sx, double *sy) {
  *sx = 0.0; *sy = 0.0;
  const double gap = kPmlGap * b.hr0;
  const double din = x - gap;  // distance from the entry plane, past the gap
  if (din >= 0.0 && din < W) *sx += smax * std::pow((W - din) / W, m);
  const double ph = std::fabs(b.phi);
  const double ry = 0.5 * b.w - b.cen1;  // bend entry relative to the centre: (0, ry), |ry| = R
  const double sg = ry > 0.0 ? -1.0 : 1.0;
  const double t0 = std::cos(ph), t1 = sg * std::sin(ph);
  const double e0 = b.cen0 + b.R * std::sin(ph) + b.La * t0;
  const double e1 = b.cen1 - sg * b.R * std::cos(ph) + b.La * t1;
  const double dout = (e0 - x) * t0 + (e1 - y) * t1 - gap;  // from the end plane, past the gap
  if (dout >= 0.0 && dout < W) {
    const double v = smax * std::pow((W - dout) / W, m);
    *sx += v * std::fabs(t0);
    *sy += v * std::fabs(t1);
  }
}

// The convolution's recursion over the update interval dt':
// b = exp(-sigma dt'/eps0), a = b - 1.
void pml_coef(double sigma, double dtp, double *b, double *a) {
  if (!(sigma > 0.0)) { *b = 1.0; *a = 0.0; return; }
  *b = std::exp(-sigma * dtp / kEps0);
  *a = *b - 1.0;
}

}  // namespace

extern "C" {

int csrst_set_pml(csrst_handle *h, int width, int order, double reflection) {
  if (!h) return CSRST_E_ARG;
  if (width < 0 || width > 1000 || order < 0 || order > 8 || (width > 0 && !(reflection > 0 && reflection < 1)))
    return fail(h, CSRST_E_ARG, "absorbing layer: width 0..1000 cells, order 0..8, reflection in (0, 1)");
  CK(cudaStreamSynchronize(h->s));
  cudaFree(h->pml); cudaFree(h->pml32); cudaFree(h->pml_rows); cudaFree(h->psi);
  h->pml = nullptr; h->pml32 = nullptr; h->pml_rows = nullptr; h->psi = nullptr; h->npml = 0;
  drop_graphs(h);
  if (width == 0) return CSRST_OK;
  const int Nx = h->b.Nx, Ny = h->b.Ny;
  std::vector<uint8_t> inside((size_t)Nx * Ny);
  CK(cudaMemcpy(inside.data(), h->mask, inside.size(), cudaMemcpyDeviceToHost));
  const FieldArgs f = field_args(h, 0);
  const double h0 = h->b.hr0, h1 = h->b.hr1, o0 = h->b.org0, o1 = h->b.org1, dt = h->dt;
  const double W = width * h0;
  const double smax = -(order + 1) * kEps0 * kC * std::log(reflection) / (2.0 * W);
  // per row: the regular sweep's columns [lo, hi); the cells outside them are the layer's
  std::vector<int2> rows(Ny);
  std::vector<PmlCellT<double>> cells;
  for (int j = 0; j < Ny; ++j) {
    int lo = 0, hi = Nx;
    for (int i = 0; i < Nx; ++i) {
      if (!inside[(size_t)j * Nx + i]) continue;
      double sx, sy, tx, ty, ux, uy;
      pml_sigma(h->b, W, order, smax, o0 + (i + 0.5) * h0, o1 + (j + 0.5) * h1, &sx, &sy);   // Hz
      pml_sigma(h->b, W, order, smax, o0 + (i + 0.5) * h0, o1 + j * h1, &tx, &ty);           // Ex
      pml_sigma(h->b, W, order, smax, o0 + i * h0, o1 + (j + 0.5) * h1, &ux, &uy);           // Ey
      if (sx > 0 || sy > 0 || ty > 0 || ux > 0) {
        if (i < Nx / 2) lo = std::max(lo, i + 1);
        else hi = std::min(hi, i);
      }
    }
    if (hi < lo) hi = lo;
    rows[j] = make_int2(lo, hi);
    for (int i = 0; i < Nx; ++i) {
      if (!inside[(size_t)j * Nx + i] || (i >= lo && i < hi)) continue;
      double sx, sy, tx, ty, ux, uy;
      pml_sigma(h->b, W, order, smax, o0 + (i + 0.5) * h0, o1 + (j + 0.5) * h1, &sx, &sy);
      pml_sigma(h->b, W, order, smax, o0 + (i + 0.5) * h0, o1 + j * h1, &tx, &ty);
      pml_sigma(h->b, W, order, smax, o0 + i * h0, o1 + (j + 0.5) * h1, &ux, &uy);
      PmlCellT<double> c{};
      c.i = i; c.j = j;
      pml_coef(sx, 0.5 * dt, &c.bhx, &c.ahx);
      pml_coef(sy, 0.5 * dt, &c.bhy, &c.ahy);
      pml_coef(ty, dt, &c.bex, &c.aex);
      pml_coef(ux, dt, &c.bey, &c.aey);
      cells.push_back(c);
    }
  }
  std::vector<PmlCellT<float>> c32(cells.size());
  for (size_t k = 0; k < cells.size(); ++k) {
    const PmlCellT<double> &c = cells[k];
    c32[k] = PmlCellT<float>{c.i, c.j, (float)c.bhx, (float)c.ahx, (float)c.bhy, (float)c.ahy,
                             (float)c.bex, (float)c.aex, (float)c.bey, (float)c.aey};
  }
  h->npml = (int)cells.size();
  CK(cudaMalloc(&h->pml_rows, rows.size() * sizeof(int2)));
  CK(cudaMemcpy(h->pml_rows, rows.data(), rows.size() * sizeof(int2), cudaMemcpyHostToDevice));
  if (h->npml > 0) {
    CK(cudaMalloc(&h->pml, cells.size() * sizeof(PmlCellT<double>)));
    CK(cudaMemcpy(h->pml, cells.data(), cells.size() * sizeof(PmlCellT<double>), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&h->pml32, c32.size() * sizeof(PmlCellT<float>)));
    CK(cudaMemcpy(h->pml32, c32.data(), c32.size() * sizeof(PmlCellT<float>), cudaMemcpyHostToDevice));
    const size_t pb = 4 * cells.size() * (h->fp32 ? sizeof(float) : sizeof(double));
    CK(cudaMalloc(&h->psi, pb));
    CK(cudaMemset(h->psi, 0, pb));
  }
  // a loaded window must not overlap a layer
  if (h->win || h->winf) {
    if (h->fp32) launch_check_window(field_args32(h, 0), h->s);
    else launch_check_window(field_args(h, 0), h->s);
    return check_err(h);
  }
  return CSRST_OK;
}

int csrst_get_pml(csrst_handle *h, int *ncells, int *rows2) {
  if (!h || !ncells) return CSRST_E_ARG;
  *ncells = h->npml;
  if (rows2) {
    if (h->pml_rows) {
      CK(cudaMemcpy(rows2, h->pml_rows, (size_t)h->b.Ny * sizeof(int2), cudaMemcpyDeviceToHost));
    } else {
      for (int j = 0; j < h->b.Ny; ++j) { rows2[2 * j] = 0; rows2[2 * j + 1] = h->b.Nx; }
    }
  }
  return CSRST_OK;
}

// ---- stand-alone ScatterGatherImpl / ShapeFunction entry points ----

int csrst_gather(int order, int comp, const double *patch, int nx, int ny, const double *o2, const double *hh2,
                 const double *x, const double *y, size_t n, double *out) {
  csrst_handle *h = nullptr;
  if (order < 0 || order > 2 || comp < 0 || comp > 2 || !patch || nx <= 0 || ny <= 0 || !o2 || !hh2)
    return fail(h, CSRST_E_ARG, "invalid gather arguments");
  if (n == 0) return CSRST_OK;
  double *dp, *dx, *dy, *dout;
  CK(cudaMalloc(&dp, (size_t)nx * ny * 8)); CK(cudaMalloc(&dx, n * 8)); CK(cudaMalloc(&dy, n * 8));
  CK(cudaMalloc(&dout, n * 8));
  CK(cudaMemcpy(dp, patch, (size_t)nx * ny * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dx, x, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dy, y, n * 8, cudaMemcpyHostToDevice));
  launch_gather(order, comp, dp, nx, o2[0], o2[1], hh2[0], hh2[1], dx, dy, (long long)n, dout, 0);
  CK(cudaMemcpy(out, dout, n * 8, cudaMemcpyDeviceToHost));
  cudaFree(dp); cudaFree(dx); cudaFree(dy); cudaFree(dout);
  CK(cudaGetLastError());
  return CSRST_OK;
}

static int run_fixed(int kind, int order, int comp, const double *ox, const double *oy, const double *x,
                     const double *y, const double *q, size_t n, const double *o2, const double *hh2, double dt,
                     int i0, int j0, int ni, int nj, double scale, double *J) {
  csrst_handle *h = nullptr;
  if (order < 0 || order > 2 || ni <= 0 || nj <= 0 || !o2 || !hh2 || !J || !(scale > 0))
    return fail(h, CSRST_E_ARG, "invalid deposit arguments");
  const size_t m = (size_t)ni * nj;
  unsigned long long *acc;
  double *dJ;
  int *derr;  // crossing overflow, dropped contribution
  CK(cudaMalloc(&acc, m * 8)); CK(cudaMalloc(&dJ, m * 8)); CK(cudaMalloc(&derr, 8));
  CK(cudaMemset(acc, 0, m * 8)); CK(cudaMemset(derr, 0, 8));
  double *d[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  const double *s[5] = {ox, oy, x, y, q};
  if (n > 0)
    for (int k = 0; k < 5; ++k) {
      CK(cudaMalloc(&d[k], n * 8));
      CK(cudaMemcpy(d[k], s[k], n * 8, cudaMemcpyHostToDevice));
    }
  if (kind == 0)
    launch_deposit(order, comp, d[0], d[1], d[2], d[3], d[4], (long long)n, o2[0], o2[1], hh2[0], hh2[1], dt,
                   i0, j0, ni, nj, acc, scale, derr, 0);
  else
    launch_charge_diff(order, d[0], d[1], d[2], d[3], d[4], (long long)n, o2[0], o2[1], hh2[0], hh2[1], i0, j0,
                       ni, nj, acc, scale, derr + 1, 0);
  launch_fixed_to_double(acc, dJ, (long long)m, 1.0 / scale, 0);
  int e[2] = {0, 0};
  CK(cudaMemcpy(J, dJ, m * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(e, derr, 8, cudaMemcpyDeviceToHost));
  if (kind == 1)
    for (size_t k = 0; k < m; ++k) J[k] = J[k] / (hh2[0] * hh2[1]);
  cudaFree(acc); cudaFree(dJ); cudaFree(derr);
  for (double *p : d) cudaFree(p);
  CK(cudaGetLastError());
  if (e[0]) return fail(h, e[0], "too many cell-border crossings");
  if (e[1]) {
    fail(h, CSRST_W_OUTSIDE, "contributions outside the patch were dropped");
    return CSRST_W_OUTSIDE;
  }
  return CSRST_OK;
}

int csrst_deposit(int order, int comp, const double *ox, const double *oy, const double *x, const double *y,
                  const double *q, size_t n, const double *o2, const double *hh2, double dt, int i0, int j0,
                  int ni, int nj, double scale, double *J) {
  if (comp != 0 && comp != 1) return fail(nullptr, CSRST_E_ARG, "comp must be 0 or 1");
  return run_fixed(0, order, comp, ox, oy, x, y, q, n, o2, hh2, dt, i0, j0, ni, nj, scale, J);
}

int csrst_charge_diff(int order, const double *ox, const double *oy, const double *x, const double *y,
                      const double *q, size_t n, const double *o2, const double *hh2, int i0, int j0, int ni,
                      int nj, double scale, double *rho) {
  return run_fixed(1, order, 0, ox, oy, x, y, q, n, o2, hh2, 0.0, i0, j0, ni, nj, scale, rho);
}

int csrst_flux32(int order, int comp, const int *cell0, const float *a0, const float *a1, const int *cell1,
                 const float *b0, const float *b1, const float *q, size_t n, double scale, int i0, int j0, int ni,
                 int nj, long long *F, long long *drho) {
  csrst_handle *h = nullptr;
  if (order < 0 || order > 2 || (comp != 0 && comp != 1) || ni <= 0 || nj <= 0 || !F || !(scale > 0) ||
      (n > 0 && (!cell0 || !a0 || !a1 || !cell1 || !b0 || !b1 || !q)))
    return fail(h, CSRST_E_ARG, "invalid flux arguments");
  const size_t m = (size_t)ni * nj;
  unsigned long long *dF = nullptr, *dR = nullptr;
  int *derr = nullptr;
  CK(cudaMalloc(&dF, m * 8)); CK(cudaMemset(dF, 0, m * 8));
  if (drho) { CK(cudaMalloc(&dR, m * 8)); CK(cudaMemset(dR, 0, m * 8)); }
  CK(cudaMalloc(&derr, 8)); CK(cudaMemset(derr, 0, 8));
  void *d[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  const void *src[7] = {cell0, a0, a1, cell1, b0, b1, q};
  if (n > 0)
    for (int k = 0; k < 7; ++k) {
      CK(cudaMalloc(&d[k], n * 4));
      CK(cudaMemcpy(d[k], src[k], n * 4, cudaMemcpyHostToDevice));
    }
  launch_flux32(order, comp, (const int *)d[0], (const float *)d[1], (const float *)d[2], (const int *)d[3],
                (const float *)d[4], (const float *)d[5], (const float *)d[6], (long long)n, scale, i0, j0, ni, nj, dF,
                dR, derr, 0);
  int e[2] = {0, 0};
  CK(cudaMemcpy(F, dF, m * 8, cudaMemcpyDeviceToHost));
  if (drho) CK(cudaMemcpy(drho, dR, m * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(e, derr, 8, cudaMemcpyDeviceToHost));
  cudaFree(dF); cudaFree(dR); cudaFree(derr);
  for (void *p : d) cudaFree(p);
  CK(cudaGetLastError());
  if (e[0]) return fail(h, e[0], "a move spans more than one cell on an axis");
  if (e[1]) {
    fail(h, CSRST_W_OUTSIDE, "contributions outside the patch were dropped");
    return CSRST_W_OUTSIDE;
  }
  return CSRST_OK;
}

int csrst_get_bunch32(csrst_handle *h, int which, int *cell, float *o0, float *o1, float *d0, float *d1, float *q) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!h->fp32) return fail(h, CSRST_E_ARG, "csrst_get_bunch32 reads an FP32-mode bunch");
  if (which != 0 && which != 1) return fail(h, CSRST_E_ARG, "which must be 0 (bunch) or 1 (start of the last move)");
  if (which == 1 && !h->old_cell)
    return fail(h, CSRST_E_ARG, "create the handle with CSRST_FLAG_KEEP_OLD to keep the start of each move");
  if (which == 1 && (d0 || d1 || q)) return fail(h, CSRST_E_ARG, "the start of a move has no momentum or charge");
  const size_t n4 = (size_t)h->n * 4;
  const void *src[6] = {which ? (const void *)h->old_cell : h->b32.cell, which ? (const void *)h->old_o0 : h->b32.ox,
                        which ? (const void *)h->old_o1 : h->b32.oy, h->b32.dpx, h->b32.dpy, h->b32.q};
  void *dst[6] = {cell, o0, o1, d0, d1, q};
  for (int k = 0; k < 6; ++k)
    if (dst[k]) CK(cudaMemcpyAsync(dst[k], src[k], n4, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CSRST_OK;
}

}  // extern "C"

// ---- checkpoint / restart ----

namespace {

constexpr char kCkMagic[8] = {'C', 'S', 'R', 'S', 'T', 'C', 'K', '1'};
constexpr char kCkEnd[8] = {'C', 'S', 'R', 'S', 'T', 'E', 'N', 'D'};
constexpr uint32_t kCkVersion = 2;  // 2: FP32 mode's current accumulator holds flux units

bool ck_put(FILE *f, const void *p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }
bool ck_get(FILE *f, void *p, size_t n) { return n == 0 || std::fread(p, 1, n, f) == n; }

bool ck_put_dev(FILE *f, const void *d, size_t n, std::vector<unsigned char> &buf, cudaStream_t s) {
  if (n == 0) return true;
  buf.resize(n);
  if (cudaMemcpyAsync(buf.data(), d, n, cudaMemcpyDeviceToHost, s) != cudaSuccess) return false;
  if (cudaStreamSynchronize(s) != cudaSuccess) return false;
  return ck_put(f, buf.data(), n);
}

bool ck_get_dev(FILE *f, void *d, size_t n, std::vector<unsigned char> &buf, cudaStream_t s) {
  if (n == 0) return true;
  buf.resize(n);
  if (!ck_get(f, buf.data(), n)) return false;
  if (cudaMemcpyAsync(d, buf.data(), n, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
  return cudaStreamSynchronize(s) == cudaSuccess;
}

// The state a time step reads and writes, as (device pointer, bytes) in file order.
struct CkPlan {
  std::vector<std::pair<void *, size_t>> planes, window, bunch;
};

CkPlan ck_plan(csrst_handle *h) {
  CkPlan P;
  const size_t ny = (size_t)h->cfg.Ny + 2;
  if (h->fp32) {
    for (float *p : {h->Exf, h->Eyf, h->Hxf, h->Hyf}) P.planes.push_back({p, (size_t)h->pitch32 * ny * 4});
  } else {
    for (double *p : {h->Ex, h->Ey, h->Hx, h->Hy}) P.planes.push_back({p, (size_t)h->pitch * ny * 8});
  }
  const size_t wp = (size_t)h->wpitch * (h->L1 + 2);
  P.window.push_back({h->ws, sizeof(WinState)});
  P.window.push_back({h->fp32 ? (void *)h->winf : (void *)h->win, 6 * wp * (h->fp32 ? 4 : 8)});
  P.window.push_back({h->acc, 2 * (size_t)h->L0 * h->L1 * sizeof(unsigned long long)});
  const size_t n = (size_t)h->n;
  if (h->fp32) {
    P.bunch.push_back({h->b32.cell, n * 4});
    for (float *p : {h->b32.ox, h->b32.oy, h->b32.dpx, h->b32.dpy, h->b32.q}) P.bunch.push_back({p, n * 4});
  } else {
    for (double *p : {h->x, h->y, h->px, h->py, h->q, h->ox, h->oy}) P.bunch.push_back({p, n * 8});
  }
  return P;
}

}  // namespace

extern "C" {

int csrst_get_num_particles(csrst_handle *h, long long *n) {
  if (!h || !n) return CSRST_E_ARG;
  *n = h->n;
  return CSRST_OK;
}

int csrst_checkpoint_write(csrst_handle *h, const char *path, long long step, double time) {
  int rc = need_bunch(h);
  if (rc) return rc;
  if (!path) return fail(h, CSRST_E_ARG, "checkpoint: no path");
  CK(cudaStreamSynchronize(h->s));
  if ((rc = check_err(h))) return rc;  // a run that stopped on a device error is not saved
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(h, CSRST_E_IO, std::string("checkpoint: cannot open ") + path);
  std::vector<unsigned char> buf;
  const CkPlan P = ck_plan(h);
  const uint32_t head[2] = {kCkVersion, h->fp32 ? 1u : 0u};
  const int32_t win[3] = {h->L0, h->L1, h->wpitch};
  const uint8_t flags[4] = {(uint8_t)h->pending, (uint8_t)h->fresh, (uint8_t)h->acc_fresh[0],
                            (uint8_t)h->acc_fresh[1]};
  const int32_t bb = (int32_t)h->bb;
  const double mom[2] = {h->P0, h->P1};
  bool ok = ck_put(f, kCkMagic, 8) && ck_put(f, head, sizeof(head)) && ck_put(f, &h->cfg, sizeof(csrst_config)) &&
            ck_put(f, &step, 8) && ck_put(f, &time, 8);
  for (auto &pl : P.planes) ok = ok && ck_put_dev(f, pl.first, pl.second, buf, h->s);
  ok = ok && ck_put(f, win, sizeof(win)) && ck_put(f, &h->acc_scale, 8);
  for (auto &pl : P.window) ok = ok && ck_put_dev(f, pl.first, pl.second, buf, h->s);
  ok = ok && ck_put(f, &h->n, 8) && ck_put(f, flags, sizeof(flags)) && ck_put(f, &bb, 4) && ck_put(f, mom, 16);
  for (auto &pl : P.bunch) ok = ok && ck_put_dev(f, pl.first, pl.second, buf, h->s);
  ok = ok && ck_put(f, kCkEnd, 8);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? CSRST_OK : fail(h, CSRST_E_IO, std::string("checkpoint: writing ") + path + " failed");
}

int csrst_checkpoint_read(csrst_handle *h, const char *path, long long *step, double *time) {
  if (!h || !path) return CSRST_E_ARG;
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(h, CSRST_E_IO, std::string("restart: cannot open ") + path);
  auto bad = [&](int code, const std::string &why) {
    std::fclose(f);
    return fail(h, code, "restart: " + why);
  };
  char magic[8];
  uint32_t head[2];
  csrst_config cfg{};
  long long st = 0;
  double tm = 0;
  if (!ck_get(f, magic, 8) || std::memcmp(magic, kCkMagic, 8) != 0) return bad(CSRST_E_IO, "not a checkpoint file");
  if (!ck_get(f, head, sizeof(head)) || head[0] != kCkVersion) return bad(CSRST_E_IO, "unknown checkpoint version");
  if (!ck_get(f, &cfg, sizeof(cfg)) || std::memcmp(&cfg, &h->cfg, sizeof(cfg)) != 0 || (head[1] != 0) != h->fp32)
    return bad(CSRST_E_ARG, "the checkpoint was written for another configuration");
  if (!ck_get(f, &st, 8) || !ck_get(f, &tm, 8)) return bad(CSRST_E_IO, "truncated file");
  CK(cudaStreamSynchronize(h->s));
  free_particles(h);  // window, bunch and the captured step go; the handle is rebuilt from the file
  std::vector<unsigned char> buf;
  CkPlan P = ck_plan(h);
  for (auto &pl : P.planes)
    if (!ck_get_dev(f, pl.first, pl.second, buf, h->s)) return bad(CSRST_E_IO, "truncated file (static fields)");
  int32_t win[3];
  if (!ck_get(f, win, sizeof(win)) || !ck_get(f, &h->acc_scale, 8)) return bad(CSRST_E_IO, "truncated file");
  if (win[0] <= 0 || win[1] <= 0 || win[2] != win[0] + 2) return bad(CSRST_E_IO, "corrupt window size");
  h->L0 = win[0]; h->L1 = win[1]; h->wpitch = win[2];
  const size_t wp = (size_t)h->wpitch * (h->L1 + 2);
  const size_t es = h->fp32 ? 4 : 8;
  if (h->fp32) {
    CK(cudaMalloc(&h->winf, 6 * wp * es));
    CK(cudaMalloc(&h->scratchf, 6 * wp * es));
  } else {
    CK(cudaMalloc(&h->win, 6 * wp * es));
    CK(cudaMalloc(&h->scratch, 6 * wp * es));
  }
  CK(cudaMalloc(&h->acc, 2 * (size_t)h->L0 * h->L1 * sizeof(unsigned long long)));
  P = ck_plan(h);
  for (auto &pl : P.window)
    if (!ck_get_dev(f, pl.first, pl.second, buf, h->s)) return bad(CSRST_E_IO, "truncated file (window)");
  long long n = 0;
  uint8_t flags[4];
  int32_t bb = 0;
  double mom[2];
  if (!ck_get(f, &n, 8) || n <= 0 || !ck_get(f, flags, 4) || !ck_get(f, &bb, 4) || !ck_get(f, mom, 16))
    return bad(CSRST_E_IO, "truncated file (bunch)");
  const size_t nb = (size_t)n * 8;
  h->n = n;
  if (h->fp32) {
    Bunch32 &b = h->b32;
    b.n = n;
    CK(palloc(&b.cell, (size_t)n * sizeof(int), h->s));
    for (float **p : {&b.ox, &b.oy, &b.dpx, &b.dpy, &b.q}) CK(palloc(p, (size_t)n * sizeof(float), h->s));
    CK(palloc(&h->d64, 4 * nb, h->s));
  } else {
    for (double **p : {&h->x, &h->y, &h->px, &h->py, &h->q, &h->ox, &h->oy}) CK(palloc(p, nb, h->s));
  }
  P = ck_plan(h);
  for (auto &pl : P.bunch)
    if (!ck_get_dev(f, pl.first, pl.second, buf, h->s)) return bad(CSRST_E_IO, "truncated file (bunch)");
  if (!ck_get(f, magic, 8) || std::memcmp(magic, kCkEnd, 8) != 0) return bad(CSRST_E_IO, "corrupt end of file");
  std::fclose(f);
  h->pending = flags[0] != 0;
  h->fresh = flags[1] != 0;
  h->acc_fresh[0] = flags[2] != 0;
  h->acc_fresh[1] = flags[3] != 0;
  h->bb = (BBoxState)bb;
  h->P0 = mom[0];
  h->P1 = mom[1];
  if (h->fp32) {
    set_ref32(h);
    CK(alloc_old32(h));
  }
  if (step) *step = st;
  if (time) *time = tm;
  return CSRST_OK;
}

}  // extern "C"
