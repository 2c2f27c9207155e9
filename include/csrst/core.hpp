// Core of the C++ facade over the C ABI (include/csrst.h): errors, the
// shape-function tags, the host views that stand in for the reference's IPPL
// types, and the Simulation that owns one GPU handle.  The reference-shaped
// classes live in the headers named after the reference's (TETMSolver.hh,
// PartBunch.hh, ScatterGatherImpl.hh, PoissonSolver.hh); csrst.hpp includes
// them all.
#pragma once

#include <array>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../csrst.h"

namespace csrst {

// Failures throw csrst::Error (the reference aborts through PAssert).
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Throws on a failure (negative status); a warning (positive status, the
// call succeeded) is returned to the caller.
inline int check(int code, const csrst_handle *h = nullptr) {
  if (code >= CSRST_OK) return code;
  char buf[512];
  csrst_get_error(h, buf, sizeof(buf));
  throw Error(code, "csrst error " + std::to_string(code) + ": " + buf);
}

// IntOp tags (src/defs.hh:55-57)
struct IntCIC { static constexpr int order = 0; };
struct IntS1 { static constexpr int order = 1; };
struct IntS2 { static constexpr int order = 2; };

// Vector_t of the reference (Vektor<double, 2>).
using Vector2 = std::array<double, 2>;

// One component of a field on the host, in place of an IPPL
// Field<double, 2> over its NDIndex with a guard ring: element (i, j),
// i in [-guard, nx + guard), j in [-guard, ny + guard), at
// ptr[(j + guard) * pitch + (i + guard)].  origin and h describe the mesh of
// vertex (0, 0).  A view with ptr == nullptr is unbound: calls that take it
// skip it.
struct FieldView {
  double *ptr = nullptr;
  int nx = 0, ny = 0, pitch = 0, guard = 0;
  Vector2 origin{0.0, 0.0}, h{0.0, 0.0};
  bool bound() const { return ptr != nullptr; }
  double &operator()(int i, int j) const { return ptr[(size_t)(j + guard) * pitch + (i + guard)]; }
};

// VField_Edge_t (E or J: x and y components on the cell edges).
struct EdgeFieldView {
  FieldView x, y;
};

// VField_Cell_t (Hz, stored split as Hzx and Hzy: the TE/TM split scheme
// keeps the two parts of Hz apart, their sum is Hz).
struct CellFieldView {
  FieldView x, y;
};

// Positions R (and momenta P where a call needs them) of n particles, in
// place of ParticleAttrib<Vector_t>.
struct ParticleView {
  double *x = nullptr, *y = nullptr, *px = nullptr, *py = nullptr;
  size_t n = 0;
};

// A vector attribute of n particles (ParticleAttrib<Vector_t>), by component.
struct VectorAttribView {
  double *c[2] = {nullptr, nullptr};
  size_t n = 0;
};

// NDIndex<2> with unit stride: cells [i0, i1] x [j0, j1] (inclusive, as
// Index::first() .. Index::last()).
struct NDIndex2 {
  int i0 = 0, i1 = -1, j0 = 0, j1 = -1;
  int length(int d) const { return d == 0 ? i1 - i0 + 1 : j1 - j0 + 1; }
  bool operator==(const NDIndex2 &o) const { return i0 == o.i0 && i1 == o.i1 && j0 == o.j0 && j1 == o.j1; }
  bool operator!=(const NDIndex2 &o) const { return !(*this == o); }
};

// Static mesh, moving window and bunch on one GPU.
class Simulation {
 public:
  explicit Simulation(const csrst_config &cfg) : cfg_(cfg) { check(csrst_create(&cfg, &h_)); }
  ~Simulation() { csrst_destroy(h_); }
  Simulation(const Simulation &) = delete;
  Simulation &operator=(const Simulation &) = delete;

  csrst_handle *handle() const { return h_; }
  const csrst_config &config() const { return cfg_; }

  void setStaticFields(const double *ex, const double *ey, const double *hzx, const double *hzy) {
    check(csrst_set_static_fields(h_, ex, ey, hzx, hzy), h_);
  }
  void loadBunch(const std::vector<double> &x, const std::vector<double> &y, const std::vector<double> &px,
                 const std::vector<double> &py, const std::vector<double> &q) {
    check(csrst_load_particles(h_, x.data(), y.data(), px.data(), py.data(), q.data(), x.size()), h_);
    n_ = x.size();
    qtotal_ = 0.0;
    for (double v : q) qtotal_ += v;
  }
  size_t size() const { return n_; }
  double qtotal() const { return qtotal_; }
  void step(int n) { check(csrst_step(h_, n), h_); }
  void sync() { check(csrst_sync(h_), h_); }
  // info: hx, hy, origin x, origin y, dt, fixed-point scale, cut cells, window pitch
  std::array<double, 8> info() const {
    std::array<double, 8> v{};
    check(csrst_get_info(h_, v.data()), h_);
    return v;
  }
  // The window's domain on the static mesh (the reference's ddim) and the
  // bunch's cell bounds of the last push (getGlobalBounds).
  void window(NDIndex2 &ddim, NDIndex2 &bounds, Vector2 &origin) const {
    int w[4], gb[4];
    double o[2];
    check(csrst_get_window(h_, w, o, gb), h_);
    ddim = {w[0], w[0] + w[2] - 1, w[1], w[1] + w[3] - 1};
    bounds = {gb[0], gb[1], gb[2], gb[3]};
    origin = {o[0], o[1]};
  }
  // Restart dump (LoadH5Part, src/Commands/LoadH5Part.cpp:60-321): everything a step reads, so
  // that a Simulation of the same configuration restored from the file continues bit for bit.
  void checkpoint(const std::string &path, long long step, double time) {
    check(csrst_checkpoint_write(h_, path.c_str(), step, time), h_);
  }
  void restore(const std::string &path, long long &step, double &time) {
    check(csrst_checkpoint_read(h_, path.c_str(), &step, &time), h_);
    long long n = 0;
    check(csrst_get_num_particles(h_, &n), h_);
    n_ = (size_t)n;
  }

 private:
  csrst_config cfg_;
  csrst_handle *h_ = nullptr;
  size_t n_ = 0;
  double qtotal_ = 0.0;
};

namespace detail {

// Copies an nx x ny array (x fastest, no guards) into a bound view's interior.
inline void to_view(const FieldView &v, const double *src, int nx, int ny) {
  if (!v.bound()) return;
  if (v.nx != nx || v.ny != ny || v.pitch < nx + 2 * v.guard)
    throw Error(CSRST_E_ARG, "field view: " + std::to_string(v.nx) + " x " + std::to_string(v.ny) +
                                 " does not match the mesh's " + std::to_string(nx) + " x " + std::to_string(ny));
  for (int j = 0; j < ny; ++j) std::memcpy(&v(0, j), src + (size_t)j * nx, nx * sizeof(double));
}

// The static mesh's fields into bound views (E, split Hz; the static J is
// zero in the loop, as main.cpp:388 and :494 reset it).
inline void mirror_static(Simulation &s, EdgeFieldView &E, CellFieldView &H, EdgeFieldView &J) {
  const int nx = s.config().Nx, ny = s.config().Ny;
  const bool any = E.x.bound() || E.y.bound() || H.x.bound() || H.y.bound();
  const auto inf = s.info();
  for (FieldView *v : {&E.x, &E.y, &H.x, &H.y, &J.x, &J.y}) {
    v->origin = {inf[2], inf[3]};
    v->h = {inf[0], inf[1]};
  }
  if (any) {
    std::vector<double> f[4];
    double *p[4] = {nullptr, nullptr, nullptr, nullptr};
    const FieldView *dst[4] = {&E.x, &E.y, &H.x, &H.y};
    for (int k = 0; k < 4; ++k)
      if (dst[k]->bound()) { f[k].resize((size_t)nx * ny); p[k] = f[k].data(); }
    check(csrst_get_static_fields(s.handle(), p[0], p[1], p[2], p[3]), s.handle());
    for (int k = 0; k < 4; ++k) to_view(*dst[k], p[k], nx, ny);
  }
  for (const FieldView *v : {&J.x, &J.y}) {
    if (!v->bound()) continue;
    std::vector<double> zero((size_t)nx * ny, 0.0);
    to_view(*v, zero.data(), nx, ny);
  }
}

// The window's fields (guard ring included) into bound views of the window's
// size; which: 0 Ex, 1 Ey, 2 Hzx, 3 Hzy, 4 Jx, 5 Jy.
inline void mirror_window(Simulation &s, const FieldView *const v[6], const NDIndex2 &ddim, const Vector2 &org) {
  const int L0 = ddim.length(0), L1 = ddim.length(1);
  const auto inf = s.info();
  std::vector<double> buf;
  for (int k = 0; k < 6; ++k) {
    FieldView &w = *const_cast<FieldView *>(v[k]);
    w.origin = org;
    w.h = {inf[0], inf[1]};
    if (!w.bound()) continue;
    if (w.nx != L0 || w.ny != L1 || w.guard > 1 || w.pitch < L0 + 2 * w.guard)
      throw Error(CSRST_E_ARG, "window view: " + std::to_string(w.nx) + " x " + std::to_string(w.ny) +
                                   " does not match the window's " + std::to_string(L0) + " x " +
                                   std::to_string(L1) + " (guard 0 or 1)");
    buf.resize((size_t)(L0 + 2) * (L1 + 2));
    check(csrst_get_window_field(s.handle(), k, buf.data()), s.handle());
    for (int j = -w.guard; j < L1 + w.guard; ++j)
      for (int i = -w.guard; i < L0 + w.guard; ++i) w(i, j) = buf[(size_t)(j + 1) * (L0 + 2) + (i + 1)];
  }
}

}  // namespace detail
}  // namespace csrst
