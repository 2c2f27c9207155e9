// C++ facade over the C ABI (include/csrst.h) that keeps the call shapes of
// the reference's PIC-loop classes:
//   TETMSolver::updateField_firstStep / updateField_secondStep  (src/TETMSolver.hh:50-70)
//   PartBunch::push_particles / drift_particles / calcBeamParameters /
//             getGlobalBounds                                   (src/PartBunch.hh:46-112)
//   ScatterGatherImpl<IntOp, double>::gather                    (src/ScatterGatherImpl.hh:27-64)
//   moveMesh                                                    (src/main.cpp:562-652)
//   PoissonSolver::computeField                                 (src/PoissonSolver.cpp:85-201)
// IPPL field and attribute types are replaced by plain host arrays; the
// fields and the bunch themselves live on the GPU inside a Simulation.
// Failures throw csrst::Error (the reference aborts through PAssert).
#pragma once

#include <array>
#include <stdexcept>
#include <string>
#include <vector>

#include "../csrst.h"

namespace csrst {

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
    n_ = x.size();
    check(csrst_load_particles(h_, x.data(), y.data(), px.data(), py.data(), q.data(), n_), h_);
  }
  size_t size() const { return n_; }
  void step(int n) { check(csrst_step(h_, n), h_); }
  void sync() { check(csrst_sync(h_), h_); }
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
};

// PartBunchState fields the diagnostics use (src/PartBunch.hh:290-323).
struct PartBunchState {
  std::array<double, 2> rmean, pmean, rrms, prms, epsNorm, rmin, rmax;
  double Ekin = 0, dE = 0;
};

class PartBunch {
 public:
  explicit PartBunch(Simulation &s) : s_(s) {}
  void push_particles(unsigned Jcomp) { check(csrst_push(s_.handle(), (int)Jcomp), s_.handle()); }
  void drift_particles(double dt) { check(csrst_drift(s_.handle(), dt), s_.handle()); }
  void calcBeamParameters(PartBunchState &st) const {
    double m[18];
    check(csrst_diag_moments(s_.handle(), m), s_.handle());
    st.rmean = {m[0], m[1]}; st.pmean = {m[2], m[3]}; st.rrms = {m[4], m[5]};
    st.prms = {m[6], m[7]}; st.epsNorm = {m[8], m[9]}; st.rmin = {m[10], m[11]};
    st.rmax = {m[12], m[13]}; st.Ekin = m[14]; st.dE = m[15];
  }
  // first x, last x, first y, last y (window cells)
  std::array<int, 4> getGlobalBounds() const {
    int w[4], gb[4];
    double o[2];
    check(csrst_get_window(s_.handle(), w, o, gb), s_.handle());
    return {gb[0], gb[1], gb[2], gb[3]};
  }
  void getParticles(std::vector<double> &x, std::vector<double> &y, std::vector<double> &px,
                    std::vector<double> &py) const {
    x.resize(s_.size()); y.resize(s_.size()); px.resize(s_.size()); py.resize(s_.size());
    check(csrst_get_particles(s_.handle(), x.data(), y.data(), px.data(), py.data()), s_.handle());
  }

 private:
  Simulation &s_;
};

class TETMSolver {
 public:
  explicit TETMSolver(Simulation &s) : s_(s) {
    double info[8];
    check(csrst_get_info(s.handle(), info), s.handle());
    dt_ = info[4];
  }
  double getDT() const { return dt_; }
  void updateField_firstStep() { check(csrst_step_first(s_.handle()), s_.handle()); }
  void updateField_secondStep() { check(csrst_step_second(s_.handle()), s_.handle()); }

 private:
  Simulation &s_;
  double dt_ = 0;
};

inline void moveMesh(Simulation &s) { check(csrst_move_window(s.handle()), s.handle()); }

// Initial fields of the loaded bunch (PoissonSolver::computeField,
// src/PoissonSolver.cpp:85-201, followed by resetOutsideDomain as in
// src/main.cpp:232-248).  tol is the first solve's relative residual; the
// other two use 1e-6 as the reference does (PoissonSolver.cpp:172).
class PoissonSolver {
 public:
  explicit PoissonSolver(Simulation &s) : s_(s) {}
  void computeField(double tol = 1e-12, int maxIterations = 500) {
    check(csrst_initial_fields(s_.handle(), tol, 1e-6, maxIterations, report_.data()), s_.handle());
  }
  // gamma, (iterations, relative residual) of each solve, multigrid levels
  const std::array<double, 8> &report() const { return report_; }

 private:
  Simulation &s_;
  std::array<double, 8> report_{};
};

// A dense field patch on the host (the reference's FieldPatch<double>,
// src/FieldPatch.hh:33-132): element (i, j) at data[j * nx + i].
struct FieldPatch {
  const double *data;
  int nx, ny;
  std::array<double, 2> origin, spacing;
};

template <class IntOp>
struct ScatterGatherImpl {
  // Edge component comp of fp at R[from, to) into fld (ScatterGatherImpl.hh:31-38).
  static void gather(const FieldPatch &fp, double *fld, const double *x, const double *y, size_t comp,
                     size_t from, size_t to) {
    if (to <= from) return;
    check(csrst_gather(IntOp::order, (int)(comp % 2), fp.data, fp.nx, fp.ny, fp.origin.data(),
                       fp.spacing.data(), x + from, y + from, to - from, fld + from));
  }
  // Cell-centred field (ScatterGatherImpl.hh:40-47).
  static void gather(const FieldPatch &fp, double *fld, const double *x, const double *y, size_t from,
                     size_t to) {
    if (to <= from) return;
    check(csrst_gather(IntOp::order, 2, fp.data, fp.nx, fp.ny, fp.origin.data(), fp.spacing.data(),
                       x + from, y + from, to - from, fld + from));
  }
};

}  // namespace csrst
