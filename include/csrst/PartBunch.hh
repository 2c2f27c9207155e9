// PartBunch of the reference (src/PartBunch.hh:37-180) over the GPU
// Simulation: the same method names, argument order and meaning, with the
// host views of core.hpp in place of IPPL fields and particle attributes.
// The bunch itself lives on the device; R, P and q are read back on request.
#pragma once

#include <algorithm>
#include <cmath>

#include "core.hpp"

namespace csrst {

// PartBunchState fields the diagnostics use (src/PartBunch.hh:290-323).
struct PartBunchState {
  std::array<double, 2> rmean, pmean, rrms, prms, epsNorm, rmin, rmax;
  double Ekin = 0, dE = 0;
};

class PartBunch {
 public:
  explicit PartBunch(Simulation &s) : s_(s) {}
  Simulation &simulation() const { return s_; }

  // oldR = R - dt c P / gamma (PartBunch.cpp:165-177): csrst_load_particles
  // sets this up on the device for the Simulation's dt; a different dt is an
  // error (the step length is part of the Simulation's configuration).
  void makeReady(const double &dt) { require_dt(dt, "makeReady"); }

  // PartBunch::push_particles(EFD, BFD, JFD, dt, Jcomp) (PartBunch.cpp:215-519):
  // gather from the window's E and split Hz, kick, drift, deposit component
  // Jcomp of the current.  The fields are the window's on the device; bound
  // views receive them after the push (EFD, BFD unchanged by it; JFD the
  // current this push deposited).
  void push_particles(EdgeFieldView &EFD, CellFieldView &BFD, EdgeFieldView &JFD, const double &dt,
                      const unsigned int &Jcomp) {
    require_dt(dt, "push_particles");
    if (Jcomp > 1) throw Error(CSRST_E_ARG, "push_particles: Jcomp must be 0 or 1");
    push_particles(Jcomp);
    NDIndex2 ddim, gb;
    Vector2 org;
    s_.window(ddim, gb, org);
    const FieldView *v[6] = {&EFD.x, &EFD.y, &BFD.x, &BFD.y, &JFD.x, &JFD.y};
    detail::mirror_window(s_, v, ddim, org);
  }
  void push_particles(unsigned Jcomp) { check(csrst_push(s_.handle(), (int)Jcomp), s_.handle()); }

  // PartBunch::drift_particles(dt) (PartBunch.cpp:179-187).
  void drift_particles(const double &dt) { check(csrst_drift(s_.handle(), dt), s_.handle()); }

  // PartBunch::calcBeamParameters (PartBunch.cpp:552-660).
  void calcBeamParameters(PartBunchState &st) const {
    double m[18];
    check(csrst_diag_moments(s_.handle(), m), s_.handle());
    st.rmean = {m[0], m[1]}; st.pmean = {m[2], m[3]}; st.rrms = {m[4], m[5]};
    st.prms = {m[6], m[7]}; st.epsNorm = {m[8], m[9]}; st.rmin = {m[10], m[11]};
    st.rmax = {m[12], m[13]}; st.Ekin = m[14]; st.dE = m[15];
  }
  void get_rmean(Vector2 &spos) const {
    PartBunchState st;
    calcBeamParameters(st);
    spos = st.rmean;
  }
  void get_pmean(Vector2 &pmean) const {
    PartBunchState st;
    calcBeamParameters(st);
    pmean = st.pmean;
  }
  double get_qtotal() const { return s_.qtotal(); }
  size_t getLocalNP() const { return s_.size(); }

  // Bounding box of particles [from, to) (PartBunch::getBounds).
  void getBounds(Vector2 &Rmin, Vector2 &Rmax, size_t from, size_t to) const {
    std::vector<double> x, y, px, py;
    read(x, y, px, py);
    to = std::min(to, x.size());
    Rmin = {INFINITY, INFINITY};
    Rmax = {-INFINITY, -INFINITY};
    for (size_t i = from; i < to; ++i) {
      Rmin = {std::min(Rmin[0], x[i]), std::min(Rmin[1], y[i])};
      Rmax = {std::max(Rmax[0], x[i]), std::max(Rmax[1], y[i])};
    }
  }

  // The bunch's cell bounds of the last push, in window cells (getGlobalBounds,
  // PartBunch.hh:104-106).
  NDIndex2 getGlobalBounds() const {
    NDIndex2 ddim, gb;
    Vector2 org;
    s_.window(ddim, gb, org);
    return gb;
  }

  // R and P into a bound view of size() particles (x, y and, if bound, px, py).
  void getParticles(ParticleView &R) const {
    if (R.n != s_.size()) throw Error(CSRST_E_ARG, "getParticles: view size differs from the bunch");
    std::vector<double> px, py;
    double *ppx = R.px, *ppy = R.py;
    if (!ppx) { px.resize(R.n); ppx = px.data(); }
    if (!ppy) { py.resize(R.n); ppy = py.data(); }
    check(csrst_get_particles(s_.handle(), R.x, R.y, ppx, ppy), s_.handle());
  }
  void getParticles(std::vector<double> &x, std::vector<double> &y, std::vector<double> &px,
                    std::vector<double> &py) const {
    read(x, y, px, py);
  }

 private:
  void read(std::vector<double> &x, std::vector<double> &y, std::vector<double> &px,
            std::vector<double> &py) const {
    x.resize(s_.size()); y.resize(s_.size()); px.resize(s_.size()); py.resize(s_.size());
    check(csrst_get_particles(s_.handle(), x.data(), y.data(), px.data(), py.data()), s_.handle());
  }
  void require_dt(double dt, const char *what) const {
    const double own = s_.info()[4];
    if (!(std::abs(dt - own) <= 1e-12 * own))
      throw Error(CSRST_E_ARG, std::string(what) + ": dt differs from the Simulation's time step");
  }
  Simulation &s_;
};

}  // namespace csrst
