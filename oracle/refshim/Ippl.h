// Minimal single-process stand-in for the parts of IPPL's interface that the
// reference's shape functions and utils.hh use, so that those reference
// sources compile and run here as a check of the oracle (test
// infrastructure; nothing in the product uses it).  Only the operations the
// deposit and the crossing split execute do real work (small vectors,
// particle attributes, index ranges, a mesh with origin and spacing); the
// rest of IPPL's interface is declared so the other functions of those files
// compile, and does nothing.
#ifndef CSRST_REFSHIM_IPPL_H
#define CSRST_REFSHIM_IPPL_H

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <sstream>
#include <stdexcept>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

// ---- small vectors -------------------------------------------------------
template <class T, unsigned D>
class Vektor {
 public:
  Vektor() { for (unsigned d = 0; d < D; ++d) v_[d] = T(0); }
  explicit Vektor(const T &a) { for (unsigned d = 0; d < D; ++d) v_[d] = a; }
  Vektor(const T &a, const T &b) { v_[0] = a; v_[1] = b; }
  Vektor(const T &a, const T &b, const T &c) { v_[0] = a; v_[1] = b; v_[2] = c; }
  T &operator()(unsigned d) { return v_[d]; }
  const T &operator()(unsigned d) const { return v_[d]; }
  T &operator[](unsigned d) { return v_[d]; }
  const T &operator[](unsigned d) const { return v_[d]; }
  Vektor &operator+=(const Vektor &o) { for (unsigned d = 0; d < D; ++d) v_[d] += o.v_[d]; return *this; }
  Vektor &operator-=(const Vektor &o) { for (unsigned d = 0; d < D; ++d) v_[d] -= o.v_[d]; return *this; }
  Vektor &operator*=(const T &s) { for (unsigned d = 0; d < D; ++d) v_[d] *= s; return *this; }
  Vektor &operator/=(const T &s) { for (unsigned d = 0; d < D; ++d) v_[d] /= s; return *this; }
  Vektor &operator=(const T &s) { for (unsigned d = 0; d < D; ++d) v_[d] = s; return *this; }

 private:
  T v_[D];
};

#define CSRST_SHIM_BINOP(op)                                                                   \
  template <class T, unsigned D>                                                               \
  Vektor<T, D> operator op(const Vektor<T, D> &a, const Vektor<T, D> &b) {                     \
    Vektor<T, D> r;                                                                            \
    for (unsigned d = 0; d < D; ++d) r(d) = a(d) op b(d);                                      \
    return r;                                                                                  \
  }                                                                                            \
  template <class T, unsigned D>                                                               \
  Vektor<T, D> operator op(const Vektor<T, D> &a, const T &s) {                                \
    Vektor<T, D> r;                                                                            \
    for (unsigned d = 0; d < D; ++d) r(d) = a(d) op s;                                         \
    return r;                                                                                  \
  }                                                                                            \
  template <class T, unsigned D>                                                               \
  Vektor<T, D> operator op(const T &s, const Vektor<T, D> &a) {                                \
    Vektor<T, D> r;                                                                            \
    for (unsigned d = 0; d < D; ++d) r(d) = s op a(d);                                         \
    return r;                                                                                  \
  }
CSRST_SHIM_BINOP(+)
CSRST_SHIM_BINOP(-)
CSRST_SHIM_BINOP(*)
CSRST_SHIM_BINOP(/)
#undef CSRST_SHIM_BINOP

template <class T, unsigned D>
Vektor<T, D> operator-(const Vektor<T, D> &a) {
  Vektor<T, D> r;
  for (unsigned d = 0; d < D; ++d) r(d) = -a(d);
  return r;
}

// IPPL's dot accumulates d = 0 .. D-1 from the first product.
template <class T, unsigned D>
T dot(const Vektor<T, D> &a, const Vektor<T, D> &b) {
  T s = a(0) * b(0);
  for (unsigned d = 1; d < D; ++d) s += a(d) * b(d);
  return s;
}

template <class T, unsigned D>
std::ostream &operator<<(std::ostream &o, const Vektor<T, D> &v) {
  o << "(";
  for (unsigned d = 0; d < D; ++d) o << (d ? "," : "") << v(d);
  return o << ")";
}

// ---- index ranges ----------------------------------------------------------
class Index {
 public:
  Index() : f_(0), l_(-1) {}
  explicit Index(int n) : f_(0), l_(n - 1) {}
  Index(int f, int l) : f_(f), l_(l) {}
  Index(int f, int l, int /*stride*/) : f_(f), l_(l) {}
  int first() const { return f_; }
  int stride() const { return 1; }
  bool operator==(const Index &o) const { return f_ == o.f_ && l_ == o.l_; }
  bool operator!=(const Index &o) const { return !(*this == o); }
  Index operator+(int k) const { return Index(f_ + k, l_ + k); }
  Index operator-(int k) const { return Index(f_ - k, l_ - k); }
  int last() const { return l_; }
  int length() const { return l_ - f_ + 1; }
  int min() const { return f_; }
  int max() const { return l_; }

 private:
  int f_, l_;
};

template <unsigned D>
class NDIndex {
 public:
  NDIndex() {}
  NDIndex(const Index &a, const Index &b) { i_[0] = a; i_[1] = b; }
  Index &operator[](unsigned d) { return i_[d]; }
  const Index &operator[](unsigned d) const { return i_[d]; }
  NDIndex intersect(const NDIndex &o) const {
    NDIndex r;
    for (unsigned d = 0; d < D; ++d)
      r[d] = Index(std::max(i_[d].first(), o[d].first()), std::min(i_[d].last(), o[d].last()));
    return r;
  }
  bool contains(const NDIndex &o) const {
    for (unsigned d = 0; d < D; ++d)
      if (o[d].first() < i_[d].first() || o[d].last() > i_[d].last()) return false;
    return true;
  }
  bool touches(const NDIndex &o) const {
    for (unsigned d = 0; d < D; ++d)
      if (o[d].last() < i_[d].first() || o[d].first() > i_[d].last()) return false;
    return true;
  }
  size_t size() const {
    size_t n = 1;
    for (unsigned d = 0; d < D; ++d) n *= (size_t)std::max(0, i_[d].length());
    return n;
  }

 private:
  Index i_[D];
};

template <unsigned D>
std::ostream &operator<<(std::ostream &o, const NDIndex<D> &n) {
  for (unsigned d = 0; d < D; ++d) o << "[" << n[d].first() << ":" << n[d].last() << "]";
  return o;
}

// ---- centerings, interpolation tags, mesh -----------------------------------
struct Vert {};
struct Edge {};
struct Cell {};
struct IntCIC {};
struct IntS1 {};
struct IntS2 {};
enum e_dim_tag { PARALLEL, SERIAL };

template <unsigned D, class T = double>
class UniformCartesian {
 public:
  UniformCartesian() : h_(T(1)), o_(T(0)) {}
  T get_meshSpacing(unsigned d) const { return h_(d); }
  Vektor<T, D> get_origin() const { return o_; }
  void set_meshSpacing(const T *h) { for (unsigned d = 0; d < D; ++d) h_(d) = h[d]; }
  void set_origin(const Vektor<T, D> &o) { o_ = o; }

 private:
  Vektor<T, D> h_, o_;
};

template <unsigned D>
class Vnode {
 public:
  int getNode() const { return 0; }
  const NDIndex<D> &getDomain() const { return dom_; }

 private:
  NDIndex<D> dom_;
};

template <class T>
class RefCountedP {
 public:
  RefCountedP() : p_(nullptr) {}
  T *operator->() const { return p_; }
  T &operator*() const { return *p_; }

 private:
  T *p_;
};

template <unsigned D>
class FieldLayout {
 public:
  typedef std::map<int, RefCountedP<Vnode<D> > > map_t;
  typedef typename map_t::const_iterator const_iterator_dv;
  FieldLayout() {}
  explicit FieldLayout(const NDIndex<D> &dom) : dom_(dom) {}
  const NDIndex<D> &getLocalNDIndex() const { return dom_; }
  const NDIndex<D> &getDomain() const { return dom_; }
  const_iterator_dv begin_rdv() const { return none_.begin(); }
  const_iterator_dv end_rdv() const { return none_.end(); }

 private:
  NDIndex<D> dom_;
  map_t none_;
};

template <unsigned D, class M, class C>
class CenteredFieldLayout : public FieldLayout<D> {
 public:
  using FieldLayout<D>::FieldLayout;
};

template <unsigned D>
class GuardCellSizes {
 public:
  GuardCellSizes() {}
  explicit GuardCellSizes(unsigned) {}
};

// A field on one process: its mesh, its layout and, once init() has sized it,
// its elements (i, j) for i in [-1, nx], j in [-1, ny] (one guard cell),
// addressed by single-element NDIndexes as IPPL's localElement does.
template <class T, unsigned D, class M, class C>
class Field {
 public:
  Field() {}
  void init(int nx, int ny) {
    nx_ = nx; ny_ = ny;
    data_.assign((size_t)(nx + 2) * (ny + 2), T());
    layout_ = FieldLayout<D>(NDIndex<D>(Index(0, nx - 1), Index(0, ny - 1)));
  }
  M &get_mesh() { return mesh_; }
  const M &get_mesh() const { return mesh_; }
  FieldLayout<D> &getLayout() { return layout_; }
  const FieldLayout<D> &getLayout() const { return layout_; }
  T &at(int i, int j) {
    if (i < -1 || j < -1 || i > nx_ || j > ny_) return dummy_;
    return data_[(size_t)(j + 1) * (nx_ + 2) + (i + 1)];
  }
  T &localElement(const NDIndex<D> &e) { return at(e[0].first(), e[1].first()); }
  const T &localElement(const NDIndex<D> &e) const {
    return const_cast<Field *>(this)->at(e[0].first(), e[1].first());
  }
  void fillGuardCells() {}
  template <class U>
  Field &operator=(const U &) { return *this; }
  // IPPL's indexed expressions (F[I][J](c) -= ...), accepted and ignored
  struct Expr {
    Expr operator[](const Index &) const { return *this; }
    Expr operator()(unsigned) const { return *this; }
    template <class U> Expr operator-=(const U &) const { return *this; }
    template <class U> Expr operator+=(const U &) const { return *this; }
    template <class U> Expr operator=(const U &) const { return *this; }
    template <class U> Expr operator-(const U &) const { return *this; }
    template <class U> Expr operator+(const U &) const { return *this; }
    template <class U> Expr operator*(const U &) const { return *this; }
  };
  Expr operator[](const Index &) const { return Expr(); }

 private:
  M mesh_;
  FieldLayout<D> layout_;
  int nx_ = 0, ny_ = 0;
  std::vector<T> data_;
  T dummy_{};
};

// ---- particles --------------------------------------------------------------
template <class T>
class ParticleAttrib {
 public:
  ParticleAttrib() {}
  T &operator[](size_t i) { return v_[i]; }
  const T &operator[](size_t i) const { return v_[i]; }
  size_t size() const { return v_.size(); }
  void create(size_t n) { v_.resize(v_.size() + n); }
  std::vector<T> &data() { return v_; }

 private:
  std::vector<T> v_;
};

template <class T, unsigned D>
class ParticleSpatialLayout {
 public:
  typedef Vektor<T, D> SingleParticlePos_t;
};
template <class T, unsigned D>
class ParticleUniformLayout {
 public:
  typedef Vektor<T, D> SingleParticlePos_t;
};

// ---- run-time services ------------------------------------------------------
struct Ippl {
  static int getNodes() { return 1; }
  static int myNode() { return 0; }
};

struct IpplTimings {
  typedef unsigned TimerRef;
  static TimerRef getTimer(const char *) { return 0; }
  static void startTimer(TimerRef) {}
  static void stopTimer(TimerRef) {}
};

class Inform {
 public:
  explicit Inform(const char * = nullptr, int = 0) {}
  template <class T>
  Inform &operator<<(const T &) { return *this; }
  Inform &operator<<(std::ostream &(*)(std::ostream &)) { return *this; }
};

// IPPL's debug assertion (the reference builds with -DIPPL_DEBUG): a failed
// one throws, so that the CPU check reports it instead of aborting.
struct PAssertFailed : std::runtime_error {
  explicit PAssertFailed(const char *w) : std::runtime_error(w) {}
};
#ifndef PAssert
#define PAssert(c) do { if (!(c)) throw PAssertFailed(#c); } while (0)
#endif
#ifndef PAssert_EQ
#define PAssert_EQ(a, b) assert((a) == (b))
#endif
#ifndef PAssert_LT
#define PAssert_LT(a, b) assert((a) < (b))
#endif
#ifndef PAssert_LE
#define PAssert_LE(a, b) assert((a) <= (b))
#endif
#ifndef PAssert_GE
#define PAssert_GE(a, b) assert((a) >= (b))
#endif
#ifndef PAssert_GT
#define PAssert_GT(a, b) assert((a) > (b))
#endif
#define ERRORMSG(x) std::cerr

#endif  // CSRST_REFSHIM_IPPL_H
