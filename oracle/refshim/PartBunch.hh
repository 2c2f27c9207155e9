// One-process stand-in for the reference's PartBunch (src/PartBunch.hh) as
// the shape functions read it: positions R, start positions oldR and charges
// Q of n particles, the bounds of R and oldR, and the particle box in cells
// (PartBunch::getLocalPDomainInclOld, src/PartBunch.cpp:854-897, restated for
// one process).  The CPU check of the oracle fills it.  It is included
// before the reference's sources under the reference header's own include
// guard, so that their #include "PartBunch.hh" adds nothing.
#ifndef OPAL_PartBunch_HH
#define OPAL_PartBunch_HH

#include "defs.hh"
#include "ShapeFunction.hh"

class PartBunch {
 public:
  ParticleAttrib<Vector_t> R, oldR;
  ParticleAttrib<double> Q;

  size_t getLocalNum() const { return R.size(); }
  size_t getLocalNP() const { return R.size(); }
  const std::vector<size_t> &getNumLocalParticles() const {
    nums_.assign(1, R.size());
    return nums_;
  }
  void getBoundsInclOld(Vector_t &mn, Vector_t &mx, size_t from, size_t to) const {
    mn = R[from]; mx = R[from];
    for (size_t i = from; i < to; ++i)
      for (unsigned d = 0; d < DIM; ++d) {
        mn(d) = std::min(mn(d), std::min(R[i](d), oldR[i](d)));
        mx(d) = std::max(mx(d), std::max(R[i](d), oldR[i](d)));
      }
  }
  NDIndex<DIM> getLocalPDomainInclOld(const Mesh_t &mesh) const {
    if (getLocalNum() == 0) return NDIndex<DIM>(Index(0), Index(0));
    const Vector_t origin = mesh.get_origin();
    const Vector_t dx(mesh.get_meshSpacing(0), mesh.get_meshSpacing(1));
    Vector_t lRmin, lRmax;
    getBoundsInclOld(lRmin, lRmax, 0, getLocalNum());
    NDIndex<DIM> ret;
    for (unsigned d = 0; d < DIM; ++d) {
      lRmin(d) = (lRmin(d) - origin(d)) / dx(d);
      lRmax(d) = (lRmax(d) - origin(d)) / dx(d);
      ret[d] = Index(std::floor(lRmin(d)), std::floor(lRmax(d)));
    }
    return ret;
  }
  NDIndex<DIM> getLocalPDomain(const Mesh_t &mesh) const { return getLocalPDomainInclOld(mesh); }
  NDIndex<DIM> getGlobalPDomainInclOld(const Mesh_t &mesh) const { return getLocalPDomainInclOld(mesh); }
  NDIndex<DIM> getGlobalPDomain(const Mesh_t &mesh) const { return getLocalPDomainInclOld(mesh); }
  template <class... A>
  void setGlobalBounds(A &&...) const {}

 private:
  mutable std::vector<size_t> nums_;
};

#endif
