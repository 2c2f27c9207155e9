// Writes the Halton command-line bunch of include/csrst/distribution.hpp
// (x, y, px, py, q as consecutive doubles) to argv[1].
#include <cstdio>

#include "csrst/distribution.hpp"

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  csrst::DistributionParams p;
  p.n = 3000;
  p.mean_rx = 1.7e-3; p.mean_ry = 1.0e-3; p.sigma_x = 40e-6; p.ekin_mev = 510.489;
  p.sigma_p = 1.0; p.qtotal_nc = 1.0;
  p.origin[0] = -20e-6; p.origin[1] = -20e-6; p.spacing[0] = 20e-6; p.spacing[1] = 20e-6;
  const csrst::HostBunch b = csrst::halton_bunch(p);
  std::FILE *f = std::fopen(argv[1], "wb");
  for (const auto *v : {&b.x, &b.y, &b.px, &b.py, &b.q}) std::fwrite(v->data(), sizeof(double), v->size(), f);
  std::fclose(f);
  return 0;
}
