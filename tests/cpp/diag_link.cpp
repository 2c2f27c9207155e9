// Links the GPU-facing commands of include/csrst/diagnostics.hpp against the
// C ABI library (their entry points and signatures); run() is never called.
#include "csrst/diagnostics.hpp"

void run(csrst::Simulation &s) {
  csrst::DataSinkCommand ds(s, "maxwadis.stat");
  ds.execute(0.0);
  csrst::SaveEMFieldsCommand sf(s, ".", true);
  sf.execute();
  sf.execute(false);
  csrst::PlotBinaryVTKCommand plot(s), mini(s, "mm", ".", true);
  plot.execute(0.0);
  mini.execute(0.0);
  csrst::IntegrateElongCommand ielc(s, 1e-12);
  ielc.execute();
  if (csrst::inside_bend(csrst::bend_frame(s.config()), 0.0, 0.0)) ielc.write("energyChangeBefore.dat");
  ielc.reset();
}

int main(int argc, char **) { return argc > 99 ? (run(*(csrst::Simulation *)nullptr), 0) : 0; }
