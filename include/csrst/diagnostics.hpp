// Run statistics and field dumps in the reference's file formats, for C++
// programs that drive the loop through include/csrst/csrst.hpp:
//   DataSinkCommand      SDDS1 statistics file   (src/Commands/DataSink.cpp:22-149)
//   CalcEnergyCommand    total field energy       (src/Commands/CalcEnergy.cpp:19-120)
//   SaveEMFieldsCommand  FieldOnLine_NNNN.dat     (src/Commands/SaveEMFields.cpp:34-189)
//   PlotBinaryVTKCommand XML RectilinearGrid      (src/Commands/PlotBinaryVTK.cpp:29-119,
//                        series + collection       src/Commands/BinaryVTKFile.cpp:25-78)
//   IntegrateElongCommand energyChange*.dat       (src/Commands/IntegrateElong.cpp:14-125)
// The GPU supplies the numbers (moments, field-energy sums, line samples,
// field read-back); the files are written here on the host, byte for byte as
// csrst_b200/diagnostics.py writes them.  The functions in `format` take
// plain host arrays and touch no GPU.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "csrst.hpp"

namespace csrst {

constexpr double kEpsilon0 = 8.854187817e-12;  // Physics::epsilon_0 (src/Physics.cpp:43)
constexpr double kMu0 = 1.256637061e-06;       // Physics::mu_0 (src/Physics.cpp:42)

namespace format {

struct Column {
  const char *name, *units, *desc;
};

// The 16 columns of the statistics file (DataSink.cpp:41-76).
inline const std::array<Column, 16> &stat_columns() {
  static const std::array<Column, 16> c = {{
      {"t", "s", "1 Time"}, {"energy", "MeV", "2 Mean Energy"},
      {"rms_x", "m ", "3 RMS Beamsize in x  "}, {"rms_y", "m ", "4 RMS Beamsize in y  "},
      {"rms_px", "1 ", "5 RMS Momenta in x  "}, {"rms_py", "1 ", "6 RMS Momenta in y  "},
      {"emit_x", "m ", "7 Normalized Emittance x  "}, {"emit_y", "m ", "8 Normalized Emittance y  "},
      {"mean_x", "m ", "9 Mean Beam Position in x  "}, {"mean_y", "m ", "10 Mean Beam Position in y  "},
      {"mean_px", "1 ", "11 Mean Beam Momentum in x  "}, {"mean_py", "1 ", "12 Mean Beam Momentum in y  "},
      {"Dy", "m ", "13 Dispersion in y  "}, {"DDy", "1 ", "14 Derivative of dispersion in y  "},
      {"dE", "MeV ", "15 energy spread of the beam  "}, {"Efld", "nJ ", "16 total field energy   "},
  }};
  return c;
}

inline void sdds_header(std::FILE *f, int processors, const std::string &revision) {
  std::fputs("SDDS1\n", f);
  std::fputs("&description text=\"Statistics data \", contents=\"stat parameters\" &end\n", f);
  std::fputs("&parameter name=processors, type=long, description=\"Number of Processors\" &end\n", f);
  std::fputs("&parameter name=revision, type=string, description=\"svn revision of CSRST\" &end\n", f);
  for (const Column &c : stat_columns())
    std::fprintf(f, "&column name=%s, type=double, units=%s, description=\"%s\" &end\n", c.name, c.units, c.desc);
  std::fputs("&data mode=ascii &end\n", f);
  std::fprintf(f, "Cores used %d\n", processors);
  std::fprintf(f, "%s\n", revision.c_str());
}

// One statistics row from the GPU moments (out[18] of csrst_diag_moments)
// and the field energy in J.
inline std::array<double, 16> stat_row(double t, const double *m, double efield) {
  return {t,    m[14], m[4], m[5], m[6],  m[7],  m[8],  m[9],
          m[0], m[1],  m[2], m[3], m[16], m[17], m[15], efield * 1e9};
}

inline void sdds_row(std::FILE *f, const std::array<double, 16> &v) {
  for (double x : v) std::fprintf(f, "%25.15e", x);
  std::fputc('\n', f);
}

// CalcEnergyCommand's time average: 0.25 eps0 (E_now + E_last) + 0.5 mu0 H,
// from the sums {sum E^2, sum Hz^2} x cell area; E_last starts from the
// static mesh alone when the command is made (CalcEnergy.cpp:19-39).
struct EnergyAverage {
  double e_last;
  double operator()(double ee, double hh) {
    const double total = 0.25 * kEpsilon0 * (ee + e_last) + 0.5 * kMu0 * hh;
    e_last = ee;
    return total;
  }
};

// FieldOnLine file: n samples of 7 values, tab-separated, "%g" (the default
// C++ stream format of SaveEMFields.cpp).
inline void field_on_line(const std::string &path, const double *rows, int n) {
  std::FILE *f = std::fopen(path.c_str(), "w");
  if (!f) throw Error(CSRST_E_IO, "cannot write " + path);
  for (int k = 0; k < n; ++k)
    for (int c = 0; c < 7; ++c) std::fprintf(f, c < 6 ? "%g\t" : "%g\n", rows[7 * k + c]);
  std::fclose(f);
}

// The fields a plot step writes, [ny][nx] with x fastest: Ex, Ey, Hz (= Hzx +
// Hzy), Jx, Jy.
struct PlotFields {
  int nx = 0, ny = 0;
  double ox = 0, oy = 0, hx = 0, hy = 0;  // coordinates i h + origin
  std::vector<double> ex, ey, hz, jx, jy;
};

// The static mesh [Ny][Nx] with the window interior [L1][L0] (window cell
// (0, 0) on static cell (P0, P1)) copied over the points it covers, as
// copyFields leaves it on a plot step (main.cpp:54-66, :417); the current
// only from the window and only with_current.  win: 6 interior planes Ex,
// Ey, Hzx, Hzy, Jx, Jy.
inline void overlay(PlotFields &p, const double *const stat[4], const double *const win[6], int P0, int P1, int L0,
                    int L1, bool with_current) {
  const int Nx = p.nx, Ny = p.ny;
  const size_t N = (size_t)Nx * Ny;
  p.ex.assign(stat[0], stat[0] + N);
  p.ey.assign(stat[1], stat[1] + N);
  p.hz.resize(N);
  for (size_t k = 0; k < N; ++k) p.hz[k] = stat[2][k] + stat[3][k];
  p.jx.assign(N, 0.0);
  p.jy.assign(N, 0.0);
  for (int j = P1 < 0 ? 0 : P1; j < P1 + L1 && j < Ny; ++j)
    for (int i = P0 < 0 ? 0 : P0; i < P0 + L0 && i < Nx; ++i) {
      const size_t s = (size_t)j * Nx + i, w = (size_t)(j - P1) * L0 + (i - P0);
      p.ex[s] = win[0][w];
      p.ey[s] = win[1][w];
      p.hz[s] = win[2][w] + win[3][w];
      if (with_current) { p.jx[s] = win[4][w]; p.jy[s] = win[5][w]; }
    }
}

// One plot step: <dir>/<base>_NNNN_node00000.vtr (appended raw little-endian
// Float32 arrays, each after its byte count as a 32-bit integer) and the
// parallel header <dir>/<base>_NNNN.pvtr.  Returns the piece's path.
inline std::string vtk_step(const std::string &dir, const std::string &base, int index, const PlotFields &p) {
  char stem_c[64];
  std::snprintf(stem_c, sizeof stem_c, "%s_%04d", base.c_str(), index);
  const std::string stem = dir + "/" + stem_c, piece_name = std::string(stem_c) + "_node00000.vtr";
  const int nx = p.nx, ny = p.ny;
  struct Arr {
    bool point;
    const char *name;
    int comps;
    std::vector<float> v;
  };
  std::vector<Arr> arrs;
  std::vector<float> cx(nx), cy(ny), cz(1, 0.0f);
  for (int i = 0; i < nx; ++i) cx[i] = (float)((double)i * p.hx + p.ox);
  for (int j = 0; j < ny; ++j) cy[j] = (float)((double)j * p.hy + p.oy);
  arrs.push_back({false, "X_COORDINATES", 1, cx});
  arrs.push_back({false, "Y_COORDINATES", 1, cy});
  arrs.push_back({false, "Z_COORDINATES", 1, cz});
  const size_t N = (size_t)nx * ny;
  std::vector<float> e(3 * N), jv(3 * N), h(N);
  for (size_t k = 0; k < N; ++k) {
    e[3 * k] = (float)p.ex[k]; e[3 * k + 1] = (float)p.ey[k]; e[3 * k + 2] = 0.0f;
    jv[3 * k] = (float)p.jx[k]; jv[3 * k + 1] = (float)p.jy[k]; jv[3 * k + 2] = 0.0f;
    h[k] = (float)p.hz[k];
  }
  arrs.push_back({true, "E-Field", 3, e});
  arrs.push_back({true, "J-Field", 3, jv});
  arrs.push_back({true, "H-Field", 1, h});
  std::vector<size_t> off(arrs.size());
  size_t o = 0;
  for (size_t k = 0; k < arrs.size(); ++k) { off[k] = o; o += 4 + 4 * arrs[k].v.size(); }
  char ext[64];
  std::snprintf(ext, sizeof ext, "\"0 %d 0 %d 1 1\"", nx - 1, ny - 1);
  std::ostringstream hd;
  hd << "<?xml version=\"1.0\"?>\n<VTKFile type=\"RectilinearGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
     << "  <RectilinearGrid WholeExtent=" << ext << ">\n    <Piece Extent=" << ext << ">\n"
     << "      <PointData Scalars=\"H-Field\" Vectors=\"E-Field, J-Field\">\n";
  for (size_t k = 0; k < arrs.size(); ++k)
    if (arrs[k].point)
      hd << "        <DataArray type=\"Float32\" Name=\"" << arrs[k].name << "\" NumberOfComponents=\""
         << arrs[k].comps << "\" format=\"appended\" offset=\"" << off[k] << "\"/>\n";
  hd << "      </PointData>\n      <Coordinates>\n";
  for (size_t k = 0; k < arrs.size(); ++k)
    if (!arrs[k].point)
      hd << "        <DataArray type=\"Float32\" name=\"" << arrs[k].name << "\" NumberOfComponents=\""
         << arrs[k].comps << "\" format=\"appended\" offset=\"" << off[k] << "\"/>\n";
  hd << "      </Coordinates>\n    </Piece>\n  </RectilinearGrid>\n  <AppendedData encoding=\"raw\">\n    _";
  const std::string piece = stem + "_node00000.vtr";
  {
    std::ofstream f(piece, std::ios::binary);
    if (!f) throw Error(CSRST_E_IO, "cannot write " + piece);
    const std::string s = hd.str();
    f.write(s.data(), (std::streamsize)s.size());
    for (const Arr &a : arrs) {  // little-endian hosts (x86-64, aarch64) write their own byte order
      const uint32_t nb = (uint32_t)(4 * a.v.size());
      f.write(reinterpret_cast<const char *>(&nb), 4);
      f.write(reinterpret_cast<const char *>(a.v.data()), (std::streamsize)nb);
    }
    f << "\n  </AppendedData>\n</VTKFile>\n";
  }
  std::ofstream f(stem + ".pvtr");
  if (!f) throw Error(CSRST_E_IO, "cannot write " + stem + ".pvtr");
  f << "<?xml version=\"1.0\"?>\n<VTKFile type=\"PRectilinearGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
    << "  <PRectilinearGrid WholeExtent=" << ext << " GhostLevel=\"1\">\n"
    << "    <PPointData Scalars=\"H-Field\" Vectors=\"E-Field, J-Field\">\n";
  for (const Arr &a : arrs)
    if (a.point)
      f << "      <PDataArray type=\"Float32\" Name=\"" << a.name << "\" NumberOfComponents=\"" << a.comps << "\"/>\n";
  f << "    </PPointData>\n    <PCoordinates>\n";
  for (const char *n : {"X_COORDINATES", "Y_COORDINATES", "Z_COORDINATES"})
    f << "      <PDataArray type=\"Float32\" name=\"" << n << "\" NumberOfComponents=\"1\"/>\n";
  f << "    </PCoordinates>\n    <Piece Extent=" << ext << " Source=\"" << piece_name << "\"/>\n"
    << "  </PRectilinearGrid>\n</VTKFile>\n";
  return piece;
}

// <dir>/<base>_collection.pvd listing the steps written so far.
inline void vtk_collection(const std::string &dir, const std::string &base, const std::vector<double> &times) {
  const std::string path = dir + "/" + base + "_collection.pvd";
  std::FILE *f = std::fopen(path.c_str(), "w");
  if (!f) throw Error(CSRST_E_IO, "cannot write " + path);
  std::fputs("<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
             "  <Collection>\n", f);
  for (size_t i = 0; i < times.size(); ++i)
    std::fprintf(f, "    <DataSet timestep=\"%g\" group=\"\" part=\"0\" file=\"%s_%04d.pvtr\"/>\n", times[i],
                 base.c_str(), (int)i);
  std::fputs("  </Collection>\n</VTKFile>\n", f);
  std::fclose(f);
}

// The time steps of a collection already on disk (parseCollectionFile,
// PlotBinaryVTK.cpp:90-119), so that a resumed run continues its series.
inline std::vector<double> read_vtk_collection(const std::string &dir, const std::string &base) {
  std::vector<double> t;
  std::ifstream f(dir + "/" + base + "_collection.pvd");
  std::string line;
  const std::string key = "<DataSet timestep=\"";
  while (std::getline(f, line)) {
    const size_t a = line.find(key);
    if (a == std::string::npos) continue;
    const size_t b = line.find('"', a + key.size());
    if (b == std::string::npos) continue;
    t.push_back(std::stod(line.substr(a + key.size(), b - a - key.size())));
  }
  return t;
}

// Kahan sums in long double (Utils::KahanSum, src/utils.hh:513-521) of the
// finite samples e[k] into sum[k], corr[k].
inline void kahan_add(std::vector<long double> &sum, std::vector<long double> &corr, const double *e) {
  for (size_t k = 0; k < sum.size(); ++k) {
    if (e[k] != e[k]) continue;  // NaN: the sample's cell is off the window
    const long double y = (long double)e[k] - corr[k];
    const long double t = sum[k] + y;
    corr[k] = (t - sum[k]) - y;
    sum[k] = t;
  }
}

// IntegrateElongCommand::write (IntegrateElong.cpp:91-125): per sample at
// window column 2 + k, "origin0 + column h0 - rmean0 <tab> -dt x sum" in the
// default stream format.
inline void energy_change_file(const std::string &path, double origin0, double h0, double rmean0, double dt,
                               const std::vector<long double> &sum) {
  std::FILE *f = std::fopen(path.c_str(), "w");
  if (!f) throw Error(CSRST_E_IO, "cannot write " + path);
  for (size_t k = 0; k < sum.size(); ++k) {
    const double pos = origin0 + (double)(2 + (long long)k) * h0 - rmean0;
    std::fprintf(f, "%g\t%g\n", pos, -dt * (double)sum[k]);
  }
  std::fclose(f);
}

}  // namespace format

// The bend's frame as the reference sets it up (Bend ctor and Bend::Init,
// src/Bend.cpp:60-124): center and deflection angle.
struct BendFrame {
  double c0, c1, phi;
};

inline BendFrame bend_frame(const csrst_config &c) {
  const double mass = 0.511e6, ekin = c.ekin_mev * 1e6;
  double R = 9999999.9, phi = 0.0;
  if (std::abs(c.bz) > 1e-8) {
    R = std::sqrt(ekin * ekin + 2. * ekin * mass) / (299792458.0 * std::abs(c.bz));
    phi = -c.bz / std::abs(c.bz) * std::abs(c.phi_deg) * 3.14159265358979323846 / 180.;
  }
  return {c.length_before, c.bz <= 0.0 ? 0.5 * c.width - R : 0.5 * c.width + R, phi};
}

// Bend::isInsideBend (src/Bend.hh:308-322).
inline bool inside_bend(const BendFrame &b, double r0, double r1) {
  const double d0 = r0 - b.c0, d1 = r1 - b.c1;
  const double rot0 = std::cos(b.phi) * d0 + (-std::sin(b.phi)) * d1;
  if (d0 < 0.0 || rot0 > 0.0) return false;
  return d0 > 0.0 && rot0 < 0.0;
}

// IntegrateElongCommand (src/Commands/IntegrateElong.cpp:14-125): E_s on the
// bunch axis at window columns 2 .. L0-3 (csrst_diag_wake) summed over the
// calls; dt_sample is the time between calls (statmodulus x dt, main.cpp:370).
class IntegrateElongCommand {
 public:
  IntegrateElongCommand(Simulation &s, double dt_sample) : s_(s), dt_(dt_sample) {
    int w[4], gb[4];
    double o[2];
    check(csrst_get_window(s.handle(), w, o, gb), s.handle());
    n_ = w[2] - 4;
    sum_.assign((size_t)n_, 0.0L);
    corr_.assign((size_t)n_, 0.0L);
  }
  void execute() {
    std::vector<double> e((size_t)n_);
    check(csrst_diag_wake(s_.handle(), e.data(), n_), s_.handle());
    format::kahan_add(sum_, corr_, e.data());
  }
  void write(const std::string &path) const {
    int w[4], gb[4];
    double o[2], m[18], info[8];
    check(csrst_get_window(s_.handle(), w, o, gb), s_.handle());
    check(csrst_diag_moments(s_.handle(), m), s_.handle());
    check(csrst_get_info(s_.handle(), info), s_.handle());
    format::energy_change_file(path, o[0], info[0], m[0], dt_, sum_);
  }
  void reset() {
    sum_.assign((size_t)n_, 0.0L);
    corr_.assign((size_t)n_, 0.0L);
  }

 private:
  Simulation &s_;
  double dt_;
  int n_ = 0;
  std::vector<long double> sum_, corr_;
};

// CalcEnergyCommand over a Simulation: the total field energy [J] per call.
class CalcEnergyCommand {
 public:
  explicit CalcEnergyCommand(Simulation &s) : s_(s) {
    double out[2];
    check(csrst_diag_field_energy(s.handle(), 0, out), s.handle());
    avg_.e_last = out[0];
  }
  double execute() {
    double out[2];
    check(csrst_diag_field_energy(s_.handle(), 1, out), s_.handle());
    return avg_(out[0], out[1]);
  }

 private:
  Simulation &s_;
  format::EnergyAverage avg_{0.0};
};

// DataSinkCommand: the header on construction, a row per execute(t) (the
// reference passes currentSimulatedTime + dt).  The directory must exist.
class DataSinkCommand {
 public:
  DataSinkCommand(Simulation &s, const std::string &path = "Data/maxwadis.stat", int processors = 1,
                  const std::string &revision = "csrst_b200")
      : s_(s), energy_(s), f_(std::fopen(path.c_str(), "w")) {
    if (!f_) throw Error(CSRST_E_IO, "cannot write " + path);
    format::sdds_header(f_, processors, revision);
    std::fflush(f_);
  }
  ~DataSinkCommand() {
    if (f_) std::fclose(f_);
  }
  DataSinkCommand(const DataSinkCommand &) = delete;
  DataSinkCommand &operator=(const DataSinkCommand &) = delete;
  std::array<double, 16> execute(double t) {
    double m[18];
    check(csrst_diag_moments(s_.handle(), m), s_.handle());
    const std::array<double, 16> v = format::stat_row(t, m, energy_.execute());
    format::sdds_row(f_, v);
    std::fflush(f_);
    return v;
  }

 private:
  Simulation &s_;
  CalcEnergyCommand energy_;
  std::FILE *f_;
};

// SaveEMFieldsCommand: each execute() writes <dir>/FieldOnLine_NNNN.dat from
// 0 on; with_current takes J from the window (the reference copies the
// current only on plot steps, so its column is otherwise 0).
class SaveEMFieldsCommand {
 public:
  explicit SaveEMFieldsCommand(Simulation &s, const std::string &dir = "Data", bool with_current = false)
      : s_(s), dir_(dir), with_current_(with_current) {}
  std::string execute() { return execute(with_current_); }
  // with_current for this file only (the reference's plot steps copy the current)
  std::string execute(bool with_current) {
    int n = 0;
    check(csrst_diag_line_fields(s_.handle(), with_current ? 1 : 0, nullptr, 0, &n), s_.handle());
    std::vector<double> rows((size_t)7 * n);
    check(csrst_diag_line_fields(s_.handle(), with_current ? 1 : 0, rows.data(), n, &n), s_.handle());
    char name[32];
    std::snprintf(name, sizeof name, "/FieldOnLine_%04d.dat", iteration_++);
    const std::string path = dir_ + name;
    format::field_on_line(path, rows.data(), n);
    return path;
  }

 private:
  Simulation &s_;
  std::string dir_;
  bool with_current_;
  int iteration_ = 0;
};

// PlotBinaryVTKCommand: base "c" plots the static mesh with the window
// copied over it, base "mm" (window = true) the window alone at its own
// origin (main.cpp:358-365).  execute(t) writes one step and rewrites the
// collection; an existing collection is continued.  The directory must exist.
class PlotBinaryVTKCommand {
 public:
  PlotBinaryVTKCommand(Simulation &s, const std::string &base = "c", const std::string &dir = "Data",
                       bool window = false, bool with_current = true)
      : s_(s), base_(base), dir_(dir), window_(window), with_current_(with_current),
        times_(format::read_vtk_collection(dir, base)) {}
  std::string execute(double t) {
    csrst_handle *h = s_.handle();
    double info[8];
    check(csrst_get_info(h, info), h);
    int w[4], gb[4];
    double org[2];
    check(csrst_get_window(h, w, org, gb), h);
    const int L0 = w[2], L1 = w[3], wp = L0 + 2;
    std::vector<double> wfull((size_t)(L0 + 2) * (L1 + 2)), wplanes[6];
    for (int k = 0; k < 6; ++k) {
      check(csrst_get_window_field(h, k, wfull.data()), h);
      wplanes[k].resize((size_t)L0 * L1);
      for (int j = 0; j < L1; ++j)
        for (int i = 0; i < L0; ++i) wplanes[k][(size_t)j * L0 + i] = wfull[(size_t)(j + 1) * wp + (i + 1)];
    }
    const double *win[6] = {wplanes[0].data(), wplanes[1].data(), wplanes[2].data(),
                            wplanes[3].data(), wplanes[4].data(), wplanes[5].data()};
    format::PlotFields p;
    p.hx = info[0]; p.hy = info[1];
    if (window_) {
      p.nx = L0; p.ny = L1; p.ox = org[0]; p.oy = org[1];
      const size_t N = (size_t)L0 * L1;
      p.ex.assign(win[0], win[0] + N);
      p.ey.assign(win[1], win[1] + N);
      p.hz.resize(N);
      for (size_t k = 0; k < N; ++k) p.hz[k] = win[2][k] + win[3][k];
      p.jx.assign(win[4], win[4] + N);
      p.jy.assign(win[5], win[5] + N);
    } else {
      const csrst_config &c = s_.config();
      p.nx = c.Nx; p.ny = c.Ny; p.ox = info[2]; p.oy = info[3];
      const size_t N = (size_t)c.Nx * c.Ny;
      std::vector<double> st[4];
      for (auto &v : st) v.resize(N);
      check(csrst_get_static_fields(h, st[0].data(), st[1].data(), st[2].data(), st[3].data()), h);
      const double *stat[4] = {st[0].data(), st[1].data(), st[2].data(), st[3].data()};
      format::overlay(p, stat, win, w[0], w[1], L0, L1, with_current_);
    }
    const std::string piece = format::vtk_step(dir_, base_, (int)times_.size(), p);
    times_.push_back(t);
    closeFile();
    return piece;
  }
  void closeFile() { format::vtk_collection(dir_, base_, times_); }

 private:
  Simulation &s_;
  std::string base_, dir_;
  bool window_, with_current_;
  std::vector<double> times_;
};

}  // namespace csrst
