"""Run statistics and field dumps in the reference's file formats.

DataSink writes the SDDS1 ASCII statistics file of DataSinkCommand
(src/Commands/DataSink.cpp:22-149): the reference's header, then one row per
call with its 16 columns (time, mean kinetic energy, rms sizes and momenta,
normalised emittances, centroids, mean momenta, the dispersion terms Dy and
DDy, the energy spread and the total field energy), 15 significant digits in
25-character fields.  The beam quantities are the GPU moments
(csrst_diag_moments, PartBunch::calcBeamParameters); the field energy is
CalcEnergyCommand's (src/Commands/CalcEnergy.cpp:41-120), from the GPU
reduction csrst_diag_field_energy.  So that a run's statistics can be
compared with the reference's files line by line.
"""
import os

EPSILON_0 = 8.854187817e-12     # Physics::epsilon_0 (src/Physics.cpp:43)
MU_0 = 1.256637061e-06          # Physics::mu_0 (src/Physics.cpp:42)

# (name, units, description) of the 16 columns, DataSink.cpp:41-76
COLUMNS = [
    ("t", "s", "1 Time"), ("energy", "MeV", "2 Mean Energy"),
    ("rms_x", "m ", "3 RMS Beamsize in x  "), ("rms_y", "m ", "4 RMS Beamsize in y  "),
    ("rms_px", "1 ", "5 RMS Momenta in x  "), ("rms_py", "1 ", "6 RMS Momenta in y  "),
    ("emit_x", "m ", "7 Normalized Emittance x  "), ("emit_y", "m ", "8 Normalized Emittance y  "),
    ("mean_x", "m ", "9 Mean Beam Position in x  "), ("mean_y", "m ", "10 Mean Beam Position in y  "),
    ("mean_px", "1 ", "11 Mean Beam Momentum in x  "), ("mean_py", "1 ", "12 Mean Beam Momentum in y  "),
    ("Dy", "m ", "13 Dispersion in y  "), ("DDy", "1 ", "14 Derivative of dispersion in y  "),
    ("dE", "MeV ", "15 energy spread of the beam  "), ("Efld", "nJ ", "16 total field energy   "),
]


class FieldEnergy:
    """CalcEnergyCommand: the total field energy [J] at each call,
    0.25 eps0 (E_now + E_last) + 0.5 mu0 H, where E and H are the sums of
    csrst_diag_field_energy and E_last starts from the static mesh alone when
    the command is made (CalcEnergy.cpp:19-39)."""

    def __init__(self, sim):
        self.sim = sim
        self.e_last = float(sim.field_energy(with_window=False)[0])

    def __call__(self):
        ee, hh = (float(v) for v in self.sim.field_energy(with_window=True))
        total = 0.25 * EPSILON_0 * (ee + self.e_last) + 0.5 * MU_0 * hh
        self.e_last = ee
        return total


class DataSink:
    """DataSinkCommand for one Simulation: the header on construction, a row
    per execute(t) (the reference passes currentSimulatedTime + dt)."""

    def __init__(self, sim, path="Data/maxwadis.stat", processors=1, revision="csrst_b200"):
        self.sim = sim
        self.energy = FieldEnergy(sim)
        d = os.path.dirname(path)
        if d:
            os.makedirs(d, exist_ok=True)
        self.f = open(path, "w")
        w = self.f.write
        w("SDDS1\n")
        w('&description text="Statistics data ", contents="stat parameters" &end\n')
        w('&parameter name=processors, type=long, description="Number of Processors" &end\n')
        w('&parameter name=revision, type=string, description="svn revision of CSRST" &end\n')
        for name, units, desc in COLUMNS:
            w('&column name=%s, type=double, units=%s, description="%s" &end\n' % (name, units, desc))
        w("&data mode=ascii &end\n")
        w("Cores used %d\n" % processors)
        w("%s\n" % revision)
        self.f.flush()

    def row(self, t):
        """The 16 values of a row (also what execute writes)."""
        m = self.sim.moments()
        e = self.energy()
        return [t, m[14], m[4], m[5], m[6], m[7], m[8], m[9], m[0], m[1], m[2], m[3], m[16], m[17], m[15], e * 1e9]

    def execute(self, t):
        vals = self.row(t)
        self.f.write("".join("%25.15e" % v for v in vals) + "\n")
        self.f.flush()
        return vals

    def close(self):
        if not self.f.closed:
            self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class LineFieldSink:
    """SaveEMFieldsCommand (src/Commands/SaveEMFields.cpp:34-189): each
    execute() writes Data/FieldOnLine_NNNN.dat with one tab-separated line per
    sample (signed distance from the centroid, E along and across the mean
    momentum, Hz, J along it, x, y) in the default 6-digit C++ stream format,
    numbering the files from 0.  with_current=True takes J from the window
    (the reference does on plot steps; otherwise its column is 0)."""

    def __init__(self, sim, directory="Data", with_current=False):
        self.sim, self.dir, self.with_current, self.iteration = sim, directory, with_current, 0
        os.makedirs(directory, exist_ok=True)

    def execute(self):
        rows = self.sim.line_fields(self.with_current)
        path = os.path.join(self.dir, "FieldOnLine_%04d.dat" % self.iteration)
        with open(path, "w") as f:
            for r in rows:
                f.write("\t".join("%g" % v for v in r) + "\n")
        self.iteration += 1
        return path, rows


def read_sdds(path):
    """(column names, rows) of an ASCII statistics file written by DataSink."""
    import numpy as np
    names, rows, data = [], [], False
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while k < len(lines):
        ln = lines[k]
        if ln.startswith("&column"):
            names.append(ln.split("name=")[1].split(",")[0].strip())
        if ln.startswith("&data"):
            k += 3     # the two parameter values follow the data line
            break
        k += 1
    for ln in lines[k:]:
        if ln.strip():
            rows.append([float(v) for v in ln.split()])
    return names, np.array(rows)
