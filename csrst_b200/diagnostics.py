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


def overlaid_fields(sim, with_current=True):
    """The static mesh's fields [Ny][Nx] with the window's values over the
    points it covers, as copyFields leaves them on a plot step (main.cpp:54-66,
    called at :417 with copyCurrent true): Ex, Ey, Hz = Hzx + Hzy, Jx, Jy (the
    current only from the window, and only with_current)."""
    import numpy as np
    ex, ey, hx, hy = sim.get_static()
    jx, jy = np.zeros_like(ex), np.zeros_like(ex)
    (P0, P1, L0, L1), _, _ = sim.window()
    win = [sim.window_field(k)[1:L1 + 1, 1:L0 + 1] for k in range(6)]
    j0, j1 = max(P1, 0), min(P1 + L1, sim.Ny)
    i0, i1 = max(P0, 0), min(P0 + L0, sim.Nx)
    sl = (slice(j0, j1), slice(i0, i1))
    ws = (slice(j0 - P1, j1 - P1), slice(i0 - P0, i1 - P0))
    for dst, k in ((ex, 0), (ey, 1), (hx, 2), (hy, 3)):
        dst[sl] = win[k][ws]
    if with_current:
        jx[sl], jy[sl] = win[4][ws], win[5][ws]
    return ex, ey, hx + hy, jx, jy


def window_fields(sim):
    """The window's own fields [L1][L0] (its interior) and its origin: Ex, Ey,
    Hzx + Hzy, Jx, Jy."""
    (_, _, L0, L1), origin, _ = sim.window()
    w = [sim.window_field(k)[1:L1 + 1, 1:L0 + 1] for k in range(6)]
    return (w[0], w[1], w[2] + w[3], w[4], w[5]), origin


class VtkSink:
    """PlotBinaryVTKCommand (src/Commands/PlotBinaryVTK.cpp:29-88, with the
    collection of PlotBinaryVTK.hh:58-80) and its writer BinaryVtkFile
    (src/Commands/BinaryVTKFile.cpp:25-78, BinaryVTKFile.hh:102-380).

    The run writes two series (main.cpp:358-359): base "c", the static mesh
    with the window copied over it, and base "mm", the window alone
    (source="window").  Each execute(t) writes, for the i-th call,
    <dir>/<base>_NNNN_node00000.vtr: an XML RectilinearGrid with raw appended
    little-endian Float32 data, every array preceded by its byte count as a
    32-bit unsigned integer: X/Y/Z_COORDINATES (i h + origin; z one 0), then
    E-Field and J-Field (3 components, z 0) and H-Field (Hzx + Hzy), x fastest;
    <dir>/<base>_NNNN.pvtr, the parallel header naming that piece; and
    <dir>/<base>_collection.pvd, the time series so far (the reference writes it
    at closeFile; writing it at every step keeps it whole if a run stops).  A
    collection already on disk is read first and numbering continues after it
    (PlotBinaryVTK.cpp:90-119), so a resumed run extends its series."""

    def __init__(self, sim, base="c", directory="Data", source="static", with_current=True):
        import re
        if source not in ("static", "window"):
            raise ValueError("source must be 'static' or 'window'")
        self.sim, self.base, self.dir, self.source = sim, base, directory, source
        self.with_current = with_current
        os.makedirs(directory, exist_ok=True)
        self.times = []
        col = self._collection()
        if os.path.exists(col):
            for line in open(col):
                m = re.search(r'<DataSet timestep="(.*?)"', line)
                if m:
                    self.times.append(float(m.group(1)))

    def _collection(self):
        return os.path.join(self.dir, self.base + "_collection.pvd")

    def _fields(self):
        info = self.sim.info()
        if self.source == "static":
            f = overlaid_fields(self.sim, self.with_current)
            origin = (info["ox"], info["oy"])
        else:
            f, origin = window_fields(self.sim)
        return f, origin, (info["hx"], info["hy"])

    def execute(self, t):
        import numpy as np
        (ex, ey, hz, jx, jy), origin, h = self._fields()
        ny, nx = ex.shape
        stem = os.path.join(self.dir, "%s_%04d" % (self.base, len(self.times)))
        blocks, arrays = [], []

        def add(kind, name, values, comps):
            arrays.append((kind, name, comps, sum(4 + b.nbytes for b in blocks)))
            blocks.append(np.ascontiguousarray(values, dtype="<f4"))

        add("coord", "X_COORDINATES", np.arange(nx) * h[0] + origin[0], 1)
        add("coord", "Y_COORDINATES", np.arange(ny) * h[1] + origin[1], 1)
        add("coord", "Z_COORDINATES", np.zeros(1), 1)
        zero = np.zeros_like(ex)
        add("point", "E-Field", np.stack([ex, ey, zero], axis=-1), 3)
        add("point", "J-Field", np.stack([jx, jy, zero], axis=-1), 3)
        add("point", "H-Field", hz, 1)
        ext = '"0 %d 0 %d 1 1"' % (nx - 1, ny - 1)
        head = ('<?xml version="1.0"?>\n<VTKFile type="RectilinearGrid" version="0.1" '
                'byte_order="LittleEndian">\n  <RectilinearGrid WholeExtent=%s>\n    <Piece Extent=%s>\n'
                '      <PointData Scalars="H-Field" Vectors="E-Field, J-Field">\n' % (ext, ext))
        for kind, name, comps, off in arrays:
            if kind == "point":
                head += ('        <DataArray type="Float32" Name="%s" NumberOfComponents="%d" '
                         'format="appended" offset="%d"/>\n' % (name, comps, off))
        head += '      </PointData>\n      <Coordinates>\n'
        for kind, name, comps, off in arrays:
            if kind == "coord":
                head += ('        <DataArray type="Float32" name="%s" NumberOfComponents="%d" '
                         'format="appended" offset="%d"/>\n' % (name, comps, off))
        head += ('      </Coordinates>\n    </Piece>\n  </RectilinearGrid>\n'
                 '  <AppendedData encoding="raw">\n    _')
        piece = stem + "_node00000.vtr"
        with open(piece, "wb") as f:
            f.write(head.encode())
            for b in blocks:
                f.write(np.uint32(b.nbytes).tobytes())
                f.write(b.tobytes())
            f.write(b"\n  </AppendedData>\n</VTKFile>\n")
        with open(stem + ".pvtr", "w") as f:
            f.write('<?xml version="1.0"?>\n<VTKFile type="PRectilinearGrid" version="0.1" '
                    'byte_order="LittleEndian">\n  <PRectilinearGrid WholeExtent=%s GhostLevel="1">\n' % ext)
            f.write('    <PPointData Scalars="H-Field" Vectors="E-Field, J-Field">\n')
            for kind, name, comps, _ in arrays:
                if kind == "point":
                    f.write('      <PDataArray type="Float32" Name="%s" NumberOfComponents="%d"/>\n'
                            % (name, comps))
            f.write('    </PPointData>\n    <PCoordinates>\n')
            for name in ("X_COORDINATES", "Y_COORDINATES", "Z_COORDINATES"):
                f.write('      <PDataArray type="Float32" name="%s" NumberOfComponents="1"/>\n' % name)
            f.write('    </PCoordinates>\n    <Piece Extent=%s Source="%s"/>\n'
                    % (ext, os.path.basename(piece)))
            f.write('  </PRectilinearGrid>\n</VTKFile>\n')
        self.times.append(t)
        self.close()
        return piece

    def close(self):
        with open(self._collection(), "w") as f:
            f.write('<?xml version="1.0"?>\n<VTKFile type="Collection" version="0.1" '
                    'byte_order="LittleEndian">\n  <Collection>\n')
            for i, t in enumerate(self.times):
                f.write('    <DataSet timestep="%g" group="" part="0" file="%s_%04d.pvtr"/>\n'
                        % (t, self.base, i))
            f.write('  </Collection>\n</VTKFile>\n')


def bend_frame(cfg):
    """(center0, center1, phi) of the bend as the reference sets it up
    (Bend ctor and Bend::Init, Bend.cpp:60-124): cfg has bz [T], ekin_mev,
    phi_deg, length_before and width [m]."""
    import math
    mass, ekin = 0.511e6, cfg.ekin_mev * 1e6
    if abs(cfg.bz) > 1e-8:
        R = math.sqrt(ekin * ekin + 2. * ekin * mass) / (299792458.0 * abs(cfg.bz))
        phi = -cfg.bz / abs(cfg.bz) * abs(cfg.phi_deg) * math.pi / 180.
    else:
        R, phi = 9999999.9, 0.0
    c1 = 0.5 * cfg.width - R if cfg.bz <= 0.0 else 0.5 * cfg.width + R
    return cfg.length_before, c1, phi


def inside_bend(frame, r):
    """Bend::isInsideBend (Bend.hh:308-322): r between the entrance plane and
    the exit plane of the bend, measured from its center."""
    import math
    c0, c1, phi = frame
    d0, d1 = r[0] - c0, r[1] - c1
    rot0 = math.cos(phi) * d0 + (-math.sin(phi)) * d1
    if d0 < 0.0 or rot0 > 0.0:
        return False
    return d0 > 0.0 and rot0 < 0.0


class IntegrateElong:
    """IntegrateElongCommand (src/Commands/IntegrateElong.cpp:14-125): at each
    execute() the longitudinal field E_s sampled on the bunch axis at window
    columns 2 .. L0-3 (csrst_diag_wake: along the mean momentum through the
    centroid; NaN where the sample's cell is off the window) is added to a
    per-sample Kahan sum in long double (Utils::KahanSum, utils.hh:513-521);
    write(fname) puts one line per sample, "position from the centroid <tab>
    -dt_sample x sum" in the default 6-digit stream format, the position being
    window origin + column h - current centroid x.  dt_sample is the time
    between calls (the reference passes statmodulus x dt, main.cpp:370)."""

    def __init__(self, sim, dt_sample):
        import numpy as np
        self.sim, self.dt = sim, float(dt_sample)
        self.n = sim.window()[0][2] - 4
        self.sum = np.zeros(self.n, dtype=np.longdouble)
        self.corr = np.zeros(self.n, dtype=np.longdouble)

    def reset(self):
        self.sum[:] = 0
        self.corr[:] = 0

    def execute(self):
        import numpy as np
        e = np.asarray(self.sim.wake(), dtype=np.float64)
        ok = ~np.isnan(e)
        y = e[ok].astype(np.longdouble) - self.corr[ok]
        t = self.sum[ok] + y
        self.corr[ok] = (t - self.sum[ok]) - y
        self.sum[ok] = t

    def write(self, fname):
        import numpy as np
        d = os.path.dirname(fname)
        if d:
            os.makedirs(d, exist_ok=True)
        _, origin, _ = self.sim.window()
        r0 = float(self.sim.moments()[0])
        h0 = float(self.sim.info()["hx"])
        line = self.sum.astype(np.float64)
        with open(fname, "w") as f:
            for i in range(self.n):
                pos = float(origin[0]) + (2 + i) * h0 - r0
                f.write("%g\t%g\n" % (pos, -self.dt * float(line[i])))


class EnergyChange:
    """The reference loop's energy-change files (main.cpp:370, :445-465,
    :517): an IntegrateElong over the statistics steps, written to
    energyChangeBefore.dat when the bunch's front (rmax) first enters the
    bend, to energyChangeInBend.dat when front and back (rmin) have both
    left it, and to energyChangeAfter.dat at finish(); the sum restarts after
    each file.  Call execute() on every statistics step, after the
    statistics row (the reference reads the same step's moments)."""

    def __init__(self, sim, cfg, stat_modulus, directory="Data"):
        self.sim, self.dir = sim, directory
        self.ielc = IntegrateElong(sim, stat_modulus * sim.info()["dt"])
        self.frame = bend_frame(cfg)
        self.before, self.in_bend = True, False

    def execute(self):
        m = self.sim.moments()
        rmin, rmax = m[10:12], m[12:14]
        if self.before and inside_bend(self.frame, rmax):
            self.ielc.write(os.path.join(self.dir, "energyChangeBefore.dat"))
            self.ielc.reset()
            self.before, self.in_bend = False, True
        if self.in_bend and not inside_bend(self.frame, rmax) and not inside_bend(self.frame, rmin):
            self.ielc.write(os.path.join(self.dir, "energyChangeInBend.dat"))
            self.ielc.reset()
            self.in_bend = False
        self.ielc.execute()

    def finish(self):
        self.ielc.write(os.path.join(self.dir, "energyChangeAfter.dat"))


def read_vtr(path):
    """{name: float32 array} of a piece written by VtkSink (appended raw data)."""
    import re
    import numpy as np
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b"<AppendedData encoding=\"raw\">")
    data = rest[rest.index(b"_") + 1:]
    out = {}
    for m in re.finditer(rb'<DataArray type="Float32" [Nn]ame="([^"]+)" NumberOfComponents="(\d)" '
                         rb'format="appended" offset="(\d+)"/>', head):
        off = int(m.group(3))
        n = int(np.frombuffer(data[off:off + 4], dtype="<u4")[0])
        out[m.group(1).decode()] = np.frombuffer(data[off + 4:off + 4 + n], dtype="<f4")
    return out


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
