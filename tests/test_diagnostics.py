"""The statistics writer's file format on the CPU (a stand-in simulation
supplies moments and field sums): the reference's SDDS1 header with its 16
columns, the row layout, and the field energy's time average
0.25 eps0 (E_now + E_last) + 0.5 mu0 H (CalcEnergy.cpp)."""
import math
import os

import numpy as np

from csrst_b200.diagnostics import COLUMNS, EPSILON_0, MU_0, DataSink, read_sdds


class _Sim:
    def __init__(self):
        self.k = 0

    def moments(self):
        return np.arange(18, dtype=float) + 100.0 * self.k

    def field_energy(self, with_window=True):
        self.k += 1 if with_window else 0
        return np.array([2.0 + self.k, 3.0 * self.k]) if with_window else np.array([1.5, 0.0])


def test_header_rows_and_energy(tmp_path):
    sim = _Sim()
    path = tmp_path / "Data" / "maxwadis.stat"
    with DataSink(sim, str(path), processors=4) as ds:
        r1 = ds.execute(1e-12)
        r2 = ds.execute(2e-12)
    text = path.read_text().splitlines()
    assert text[0] == "SDDS1"
    assert "Cores used 4" in text and sum(ln.startswith("&column") for ln in text) == 16
    names, rows = read_sdds(str(path))
    assert names == [c[0] for c in COLUMNS] and rows.shape == (2, 16)
    assert np.allclose(rows[0], r1, rtol=1e-14) and np.allclose(rows[1], r2, rtol=1e-14)
    # moments are read before the row's energy (calcBeamParameters, then CalcEnergy): m = arange + 100 k
    m1 = np.arange(18) + 0.0
    assert rows[0][1] == m1[14] and rows[0][12] == m1[16] and rows[0][13] == m1[17] and rows[0][14] == m1[15]
    e1 = 0.25 * EPSILON_0 * (3.0 + 1.5) + 0.5 * MU_0 * 3.0      # E_last from the static mesh at construction
    e2 = 0.25 * EPSILON_0 * (4.0 + 3.0) + 0.5 * MU_0 * 6.0      # then the previous call's E
    assert np.isclose(rows[0][15], e1 * 1e9, rtol=1e-13) and np.isclose(rows[1][15], e2 * 1e9, rtol=1e-13)
    assert all(len(ln) == 25 * 16 for ln in text[-2:])


def test_line_field_files(tmp_path):
    """FieldOnLine_NNNN.dat: numbered from 0, one tab-separated line of 7
    values per sample in the default stream format."""
    from csrst_b200.diagnostics import LineFieldSink

    class _S:
        def line_fields(self, with_current):
            return np.array([[-1.5e-4, 1.25, -2.0, 3.0, 0.0 if not with_current else 4.0, 1e-3, 2e-3]] * 3)

    ls = LineFieldSink(_S(), str(tmp_path / "Data"))
    p0, _ = ls.execute()
    p1, _ = ls.execute()
    assert p0.endswith("FieldOnLine_0000.dat") and p1.endswith("FieldOnLine_0001.dat")
    lines = open(p0).read().splitlines()
    assert len(lines) == 3 and lines[0] == "-0.00015\t1.25\t-2\t3\t0\t0.001\t0.002"


def test_vtk_piece_header_and_collection(tmp_path):
    """VtkSink steps of both series: the static piece's appended arrays read
    back equal to the overlaid fields (window over static, J from the window),
    the window piece to the window's interior at its origin; the parallel
    header names its piece, the collection lists each time step, and a new
    sink on the same directory continues the numbering."""
    from csrst_b200.diagnostics import VtkSink, read_vtr

    class _S:
        Nx, Ny = 12, 8

        def info(self):
            return {"hx": 0.5, "hy": 0.25, "ox": -1.0, "oy": 2.0}

        def get_static(self):
            g = np.arange(96, dtype=float).reshape(8, 12)
            return [g, g + 1000, g * 2, g * 3]

        def window(self):
            return [3, 2, 4, 3], np.array([0.5, 2.5]), None

        def window_field(self, k):
            w = np.full((5, 6), 10000.0 * (k + 1))
            w[2, 2] += 1
            return w

    d = str(tmp_path / "Data")
    vs = VtkSink(_S(), directory=d)
    piece = vs.execute(1e-12)
    vs.execute(2e-12)
    a = read_vtr(piece)
    assert np.allclose(a["X_COORDINATES"], np.arange(12) * 0.5 - 1.0)
    assert np.allclose(a["Y_COORDINATES"], np.arange(8) * 0.25 + 2.0)
    E = a["E-Field"].reshape(8, 12, 3)
    g = np.arange(96, dtype=float).reshape(8, 12)
    ex = g.copy()
    ex[2:5, 3:7] = 10000.0
    ex[3, 4] += 1
    assert np.array_equal(E[..., 0], ex.astype(np.float32)) and np.all(E[..., 2] == 0)
    H = a["H-Field"].reshape(8, 12)
    hz = g * 5
    hz[2:5, 3:7] = 30000.0 + 40000.0
    hz[3, 4] += 2
    assert np.array_equal(H, hz.astype(np.float32))
    J = a["J-Field"].reshape(8, 12, 3)
    assert J[3, 4, 0] == 50001.0 and J[0, 0, 0] == 0.0
    assert 'Source="c_0000_node00000.vtr"' in open(d + "/c_0000.pvtr").read()
    col = open(d + "/c_collection.pvd").read()
    assert col.count("<DataSet") == 2 and 'timestep="2e-12"' in col and 'file="c_0001.pvtr"' in col
    assert len(VtkSink(_S(), directory=d).times) == 2           # a resumed run continues the series
    w = read_vtr(VtkSink(_S(), base="mm", directory=d, source="window").execute(0.0))
    assert np.allclose(w["X_COORDINATES"], np.arange(4) * 0.5 + 0.5)
    Ew = w["E-Field"].reshape(3, 4, 3)
    assert Ew.shape == (3, 4, 3) and Ew[1, 1, 0] == 10001.0 and Ew[0, 0, 1] == 20000.0


class _ElongSim:
    """A Simulation stand-in for IntegrateElong / EnergyChange: a 12-column
    window (8 samples), wake samples with NaN where off the window, and a
    centroid that moves along x by 1 mm per moments() call."""

    def __init__(self):
        self.calls = 0
        self.k = 0

    def window(self):
        return [3, 2, 12, 5], np.array([0.5e-3, 2.5e-3]), None

    def info(self):
        return {"hx": 0.25e-3, "hy": 0.25e-3, "dt": 1e-12}

    def wake(self):
        e = np.array([((self.k * 7 + i * 13) % 17 - 8) * 1.5e4 for i in range(8)], dtype=float)
        e[0] = np.nan
        if self.k % 2:
            e[-1] = np.nan
        self.k += 1
        return e

    def moments(self):
        m = np.zeros(18)
        x = 1e-3 * self.calls
        self.calls += 1
        m[0] = x
        m[10], m[11], m[12], m[13] = x - 0.2e-3, 1e-3, x + 0.2e-3, 1.2e-3
        return m


def elong_samples(k):
    e = np.array([((k * 7 + i * 13) % 17 - 8) * 1.5e4 for i in range(8)], dtype=float)
    e[0] = np.nan
    if k % 2:
        e[-1] = np.nan
    return e


def test_integrate_elong_kahan_sum_and_file(tmp_path):
    """IntegrateElongCommand: long-double Kahan sums of the finite samples,
    written as (position from the centroid, -dt x sum) per sample."""
    from csrst_b200.diagnostics import IntegrateElong
    sim = _ElongSim()
    ie = IntegrateElong(sim, 5e-12)
    for _ in range(3):
        ie.execute()
    ref = np.nansum(np.stack([elong_samples(k) for k in range(3)]), axis=0)
    assert np.allclose(ie.sum.astype(float), ref, rtol=1e-15, atol=0)
    p = tmp_path / "ec.dat"
    ie.write(str(p))
    rows = np.loadtxt(p)
    assert rows.shape == (8, 2)
    assert np.allclose(rows[:, 0], 0.5e-3 + (2 + np.arange(8)) * 0.25e-3 - 0.0, rtol=1e-5)
    assert np.allclose(rows[:, 1], -5e-12 * ref, rtol=1e-5)
    ie.reset()
    assert not ie.sum.any()


def test_energy_change_files_follow_the_bend():
    """The loop's three energy-change files: before the bend until the front
    enters it, in the bend until the back has left it, after at the end."""
    import tempfile
    from types import SimpleNamespace
    from csrst_b200.diagnostics import EnergyChange, bend_frame, inside_bend
    # a bend of 4.7 mm radius (1 MeV, 1 T) starting at x = 3 mm, 30 degrees; bz < 0
    # puts the center below the pipe and deflects by +30 degrees
    cfg = SimpleNamespace(bz=-1.0, ekin_mev=1.0, phi_deg=30.0, length_before=3e-3, width=4e-3)
    fr = bend_frame(cfg)
    assert fr[0] == 3e-3 and fr[1] < 0 and abs(fr[2] - math.pi / 6) < 1e-15
    assert not inside_bend(fr, (2e-3, 1e-3)) and inside_bend(fr, (4e-3, 1e-3))
    with tempfile.TemporaryDirectory() as d:
        sim = _ElongSim()
        ec = EnergyChange(sim, cfg, 5, directory=d)
        written = []
        for _ in range(12):
            before = set(os.listdir(d))
            ec.execute()
            written += sorted(set(os.listdir(d)) - before)
        ec.finish()
        assert written == ["energyChangeBefore.dat", "energyChangeInBend.dat"]
        assert "energyChangeAfter.dat" in os.listdir(d)
