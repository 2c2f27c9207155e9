"""The statistics writer's file format on the CPU (a stand-in simulation
supplies moments and field sums): the reference's SDDS1 header with its 16
columns, the row layout, and the field energy's time average
0.25 eps0 (E_now + E_last) + 0.5 mu0 H (CalcEnergy.cpp)."""
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
