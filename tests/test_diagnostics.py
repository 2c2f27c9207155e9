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
