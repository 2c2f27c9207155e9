"""The reference loop's output schedule (src/main.cpp:358-522) on the CPU,
with a stand-in simulation that records the calls it receives."""
import os
from types import SimpleNamespace

import numpy as np

from csrst_b200 import loop
from csrst_b200.diagnostics import read_sdds


class _Sim:
    Nx, Ny = 12, 8

    def __init__(self):
        self.events = []
        self.t = 0

    # the loop's calls
    def step(self, k):
        self.events.append(("graph", k))
        self.t += k

    def step_first(self):
        self.events.append(("first", self.t))

    def step_second(self):
        self.events.append(("second", self.t))

    def move(self):
        self.events.append(("move", self.t))
        self.t += 1

    # what the writers read
    def info(self):
        return {"dt": 1e-12, "hx": 0.5, "hy": 0.25, "ox": -1.0, "oy": 2.0}

    def window(self):
        return [3, 2, 8, 3], np.array([0.5, 2.5]), None

    def window_field(self, k):
        return np.full((5, 10), float(k + 1))

    def get_static(self):
        g = np.arange(96, dtype=float).reshape(8, 12)
        return [g, g, g, g]

    def moments(self):
        m = np.zeros(18)
        m[0] = m[10] = m[12] = -1.0  # far before the bend
        return m

    def field_energy(self, with_window=True):
        return np.array([1.0, 2.0])

    def line_fields(self, with_current=False):
        self.events.append(("line", self.t, with_current))
        return np.zeros((3, 7))

    def wake(self):
        return np.ones(4)


def test_output_schedule(tmp_path):
    sim = _Sim()
    cfg = SimpleNamespace(bz=-1.0, ekin_mev=1.0, phi_deg=30.0, length_before=3e-3, width=4e-3)
    d = str(tmp_path / "Data")
    t = loop.run(sim, cfg, 10, plot_modulus=4, stat_modulus=3, line_modulus=5, directory=d)
    assert abs(t - 10e-12) < 1e-24
    # iterations 0, 1 and 6 have no output and run as graph steps; the others
    # run the half steps, their output, then the window move
    ev = [e for e in sim.events if e[0] != "line"]
    expect = [("graph", 2)]
    for it in (2, 3, 4, 5):
        expect += [("first", it), ("second", it), ("move", it)]
    expect.append(("graph", 1))
    for it in (7, 8, 9):
        expect += [("first", it), ("second", it), ("move", it)]
    assert ev == expect
    # line files: before the loop and at iterations 4 and 9, never on a plot step here
    assert [e for e in sim.events if e[0] == "line"] == [("line", 0, False), ("line", 4, False), ("line", 9, False)]
    files = sorted(os.listdir(d))
    assert [f for f in files if f.startswith("FieldOnLine")] == ["FieldOnLine_0000.dat", "FieldOnLine_0001.dat",
                                                                  "FieldOnLine_0002.dat"]
    # plots at t = 0 and after iterations 3 and 7 (stamped t + dt), both series
    col = open(os.path.join(d, "c_collection.pvd")).read()
    assert col.count("<DataSet") == 3 and 'timestep="4e-12"' in col and 'timestep="8e-12"' in col
    assert open(os.path.join(d, "mm_collection.pvd")).read().count("<DataSet") == 3
    # statistics rows: the initial one stamped dt, then iterations 2, 5, 8
    _, rows = read_sdds(os.path.join(d, "maxwadis.stat"))
    assert np.allclose(rows[:, 0], [1e-12, 3e-12, 6e-12, 9e-12], rtol=1e-12)
    assert "energyChangeAfter.dat" in files and "energyChangeBefore.dat" not in files


def test_plot_and_line_on_the_same_iteration_take_the_current(tmp_path):
    sim = _Sim()
    cfg = SimpleNamespace(bz=-1.0, ekin_mev=1.0, phi_deg=30.0, length_before=3e-3, width=4e-3)
    loop.run(sim, cfg, 4, plot_modulus=2, line_modulus=2, directory=str(tmp_path / "D"), restart=True)
    assert [e for e in sim.events if e[0] == "line"] == [("line", 0, False), ("line", 1, True), ("line", 3, True)]
    # a restart writes no t = 0 plot
    assert open(str(tmp_path / "D" / "c_collection.pvd")).read().count("<DataSet") == 2
