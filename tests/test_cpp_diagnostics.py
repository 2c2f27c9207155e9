"""The C++ writers of include/csrst/diagnostics.hpp (statistics file, line
fields, VTK series) produce byte for byte the files of the Python writers in
csrst_b200/diagnostics.py on the same values.  Host code only: the values
stand in for what the GPU returns."""
import filecmp
import subprocess
from pathlib import Path

import numpy as np

from csrst_b200.diagnostics import DataSink, LineFieldSink, VtkSink

ROOT = Path(__file__).resolve().parents[1]


def val(k, salt):
    return ((k * 37 + salt * 11) % 101 - 50) * 1.25e-3


class _FakeSim:
    """What the writers read from a Simulation, with fixed values."""
    Nx, Ny = 12, 8

    def __init__(self):
        self.rows = 0
        self.energies = [np.array([3.5, 0.0]), np.array([4.25, 0.5]), np.array([5.0, 0.75])]
        self.e = 0

    def moments(self):
        m = np.array([val(k, self.rows) for k in range(18)])
        self.rows += 1
        return m

    def field_energy(self, with_window=True):
        v = self.energies[self.e]
        self.e += 1
        return v

    def line_fields(self, with_current=False):
        return np.array([val(k, 3) * (1e6 if k % 3 == 0 else 1.0) for k in range(35)]).reshape(5, 7)

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


class _ElongSim:
    """What IntegrateElong reads: a 12-column window, three wake sample sets,
    the centroid at x = 0.75 mm."""

    def __init__(self):
        self.k = 0

    def window(self):
        return [3, 2, 12, 5], np.array([0.5e-3, 2.5e-3]), None

    def info(self):
        return {"hx": 0.25e-3, "hy": 0.25e-3, "dt": 1e-12}

    def wake(self):
        e = np.array([((self.k * 7 + i * 13) % 17 - 8) * 1.5e4 for i in range(8)], dtype=float)
        e[0] = np.nan
        if self.k % 2:
            e[7] = np.nan
        self.k += 1
        return e

    def moments(self):
        m = np.zeros(18)
        m[0] = 0.75e-3
        return m


def test_cpp_writers_match_python(tmp_path):
    exe = tmp_path / "diag_main"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/diag_main.cpp"),
                    "-o", str(exe)], check=True)
    cdir, pdir = tmp_path / "cpp", tmp_path / "py"
    cdir.mkdir()
    r = subprocess.run([str(exe), str(cdir)], capture_output=True, text=True, check=True)
    assert r.stdout.split() == ["collection", "2", "2e-12", "1e-12"]
    sim = _FakeSim()
    with DataSink(sim, str(pdir / "stats.stat")) as ds:
        ds.execute(1e-12)
        ds.execute(2e-12)
    LineFieldSink(sim, str(pdir)).execute()
    vs = VtkSink(sim, directory=str(pdir))
    vs.execute(1e-12)
    vs.execute(2e-12)
    VtkSink(sim, base="mm", directory=str(pdir), source="window").execute(0.0)
    from csrst_b200.diagnostics import IntegrateElong
    ie = IntegrateElong(_ElongSim(), 5e-12)
    for _ in range(3):
        ie.execute()
    ie.write(str(pdir / "energyChange.dat"))
    names = ["stats.stat", "FieldOnLine_0000.dat", "c_0000_node00000.vtr", "c_0001_node00000.vtr", "c_0000.pvtr",
             "c_0001.pvtr", "c_collection.pvd", "mm_0000_node00000.vtr", "mm_0000.pvtr", "mm_collection.pvd",
             "energyChange.dat"]
    for n in names:
        assert filecmp.cmp(cdir / n, pdir / n, shallow=False), n


def test_cpp_commands_link_against_the_abi(tmp_path):
    """The GPU-facing commands compile and link against libcsrst_gpu.so (the
    entry points they call exist with the signatures they use)."""
    import pytest
    so_dir = ROOT / "csrst_b200"
    if not (so_dir / "libcsrst_gpu.so").exists():
        pytest.skip("libcsrst_gpu.so not built")
    exe = tmp_path / "diag_link"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/diag_link.cpp"),
                    "-L", str(so_dir), "-lcsrst_gpu", f"-Wl,-rpath,{so_dir}", "-o", str(exe)], check=True)
    assert exe.exists()
