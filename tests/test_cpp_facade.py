"""The C++ facade (include/csrst/csrst.hpp) compiles and links against the C
ABI; on a GPU it solves the initial fields, runs the reference's loop body and
agrees with the Python mirror of the same call sequence."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def exe(gpu_lib, tmp_path_factory):
    out = tmp_path_factory.mktemp("cpp") / "step_main"
    so_dir = ROOT / "csrst_b200"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/step_main.cpp"),
                    "-L", str(so_dir), "-lcsrst_gpu", f"-Wl,-rpath,{so_dir}", "-o", str(out)], check=True)
    return out


def test_facade_builds(exe):
    assert exe.exists()


@pytest.mark.gpu
def test_facade_runs_the_loop(exe):
    from csrst_b200 import Simulation, TETMSolver, moveMesh
    from csrst_b200.workloads import workload
    r = subprocess.run([str(exe), "4"], capture_output=True, text=True, check=True)
    lines = {ln.split()[0]: ln.split()[1:] for ln in r.stdout.splitlines()}
    vals = [float(v) for v in lines["rmean"][:2]]
    assert np.isfinite(vals).all()
    its = [float(v) for v in lines["poisson"][3:6]]  # iterations of the three initial-field solves
    assert all(0 < k < 50 for k in its)
    cfg, _ = workload("small-1")
    assert cfg.Nx == 512 and cfg.Ny == 104
    # the Python mirror drives the same ABI entry points
    sim = Simulation(cfg)
    assert TETMSolver(sim).getDT() > 0
    sim.close()
    _ = moveMesh


@pytest.fixture(scope="module")
def views_exe(tmp_path_factory):
    out = tmp_path_factory.mktemp("cpp") / "views_main"
    so_dir = ROOT / "csrst_b200"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests/cpp/views_main.cpp"), "-L", str(so_dir), "-lcsrst_gpu",
                    f"-Wl,-rpath,{so_dir}", "-o", str(out)], check=True)
    return out


def test_reference_argument_lists_build(views_exe):
    """A caller written against the reference's argument lists (PoissonSolver,
    TETMSolver and PartBunch constructors and methods, moveMesh) with host
    views compiles and links."""
    assert views_exe.exists()


@pytest.mark.gpu
def test_reference_argument_lists_run(views_exe, tmp_path):
    """The views the C++ caller binds receive the device's fields: their
    checksums, the window domain and the centroid agree with the same
    sequence driven from Python (bit for bit for the window domain and the
    centroid, 1e-12 relative for the sums, which add in a different order)."""
    from csrst_b200 import Simulation, TETMSolver, moveMesh
    from csrst_b200.workloads import make_bunch, workload
    cfg, spec = workload("small-1")
    b = make_bunch(spec)
    path = tmp_path / "bunch.bin"
    np.concatenate([np.asarray(v, dtype=np.float64) for v in b]).tofile(path)
    r = subprocess.run([str(views_exe), "5", str(path)], capture_output=True, text=True, check=True)
    out = {ln.split()[0]: [float(v) for v in ln.split()[1:]] for ln in r.stdout.splitlines()}
    sim = Simulation(cfg)
    sim.load(*b)
    sim.initial_fields()
    ex, ey, hx, hy = sim.get_static()
    assert np.isclose(out["poisson"][0], np.abs(ex).sum(), rtol=1e-12, atol=0)
    solver = TETMSolver(sim)
    for _ in range(5):
        solver.updateField_firstStep()
        solver.updateField_secondStep()
        moveMesh(sim)
    w, _, _ = sim.window()
    assert out["ddim"] == [w[0], w[0] + w[2] - 1, w[1], w[1] + w[3] - 1]
    for got, f in zip(out["static"], sim.get_static()):
        assert np.isclose(got, np.abs(f).sum(), rtol=1e-12, atol=0)
    for got, k in zip(out["window"], (0, 1, 5)):
        wf = sim.window_field(k)[1:-1, 1:-1]
        assert np.isclose(got, np.abs(wf).sum(), rtol=1e-12, atol=0)
    m = sim.moments()
    assert out["rmean"] == [m[0], m[1]]
    sim.close()
