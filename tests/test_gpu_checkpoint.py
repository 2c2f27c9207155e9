"""Checkpoint and restart (the restart dump LoadH5Part reads,
src/Commands/LoadH5Part.cpp:60-321, as a dependency-free binary file): a run
saved after some steps and restored into a new handle of the same
configuration continues bit for bit, in both precision modes; a file written
for another configuration is refused."""
import os
import tempfile

import numpy as np
import pytest

from csrst_b200 import CsrstError, Simulation
from csrst_b200.workloads import make_bunch, workload

pytestmark = pytest.mark.gpu


def state(s):
    return s.particles() + [s.window_field(k) for k in range(6)] + s.get_static() + [np.array(s.window()[0])]


@pytest.mark.parametrize("name,fp32", [("small-1", False), ("small-2", True), ("small-1-bend", True)])
def test_restart_continues_bitwise(gpu_lib, name, fp32):
    cfg, spec = workload(name)
    a = Simulation(cfg, fp32=fp32)
    a.load(*make_bunch(spec))
    if "bend" not in name:
        a.initial_fields()
    a.step(5)
    path = os.path.join(tempfile.mkdtemp(), "run.ckpt")
    a.checkpoint(path, step=5, time=5 * a.info()["dt"])
    a.step(7)
    b = Simulation(cfg, fp32=fp32)
    st, tm = b.restore(path)
    assert st == 5 and tm == 5 * a.info()["dt"] and b.n == a.n
    b.step(7)
    for x, y in zip(state(a), state(b)):
        assert np.array_equal(x, y)
    os.remove(path)


def test_restart_refuses_other_configuration(gpu_lib):
    cfg, spec = workload("small-1")
    a = Simulation(cfg)
    a.load(*make_bunch(spec))
    path = os.path.join(tempfile.mkdtemp(), "run.ckpt")
    a.checkpoint(path)
    other, _ = workload("small-2")
    with pytest.raises(CsrstError):
        Simulation(other).restore(path)
    with pytest.raises(CsrstError):
        Simulation(cfg, fp32=True).restore(path)
    with open(path, "r+b") as f:      # a truncated file
        f.truncate(200)
    with pytest.raises(CsrstError):
        Simulation(cfg).restore(path)
    os.remove(path)
