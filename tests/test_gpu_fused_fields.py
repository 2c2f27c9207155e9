"""The fused static sweep against the sub-step kernels, bit for bit.

csrst_step runs the static mesh's four field sub-steps (half H, Ex, half H,
Ey) as one TMA-staged pass from one plane set into the other, redoes the
cells around the window with the window's sub-steps and strip exchanges,
and swaps the sets every step (one CUDA graph per set).  A handle created
with CSRST_FLAG_SUBSTEP_FIELDS runs one launch per sub-step instead.  Both
must give the same particles, window position, static fields and window
fields after every step count: eager first steps, odd and even counts (both
graphs), every shape order, FP64 and FP32, through the dipole (window moves
in y), an ensemble in between (whose members' own steps fall back to the
sub-step kernels while it exists), and a checkpoint restored into either
plane set."""
import numpy as np
import pytest

from csrst_b200.pic import Ensemble, Simulation
from csrst_b200.workloads import make_bunch, workload

pytestmark = pytest.mark.gpu


def fields(cfg, seed):
    """Smooth random static fields (V/m; A/m for the H parts)."""
    rng = np.random.default_rng(seed)
    j, i = np.mgrid[0:cfg.Ny, 0:cfg.Nx]
    out = []
    for k in range(4):
        kx, ky = rng.uniform(0.01, 0.2, 2)
        f = rng.uniform(0.5, 1) * np.sin(kx * i + rng.uniform(0, 6)) * np.cos(ky * j + rng.uniform(0, 6))
        out.append(f * (2e5 if k < 2 else 2e5 / 376.73))
    return out


def pair(name, fp32, seed=3):
    cfg, spec = workload(name)
    bunch = make_bunch(spec)
    f = fields(cfg, seed)
    sims = []
    for sub in (False, True):
        s = Simulation(cfg, fp32=fp32, substep_fields=sub)
        s.set_static(*f)
        s.load(*bunch)
        sims.append(s)
    return sims


def assert_same(a, b):
    wa, oa, ga = a.window()
    wb, ob, gb = b.window()
    assert wa == wb and np.array_equal(oa, ob) and ga == gb
    for x, y in zip(a.particles(), b.particles()):
        assert np.array_equal(x, y)
    for x, y in zip(a.get_static(), b.get_static()):
        assert np.array_equal(x, y)
    for k in range(6):
        assert np.array_equal(a.window_field(k), b.window_field(k)), k


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("name", ["small-0", "small-1", "small-2", "small-1-bend", "small-2-bend"])
def test_fused_sweep_matches_substep_kernels(gpu_lib, fp32, name):
    a, b = pair(name, fp32)
    moves = set()
    for n in (1, 2, 7, 30, 121):
        a.step(n)
        b.step(n)
        assert_same(a, b)
        moves.add(tuple(a.window()[0][:2]))
    assert len(moves) > 1
    for s in (a, b):
        s.close()


@pytest.mark.parametrize("fp32", [False, True])
def test_fused_sweep_moves_in_y_through_the_dipole(gpu_lib, fp32):
    """c1-bend (2048 x 512 at 10 um, R = 1 m) for 1000 steps from the dipole
    entrance: the window follows the arc in y."""
    a, b = pair("c1-bend", fp32)
    p1 = {a.window()[0][1]}
    for _ in range(5):
        a.step(200)
        b.step(200)
        p1.add(a.window()[0][1])
    assert_same(a, b)
    assert len(p1) > 1
    for s in (a, b):
        s.close()


@pytest.mark.parametrize("fp32", [False, True])
def test_fused_sweep_c1_full_size(gpu_lib, fp32):
    """The 2048 x 512 mesh with 2e5 particles, 40 steps."""
    a, b = pair("c1", fp32)
    a.step(40)
    b.step(40)
    assert_same(a, b)
    for s in (a, b):
        s.close()


def test_ensemble_in_between(gpu_lib):
    """Fused steps, then 10 ensemble steps (the member's own steps use the
    sub-step kernels while the ensemble exists), then fused steps again."""
    a, b = pair("small-1", True)
    c, d = pair("small-2", True, seed=5)
    a.step(5)
    b.step(5)
    ens = Ensemble([a, c])
    ens.step(10)
    ens.sync()
    a.step(3)            # inside the ensemble's lifetime
    ens.close()
    b.step(13)
    assert_same(a, b)
    a.step(9)
    b.step(9)
    assert_same(a, b)
    for s in (a, b, c, d):
        s.close()


@pytest.mark.parametrize("fp32", [False, True])
def test_checkpoint_into_either_set(gpu_lib, fp32, tmp_path):
    """A checkpoint taken after an odd step count (the second plane set
    current) restores into a handle whose current set is the first one."""
    a, b = pair("small-1-bend", fp32)
    cfg, spec = workload("small-1-bend")
    c = Simulation(cfg, fp32=fp32)
    c.set_static(*fields(cfg, 3))
    c.load(*make_bunch(spec))
    a.step(7)
    path = str(tmp_path / "ck.bin")
    a.checkpoint(path, step=7)
    c.step(6)
    c.restore(path)
    a.step(11)
    c.step(11)
    b.step(18)
    assert_same(a, c)
    assert_same(a, b)
    for s in (a, b, c):
        s.close()
