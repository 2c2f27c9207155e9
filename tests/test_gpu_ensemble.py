"""Batched ensemble: independent members of different meshes, shape orders and
bunch sizes stepped together (one launch per phase, one CUDA graph per step).
Every member must end bitwise in the state its own unbatched run reaches."""
import numpy as np
import pytest

from csrst_b200 import CsrstError, Ensemble, Simulation
from csrst_b200.workloads import ensemble_members, make_bunch, workload

pytestmark = pytest.mark.gpu

NAMES = ["small-0", "small-1", "small-2", "small-1-bend", "c1"]


def members(fp32, names=NAMES, fields=True):
    sims = []
    for name in names:
        cfg, spec = workload(name)
        s = Simulation(cfg, fp32=fp32)
        s.load(*make_bunch(spec))
        if fields and "bend" not in name:
            s.initial_fields()
        sims.append(s)
    return sims


def state(s):
    return s.particles() + [s.window_field(k) for k in range(6)] + s.get_static() + [np.array(s.window()[0])]


def assert_same(a, b):
    for x, y in zip(state(a), state(b)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("fp32", [False, True])
def test_ensemble_matches_single_runs(gpu_lib, fp32):
    batch, single = members(fp32), members(fp32)
    ens = Ensemble(batch)
    ens.step(5)
    ens.step(4)
    ens.sync()
    for s in single:
        s.step(9)
    for a, b in zip(batch, single):
        assert_same(a, b)
    # the members stay usable on their own after batched steps
    for a, b in zip(batch, single):
        a.step(2)
        b.step(2)
        assert_same(a, b)
    ens.close()


def test_launch_shapes_do_not_change_results(gpu_lib):
    """Sub-step tiles of two shapes and the fused sweep (tx = ty = 0, one
    persistent launch over a work queue) give the same states."""
    runs = []
    for shape in ((148, 32, 8, 1), (1184, 128, 2, 3), (592, 0, 0, 2)):
        sims = members(True, NAMES[:4])
        ens = Ensemble(sims)
        ens.set_shape(*shape)
        ens.step(6)
        ens.sync()
        runs.append([state(s) for s in sims])
        ens.close()
    for other in runs[1:]:
        for ma, mb in zip(runs[0], other):
            for x, y in zip(ma, mb):
                assert np.array_equal(x, y)


def test_autotuner_steps_are_real_steps(gpu_lib):
    sims, ref = members(False, NAMES[:3]), members(False, NAMES[:3])
    ens = Ensemble(sims)
    rows = ens.tune(steps=1)
    assert len(rows) == 27 and all(r[4] > 0 for r in rows)
    assert {(r[1], r[2]) for r in rows} == {(0, 0), (32, 8), (128, 2)}
    ens.step(2)
    ens.sync()
    # one step to reach the steady state of the loop, then 27 shapes x (1 warm-up + 1 timed), then 2
    for s in ref:
        s.step(1 + 27 * 2 + 2)
    for a, b in zip(sims, ref):
        assert_same(a, b)
    ens.close()


def test_ensemble_workload_generator_members_build(gpu_lib):
    """The 64-member workload: every member's geometry builds and a sample of
    members loads and steps in one batch."""
    ms = ensemble_members(64)
    assert len(ms) == 64
    assert 1024 <= min(c.Nx for c, _ in ms) and max(c.Nx for c, _ in ms) <= 8192
    assert {c.shape_order for c, _ in ms} == {0, 1}
    sims = []
    for cfg, spec in ms[:6]:
        spec.n = 20_000
        s = Simulation(cfg, fp32=True)
        s.load(*make_bunch(spec))
        sims.append(s)
    ens = Ensemble(sims)
    ens.step(3)
    ens.sync()
    ens.close()


def test_mixed_precision_rejected(gpu_lib):
    a, b = members(False, ["small-0"]), members(True, ["small-1"])
    with pytest.raises(CsrstError):
        Ensemble(a + b)


@pytest.mark.parametrize("fp32", [False, True])
def test_staging_wait_that_gives_up(gpu_lib, fp32):
    """The fused sweep's staging waits are bounded.  With the stuck-wait hook
    (every staging wait on a barrier nothing completes, 200 polls) a batched
    step and a single handle's step report CSRST_E_STAGING instead of
    hanging; with the default limit restored, new members step correctly
    (the context is intact)."""
    from csrst_b200._lib import lib
    try:
        lib().csrst_set_staging_wait_limit(-200)
        sims = members(fp32, NAMES[:2], fields=False)
        ens = Ensemble(sims)
        ens.step(3)
        with pytest.raises(CsrstError) as ei:
            ens.sync()
        assert ei.value.code == -10
        ens.close()
        one = members(fp32, ["small-1"], fields=False)[0]
        with pytest.raises(CsrstError) as ei:
            one.step(3)
            one.sync()
        assert ei.value.code == -10
    finally:
        lib().csrst_set_staging_wait_limit(0)
    batch, single = members(fp32, NAMES[:2], fields=False), members(fp32, NAMES[:2], fields=False)
    ens = Ensemble(batch)
    ens.step(4)
    ens.sync()
    for s in single:
        s.step(4)
    for a, b in zip(batch, single):
        assert_same(a, b)
    ens.close()
