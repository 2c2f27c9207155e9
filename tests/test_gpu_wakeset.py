"""The wake data set on the GPU: the batched station read (every member's
wake diagnostic enqueued without waiting, one copy back) gives exactly what
the blocking per-member diagnostic gives, and a small batch of cases runs
through the ensemble to finite wakes."""
import numpy as np
import pytest

from csrst_b200 import wakeset as ws

pytestmark = pytest.mark.gpu


def test_batched_station_read_matches_per_member_read(gpu_lib):
    from csrst_b200.pic import Ensemble, Simulation
    cases = ws.draw_cases(4)
    sims = []
    for c in cases:
        cfg, lb = ws.case_config(c)
        s = Simulation(cfg, fp32=True)
        s.load(*ws.case_bunch(c, cfg, lb, 20_000))
        s.initial_fields()
        sims.append(s)
    ens = Ensemble(sims)
    ens.step(ws.ENTRY_STEPS + 10)
    ens.sync()
    reader = ws._WakeReader(sims, [c.sigma_s for c in cases])
    got, ok = reader.read()
    for k, (s, c) in enumerate(zip(sims, cases)):
        ref, rok = ws.sample_wake(s, c.sigma_s)
        assert np.array_equal(got[k], ref) and np.array_equal(ok[k], rok)
    ens.close()


def test_small_batch_of_cases(gpu_lib):
    W, M, facts = ws.run_cases(ws.draw_cases(3), n_particles=20_000, batch=3, log=None)
    assert np.all(np.isfinite(W)) and M.mean() > 0.5
    assert facts[0]["steps"] == ws.station_steps()[-1]
