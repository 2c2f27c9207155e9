"""The production run's checkpointing: a run stopped after half its stations
and resumed from its checkpoint gives the same wakes, bit for bit, as the run
that went straight through (a reduced mesh and bunch: 8192 x 512 cells of
10 um, 1e5 particles, 64 steps)."""
import numpy as np
import pytest

from csrst_b200 import wakescreen as ws

pytestmark = pytest.mark.gpu


def test_production_resume_matches_uninterrupted(gpu_lib, tmp_path):
    cfg = ws.production_config(nx=8192, ny=512, h=10e-6, width=4e-3, cfl=0.4)
    case = ws.c5_variants(1)[0]
    W, rec = ws.production_run(case, n=100_000, steps=64, stations=4, cfg=cfg, log=None)
    assert W.shape == (256, 4) and rec["steps"] == 64 and np.all(np.isfinite(W))
    ck = tmp_path / "production.ckpt"
    Wa, _ = ws.production_run(case, n=100_000, steps=32, stations=2, cfg=cfg, log=None, checkpoint=ck)
    Wb, rb = ws.production_run(case, n=100_000, steps=64, stations=4, cfg=cfg, log=None, resume=ck)
    assert rb["first_step"] == 32 and rb["steps"] == 32
    assert np.array_equal(np.concatenate([Wa, Wb], axis=1), W)
