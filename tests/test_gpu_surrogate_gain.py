"""The wake surrogate beats both predictors that use no network.

A small seeded data set (the first 384 cases of the seeded draw, each run
through the batched FP32 PIC with 20000 quiet-start particles) trains the
network for 6000 steps; on the held-out last 10 % its error against the PIC
wakes (relative L2 over the sampled bins) is compared with
 * the amplitude law times the mean normalised training wake, and
 * the nearest training case in the standardised inputs, rescaled by the
   amplitude law,
the two baselines `wakescreen.evaluate` reports beside the network.  The bar:
the network's mean error below half of the better baseline's mean and below
its median too, on every profile family together.  The measured figures are
printed (pytest -s) and written to the test's JSON record."""
import json
import os

import numpy as np
import pytest

from csrst_b200 import wakescreen as wsc
from csrst_b200 import wakeset as ws

pytestmark = pytest.mark.gpu

N_CASES, PARTICLES, STEPS = 384, 20_000, 6000


@pytest.fixture(scope="module")
def data(gpu_lib):
    return ws.generate(N_CASES, seed=7, n_particles=PARTICLES, batch=192, log=None)


def test_network_beats_no_network_baselines(data):
    keep = np.array([np.all(np.isfinite(w)) for w in data["W"]])
    d = {k: (np.asarray(v)[keep] if k in ("X", "W", "M") else v) for k, v in data.items()}
    d["cases"] = [c for c, k in zip(data["cases"], keep) if k]
    model, rec = wsc.train(d, steps=STEPS, batch=64, log=None)
    out, err = wsc.evaluate(model, d, log=None)
    net, mean_b, nn_b = out["surrogate"], out["baseline_mean_shape"], out["baseline_nearest_case"]
    line = {"cases": int(keep.sum()), "held_out": out["held_out"], "train_steps": STEPS,
            "train_s": rec["seconds"], "surrogate": net, "baseline_mean_shape": mean_b,
            "baseline_nearest_case": nn_b}
    print(json.dumps(line))
    path = os.environ.get("CSRST_GAIN_RECORD")
    if path:
        with open(path, "w") as f:
            json.dump(line, f)
    best = min(mean_b["mean"], nn_b["mean"])
    assert np.all(np.isfinite(err))
    assert net["mean"] < 0.5 * best
    assert net["median"] < 0.5 * min(mean_b["median"], nn_b["median"])
