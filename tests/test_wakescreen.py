"""The production prescreen's selection rule and objective on the CPU, with
stand-in models (the network itself is tested on the GPU)."""
import numpy as np
import torch

from csrst_b200 import wakescreen as ws, wakeset


class _Net:
    device = torch.device("cpu")

    def __init__(self, gain):
        self.gain = gain

    def predict(self, X, chunk=0):
        # wake at the last station: the density slope times a per-model, per-variant gain
        slope = X[:, :, 6].float()
        return (slope[:, :, None] * self.gain[:, None, None]).expand(-1, -1, 32).contiguous()


class _Model:
    def __init__(self, gain):
        self.net = _Net(gain)

    def scale(self, X6):
        return np.ones(len(X6))


def test_objective_is_weighted_rms_over_the_bunch():
    X6 = np.zeros((2, wakeset.NBINS, 7), dtype=np.float32)
    X6[:, 100:156, 0] = 1.0
    W = np.zeros((2, wakeset.NBINS, 32))
    W[0, 100:128, -1], W[0, 128:156, -1] = 1.0, -1.0     # +-1 over the bunch: rms 1
    W[1, :, -1] = 5.0                                    # uniform: no spread
    W[1, :100, -1] = 100.0                               # outside the bunch: no weight
    J = ws.objective(X6, W)
    assert abs(J[0] - 1.0) < 1e-12 and abs(J[1]) < 1e-12


def test_prescreen_picks_best_then_uncertain():
    cases = ws.c5_variants(40)
    assert cases[0].horn_pos == 0.8 and abs(cases[0].sigma_s / ws.C5_HALF_LENGTH - wakeset.profile(cases[0])[3]) < 1e-6
    g = np.random.default_rng(0)
    base = torch.from_numpy(g.uniform(0.5, 2.0, 40)).float()
    noisy = base.clone()
    noisy[[3, 7, 11]] *= 1.2                             # three variants the models disagree on
    models = [_Model(base), _Model(noisy)]
    rerun, best, mean, unc, rec = ws.prescreen(models, cases, top=5, unc_limit=0.02, max_reruns=7, log=None)
    assert list(best) == list(np.argsort(mean)[:5])
    assert set(np.nonzero(unc > 0.02)[0]) == {3, 7, 11}
    extra = [k for k in rerun if k not in set(best)]
    assert len(rerun) <= 7 and set(extra) <= {3, 7, 11}
    assert rec["variants"] == 40 and rec["over_unc_limit"] == 3
