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


def test_calibration_scales_spread_and_flags_the_training_edge():
    """k is the 0.9 quantile of error / spread on held-out cases; a variant
    with a scalar input beyond the training cases' 1 % / 99 % quantiles is
    at the edge; the prescreen reruns edge cases first, then the calibrated
    uncertain ones, within its budget."""
    g = np.random.default_rng(4)
    spreads = g.uniform(0.005, 0.02, 400)
    errors = spreads * g.uniform(0.5, 3.0, 400)
    cases = wakeset.draw_cases(200, seed=3)
    Xtr = wakeset.features(cases)
    cal = ws.calibrate(errors, spreads, Xtr)
    assert abs(cal.k - np.quantile(errors / spreads, 0.9)) < 1e-12 and 2.0 < cal.k < 3.0
    assert not cal.edge(Xtr[10:20]).any() or cal.edge(Xtr[10:20]).mean() < 0.5
    far = Xtr[:1].copy()
    far[:, :, 2] = Xtr[:, 0, 2].max() + 1.0      # a log-scaled run parameter past every training case
    assert cal.edge(far).all()
    variants = ws.c5_variants(30)
    g2 = np.random.default_rng(1)
    base = torch.from_numpy(g2.uniform(0.5, 2.0, 30)).float()
    noisy = base.clone()
    noisy[[4, 9]] *= 1.02                       # spread 1 %: over 2 % once calibrated (k > 2)
    models = [_Model(base), _Model(noisy)]
    _, _, _, unc0, rec0 = ws.prescreen(models, variants, top=3, unc_limit=0.02, max_reruns=30, log=None)
    assert rec0["over_unc_limit"] == 0
    cal_nowedge = ws.Calibration(k=cal.k, lo=np.full(6, -np.inf), hi=np.full(6, np.inf), q=0.9, q_edge=0.01)
    rerun, best, _, unc1, rec1 = ws.prescreen(models, variants, top=3, unc_limit=0.02, max_reruns=30, log=None,
                                               calib=cal_nowedge)
    assert np.allclose(unc1, cal.k * unc0) and rec1["over_unc_limit"] >= 1
    assert set(np.nonzero(unc1 > 0.02)[0]) <= {4, 9}
    assert rec1["at_training_edge"] == 0 and rec1["calibrated"]
    Xv = wakeset.features(variants)
    z = ws.scalar_inputs(Xv)
    cal_edge = ws.Calibration(k=1.0, lo=np.full(6, -np.inf), hi=z.max(0) - 1e-9, q=0.9, q_edge=0.01)
    rerun, best, _, _, rec2 = ws.prescreen(models, variants, top=3, unc_limit=0.02, max_reruns=8, log=None,
                                           calib=cal_edge)
    assert rec2["at_training_edge"] >= 1 and len(rerun) <= 8
    edge = cal_edge.edge(Xv)
    extra = [k for k in rerun if k not in set(best)]
    assert all(edge[k] for k in extra[:int(edge.sum())] if k not in set(best))
