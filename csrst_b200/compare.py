"""FP32 mode against the FP64 path on one workload (no reference counterpart:
the reference computes in FP64 only).

Both precisions run the same seeded bunch from the same initial fields;
every `every` steps the longitudinal field on the bunch axis
(IntegrateElongCommand's samples, IntegrateElong.cpp:38-89) is taken from
both and summed per static-mesh column, which is the time-integrated energy
change per unit charge the reference writes (energyChange*.dat, up to its
-dt factor).  Reported against the FP64 path, relative to its maximum:
 * wake_rel_err: the last samples;
 * integrated_rel_err: the sums over the run;
 * slice_rel_err: the energy change of 16 longitudinal slices of the bunch
   (gamma of every particle, start to end, binned by the FP64 positions).
"""
import numpy as np

from .pic import Simulation
from .workloads import make_bunch, workload


def _samples(sim):
    """Wake samples keyed by absolute static column (window columns 2 .. L0-3)."""
    w, _, _ = sim.window()
    v = sim.wake()
    cols = w[0] + 2 + np.arange(len(v))
    return dict(zip(cols.tolist(), v.tolist()))


def fp32_vs_fp64(name, steps, every=100, initial_fields=None):
    cfg, spec = workload(name)
    bunch = make_bunch(spec)
    if initial_fields is None:  # the Poisson solve covers the first straight section only
        initial_fields = "bend" not in name
    runs = {}
    for fp32 in (False, True):
        s = Simulation(cfg, fp32=fp32)
        s.load(*bunch)
        if initial_fields:
            s.initial_fields()
        _, _, px, py = s.particles()
        g0 = np.sqrt(1.0 + px * px + py * py)
        acc, last, done = {}, {}, 0
        while done < steps:
            k = min(every, steps - done)
            s.step(k)
            done += k
            last = _samples(s)
            for c, v in last.items():
                if np.isfinite(v):
                    acc[c] = acc.get(c, 0.0) + v
        x, y, px, py = s.particles()
        runs[fp32] = {"last": last, "acc": acc, "dg": np.sqrt(1.0 + px * px + py * py) - g0, "x": x, "y": y,
                      "m": s.moments(), "window": s.window()[0]}
        s.close()

    def rel(a, b):
        keys = [k for k in b if k in a and np.isfinite(a[k]) and np.isfinite(b[k])]
        av, bv = np.array([a[k] for k in keys]), np.array([b[k] for k in keys])
        return float(np.abs(av - bv).max() / np.abs(bv).max()), len(keys)

    r64, r32 = runs[False], runs[True]
    wake_err, n_last = rel(r32["last"], r64["last"])
    int_err, n_acc = rel(r32["acc"], r64["acc"])
    m = r64["m"]
    c, sn = m[2] / np.hypot(m[2], m[3]), m[3] / np.hypot(m[2], m[3])
    sl = (r64["x"] - m[0]) * c + (r64["y"] - m[1]) * sn
    idx = np.clip(np.digitize(sl, np.linspace(-3 * spec.sigma_s, 3 * spec.sigma_s, 17)) - 1, 0, 15)
    cnt = np.maximum(np.bincount(idx, minlength=16), 1)
    e64 = 0.511 * np.bincount(idx, r64["dg"], minlength=16) / cnt
    e32 = 0.511 * np.bincount(idx, r32["dg"], minlength=16) / cnt
    return {"workload": name, "steps": steps, "sample_every": every,
            "wake_rel_err": wake_err, "wake_samples": n_last,
            "integrated_rel_err": int_err, "integrated_columns": n_acc,
            "slice_rel_err": float(np.abs(e32 - e64).max() / np.abs(e64).max()),
            "slice_mev_fp64": e64.tolist(), "same_window": r64["window"] == r32["window"]}
