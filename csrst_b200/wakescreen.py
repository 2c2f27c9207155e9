"""Training, evaluation and screening with the wake surrogate.

  python -m csrst_b200.wakescreen train --data wakes.npz --out model.npz
  python -m csrst_b200.wakescreen evaluate --data wakes.npz --model model.npz

A model is the network's parameters plus the output normalisation: each case's
wake is divided by an amplitude law exp(a . phi(x)) fitted by least squares on
the training cases (phi: the four log-scaled scalars, the log of the peak line
density and of its mean squared slope), then by one global rms, so that the
network fits O(1) values whose squared error weighs each case by its own
size.  The held-out cases (the last 10 % of the seeded draw) are judged
against their PIC wakes on the bins the PIC window sampled:
  error = || E_surrogate - E_PIC ||_2 / || E_PIC ||_2 over 256 bins x 32 stations.
"""
import json
import math
import time

import numpy as np
import torch

from .surrogate import FNO, NBINS, NFEAT

HOLDOUT = 0.1


def amp_features(X6):
    """phi(x) per case from the input channels [N][256][>= 6]."""
    lam = X6[:, :, 0].astype(np.float64)
    ds = 2.0 * 4.0 / NBINS
    slope = np.diff(lam, axis=1) / ds
    return np.stack([np.ones(len(X6)), X6[:, 0, 2], X6[:, 0, 3], X6[:, 0, 4], X6[:, 0, 5],
                     np.log(lam.max(axis=1)), np.log((slope ** 2).mean(axis=1) + 1e-12)], axis=1)


def fit_amplitude(X6, W, M):
    rms = np.sqrt(np.array([np.mean(W[k][M[k]] ** 2) for k in range(len(W))]))
    A = amp_features(X6)
    coef, *_ = np.linalg.lstsq(A, np.log(rms), rcond=None)
    return coef


def pad_features(X6):
    X = np.zeros((len(X6), NBINS, NFEAT), dtype=np.float32)
    X[:, :, :X6.shape[2]] = X6
    return X


class WakeModel:
    """Network + output normalisation."""

    def __init__(self, net, coef, tstd):
        self.net, self.coef, self.tstd = net, np.asarray(coef, dtype=np.float64), float(tstd)

    def scale(self, X6):
        return np.exp(amp_features(X6) @ self.coef) * self.tstd

    def predict(self, X6, chunk=4096):
        """Wakes [N][256][32] (V/m, numpy float32) for input channels [N][256][7]."""
        X = torch.from_numpy(pad_features(X6)).to(self.net.device).to(torch.bfloat16)
        y = self.net.predict(X, chunk=chunk).cpu().numpy()
        return y * self.scale(X6).astype(np.float32)[:, None, None]

    def save(self, path):
        np.savez(path, w=self.net.w.cpu().numpy(), coef=self.coef, tstd=self.tstd,
                 dims=np.array([self.net.width, self.net.modes, self.net.layers, self.net.nout]))

    @staticmethod
    def load(path, device="cuda"):
        z = np.load(path)
        w, m, L, nout = (int(v) for v in z["dims"])
        net = FNO(w, m, L, nout, device=device)
        net.w.copy_(torch.from_numpy(z["w"]))
        net.refresh()
        return WakeModel(net, z["coef"], float(z["tstd"]))


def split(n):
    k = int(round(n * (1 - HOLDOUT)))
    return np.arange(k), np.arange(k, n)


def rel_errors(P, W, M):
    return np.array([np.linalg.norm((P[k] - W[k])[M[k]]) / np.linalg.norm(W[k][M[k]]) for k in range(len(W))])


def train(d, steps=20000, batch=64, lr0=1e-3, lr_min=1e-5, seed=0, width=128, modes=32, layers=4, graph=True,
          log=print):
    """Trains a WakeModel on the training split of a data set; returns it and
    a record (losses, seconds, steps per second)."""
    tr, _ = split(len(d["X"]))
    X6, W, M = d["X"][tr], d["W"][tr], d["M"][tr]
    coef = fit_amplitude(X6, W, M)
    s = np.exp(amp_features(X6) @ coef)
    Tn = W / s[:, None, None]
    tstd = float(np.sqrt(np.mean(Tn ** 2)))
    Tn = (Tn / tstd).astype(np.float32)
    net = FNO(width, modes, layers, Tn.shape[2], seed=seed)
    dev = net.device
    Xd = torch.from_numpy(pad_features(X6)).to(dev).to(torch.bfloat16)
    Td = torch.from_numpy(Tn).to(dev)
    N = len(tr)
    Xs = torch.empty(batch, NBINS, NFEAT, dtype=torch.bfloat16, device=dev)
    Ts = torch.empty(batch, NBINS, Tn.shape[2], dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    per_epoch = N // batch
    state = {"perm": None, "pos": per_epoch}

    def fill():
        if state["pos"] >= per_epoch:
            state["perm"], state["pos"] = torch.randperm(N, generator=gen, device=dev), 0
        idx = state["perm"][state["pos"] * batch:(state["pos"] + 1) * batch]
        state["pos"] += 1
        torch.index_select(Xd, 0, idx, out=Xs)
        torch.index_select(Td, 0, idx, out=Ts)

    def one():
        loss = net.loss_and_grad(Xs, Ts)
        net.adam(lr0=lr0, lr_min=lr_min, total=steps)
        return loss

    losses = []
    fill()
    loss = one()                       # eager first step: buffers, launch attributes
    g = None
    if graph:
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            loss = one()
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    for it in range(1, steps):
        fill()
        if g is not None:
            g.replay()
        else:
            one()
        if it % 1000 == 0 or it == steps - 1:
            losses.append((it, float(loss.item())))
            if log:
                log("step %d loss %.4g (%.1f s)" % (it, losses[-1][1], time.perf_counter() - t))
    torch.cuda.synchronize(dev)
    sec = time.perf_counter() - t
    net.check()
    del g
    return WakeModel(net, coef, tstd), {"steps": steps, "batch": batch, "seconds": sec,
                                        "steps_per_s": (steps - 1) / sec, "losses": losses,
                                        "train_cases": int(N), "params": int(net.n)}


def evaluate(model, d, log=print):
    """Held-out errors against PIC, and the same for two baselines without
    the network: the amplitude law times the mean normalised training wake,
    and the nearest training case (in the standardised inputs) rescaled by the
    amplitude law."""
    tr, te = split(len(d["X"]))
    X6, W, M = d["X"], d["W"], d["M"]
    P = model.predict(X6[te])
    err = rel_errors(P, W[te], M[te])
    s_tr = model.scale(X6[tr])
    s_te = model.scale(X6[te])
    mean_shape = np.mean(W[tr] / s_tr[:, None, None], axis=0)
    err_mean = rel_errors(mean_shape[None] * s_te[:, None, None], W[te], M[te])
    F = np.concatenate([X6[:, :, 0], np.repeat(X6[:, :1, 2:6], 16, axis=1).reshape(len(X6), -1)], axis=1)
    F = (F - F[tr].mean(0)) / (F[tr].std(0) + 1e-9)
    nn = np.array([tr[np.argmin(((F[tr] - F[k]) ** 2).sum(1))] for k in te])
    Pnn = W[nn] / s_tr[np.searchsorted(tr, nn)][:, None, None] * s_te[:, None, None]
    err_nn = rel_errors(Pnn, W[te], M[te])

    def summary(e):
        return {"mean": float(e.mean()), "median": float(np.median(e)), "p90": float(np.quantile(e, 0.9)),
                "max": float(e.max()), "frac_le_2pct": float(np.mean(e <= 0.02))}

    kinds = np.array([c.kind for c in d["cases"]])[te]
    out = {"held_out": int(len(te)), "surrogate": summary(err),
           "by_family": {name: summary(err[kinds == k]) for k, name in enumerate(("gaussian", "flat_top", "double_horn"))},
           "baseline_mean_shape": summary(err_mean), "baseline_nearest_case": summary(err_nn)}
    if log:
        log(json.dumps(out))
    return out, err


def time_inference(model, X6, n=65536, chunk=8192, reps=3):
    """Profiles per second of the surrogate at inference batch n (inputs
    resident on the device; CUDA events around the whole batch)."""
    reps_x = (n + len(X6) - 1) // len(X6)
    X = torch.from_numpy(pad_features(np.concatenate([X6] * reps_x)[:n])).to(model.net.device).to(torch.bfloat16)
    model.net.predict(X, chunk=chunk)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        model.net.predict(X, chunk=chunk)
    b.record()
    torch.cuda.synchronize()
    sec = a.elapsed_time(b) / 1e3 / reps
    model.net.check()
    flops = _flops_per_profile(model.net) * n
    return {"profiles": n, "seconds": sec, "profiles_per_s": n / sec, "tflops": flops / sec / 1e12}


def _flops_per_profile(net):
    w, m, L, no = net.width, net.modes, net.layers, net.nout
    per_layer = 2 * NBINS * w * w + 2 * w * 2 * m * NBINS * 2 + 2 * m * (2 * w) * (2 * w)
    return 2 * NBINS * NFEAT * w + L * per_layer + 2 * NBINS * w * w + 2 * NBINS * w * no


def pic_seconds_per_case(d):
    f = d["facts"]
    return sum(x["seconds"] for x in f) / sum(x["members"] for x in f)


if __name__ == "__main__":
    import argparse
    from . import wakeset
    ap = argparse.ArgumentParser(description="train / evaluate the wake surrogate")
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--data", required=True, help="data files, comma-separated")
    ap.add_argument("--model", default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    d = wakeset.load(*a.data.split(","))
    if a.cmd == "train":
        m, rec = train(d, steps=a.steps, batch=a.batch, lr0=a.lr, seed=a.seed)
        print(json.dumps(rec))
        if a.out:
            m.save(a.out)
        evaluate(m, d)
    else:
        evaluate(WakeModel.load(a.model), d)
