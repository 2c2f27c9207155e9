"""Training, evaluation and screening with the wake surrogate.

  python -m csrst_b200.wakescreen train --data wakes.npz --out model.npz
  python -m csrst_b200.wakescreen evaluate --data wakes.npz --model model.npz
  python -m csrst_b200.wakescreen time --n 65536          (inference throughput)

A model is the network's parameters plus the output normalisation: each case's
wake is divided by an amplitude law exp(a . phi(x)) fitted by least squares on
the training cases (phi: the four log-scaled scalars, the log of the peak line
density and of its mean squared slope), then by one global rms, so that the
network fits O(1) values whose squared error weighs each case by its own
size.  The held-out cases (the last 10 % of the seeded draw) are checked
against their PIC wakes on the bins the PIC window sampled:
  error = || E_surrogate - E_PIC ||_2 / || E_PIC ||_2 over 256 bins x 32 stations.
"""
import dataclasses
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
    Md = torch.from_numpy(M.astype(np.float32)).to(dev)    # bins outside the PIC window carry no target
    N = len(tr)
    Xs = torch.empty(batch, NBINS, NFEAT, dtype=torch.bfloat16, device=dev)
    Ts = torch.empty(batch, NBINS, Tn.shape[2], dtype=torch.float32, device=dev)
    Ms = torch.empty(batch, NBINS, Tn.shape[2], dtype=torch.float32, device=dev)
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
        torch.index_select(Md, 0, idx, out=Ms)

    def one():
        loss = net.loss_and_grad(Xs, Ts, Ms)
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


SHIFTS = (0.0, 0.25, 0.5, 0.75)


def pic_reference(cases, n_particles=50_000, batch=256, log=print):
    """The alignment-averaged PIC wake of each case: the case run with its
    bunch shifted by 0, 1/4, 1/2 and 3/4 of a cell, averaged.  A single run
    depends on where sub-cell features (horns, sharp edges) fall on the mesh:
    half a cell moves a double-horn wake by 6 - 9 %, a flat top's by 1 - 4 %,
    a Gaussian's by about 1 %; the average over the cell is what a
    resolution-limited PIC determines.  Returns (mean wake, mask of bins every
    run sampled, per-shift wakes)."""
    from . import wakeset
    runs, masks = [], []
    for sh in SHIFTS:
        w, m, _ = wakeset.run_cases(cases, n_particles=n_particles, batch=batch, log=log, shift=sh)
        runs.append(w)
        masks.append(m)
    runs = np.array(runs)
    return runs.mean(0), np.logical_and.reduce(masks), runs


def evaluate(model, d, log=print, ref=None):
    """Held-out errors against PIC, and the same for two baselines without
    the network: the amplitude law times the mean normalised training wake,
    and the nearest training case (in the standardised inputs) rescaled by the
    amplitude law.  ref = (wakes, masks) of the held-out cases from
    pic_reference() makes the alignment-averaged PIC wake the reference and adds
    the single runs' own scatter about it."""
    tr, te = split(len(d["X"]))
    X6, W, M = d["X"], d["W"].copy(), d["M"].copy()
    single = None
    if ref is not None:
        single = rel_errors(W[te], ref[0], ref[1])
        W[te], M[te] = ref[0], ref[1]
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
    fam = ("gaussian", "flat_top", "double_horn")
    out = {"held_out": int(len(te)), "checked_against": "alignment-averaged PIC" if ref is not None else "single PIC run",
           "surrogate": summary(err),
           "by_family": {name: summary(err[kinds == k]) for k, name in enumerate(fam)},
           "baseline_mean_shape": summary(err_mean), "baseline_nearest_case": summary(err_nn)}
    if single is not None:
        out["single_pic_run_vs_average"] = summary(single)
        out["single_pic_run_by_family"] = {name: summary(single[kinds == k]) for k, name in enumerate(fam)}
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
    byts = bytes_per_profile(model.net) * n
    return {"profiles": n, "seconds": sec, "profiles_per_s": n / sec, "tflops": flops / sec / 1e12,
            "gbs": byts / sec / 1e9, "bytes_per_profile": bytes_per_profile(model.net),
            "flops_per_profile": _flops_per_profile(model.net)}


def bytes_per_profile(net):
    """Bytes the forward pass must move per profile in this layer sequence
    (BF16 activations, each written once and read once per use): the lift
    reads the 64 input features and writes V; a layer reads V (forward DFT),
    writes and reads the spectra (mode mixing), the mixed spectra (and their
    regrouping), reads them and V again (inverse DFT + pointwise product) and
    writes the next V; the projection reads V, writes and reads its hidden
    layer and writes the FP32 output."""
    w, m, L, no = net.width, net.modes, net.layers, net.nout
    act = NBINS * w * 2                       # one activation tensor
    spec = 2 * m * w * 2                      # spectra of one layer
    lift = NBINS * NFEAT * 2 + act
    layer = act + 2 * spec + 2 * spec + 2 * spec + act + act
    proj = act + act + act + NBINS * no * 4
    return lift + L * layer + proj


def _flops_per_profile(net):
    w, m, L, no = net.width, net.modes, net.layers, net.nout
    per_layer = 2 * NBINS * w * w + 2 * w * 2 * m * NBINS * 2 + 2 * m * (2 * w) * (2 * w)
    return 2 * NBINS * NFEAT * w + L * per_layer + 2 * NBINS * w * w + 2 * NBINS * w * no


# ---- production: surrogate prescreen of profile variants, PIC reruns, the large run ----

C5_HALF_LENGTH = 50e-6      # flat top of 100 um
C5_GAMMA, C5_R = 2000.0, 2.0


def c5_variants(n, seed=5):
    """n double-horn variants of the production bunch (flat top of 100 um;
    horns at +-horn_pos x 50 um of rms width horn_w x 50 um), drawn over the
    training ranges of the double-horn family, at gamma = 2000, R = 2 m and a
    pipe of 80 sigma_s.  Variant 0 is the nominal profile: horns of 5 um at
    +-40 um, sharp edges, no tilt."""
    from . import wakeset
    g = np.random.Generator(np.random.Philox(seed))
    out = []
    for k in range(n):
        if k == 0:
            e, t, hp, hw, a, b = 0.05, 0.0, 0.8, 0.1, 1.5, 1.5
        else:
            e, t = g.uniform(0.05, 0.3), g.uniform(-0.3, 0.3)
            hp, hw = g.uniform(0.7, 0.95), g.uniform(0.04, 0.12)
            a, b = g.uniform(0.5, 2.5), g.uniform(0.5, 2.5)
        out.append(wakeset.WakeCase(kind=2, edge=float(e), tilt=float(t), horn_pos=float(hp), horn_w=float(hw),
                                    horn_a=float(a), horn_b=float(b), sigma_s=1.0, gamma=C5_GAMMA, R=C5_R,
                                    width_sigma=80.0, seed=int(g.integers(1, 2 ** 31))))
    rms = wakeset.moments_batch(out)[2]
    return [dataclasses.replace(c, sigma_s=float(r * C5_HALF_LENGTH)) for c, r in zip(out, rms)]


def objective(X6, W):
    """Charge-weighted rms of the wake over the bunch at the last station
    (the correlated energy-spread rate the bend imprints); lower is better."""
    lam = np.maximum(X6[:, :, 0].astype(np.float64), 0)
    e = W[:, :, -1].astype(np.float64)
    wsum = lam.sum(1)
    mean = (lam * e).sum(1) / wsum
    return np.sqrt((lam * (e - mean[:, None]) ** 2).sum(1) / wsum)


def scalar_inputs(X6):
    """A case's scalar inputs: the four log-scaled run parameters (gamma, R,
    sigma_s, pipe width) and the log peak line density and log mean squared
    slope of its profile (the amplitude law's features without the constant)."""
    return amp_features(X6)[:, 1:]


@dataclasses.dataclass
class Calibration:
    """The ensemble spread turned into an error estimate, from held-out cases.

    spread  = ensemble standard deviation / |ensemble mean| of a prediction;
    error   ~ k * spread, k the q-quantile over the held-out cases of
              (relative wake error against PIC) / (relative wake spread);
    edge    = a scalar input outside the [q_edge, 1 - q_edge] quantile range of
              the training cases: an extrapolation, where the networks can share
              a bias their spread does not show.
    """
    k: float
    lo: np.ndarray
    hi: np.ndarray
    q: float
    q_edge: float

    def edge(self, X6):
        z = scalar_inputs(X6)
        return np.any((z < self.lo) | (z > self.hi), axis=1)


def wake_spread(preds):
    """Relative spread of an ensemble's wake predictions [models][N][bins][stations]."""
    P = np.asarray(preds, dtype=np.float64)
    sd = P.std(0).reshape(P.shape[1], -1)
    mn = P.mean(0).reshape(P.shape[1], -1)
    return np.linalg.norm(sd, axis=1) / np.maximum(np.linalg.norm(mn, axis=1), 1e-300)


def calibrate(errors, spreads, X6_train, q=0.9, q_edge=0.01):
    """Calibration from held-out relative errors and spreads and the training
    cases' inputs (see Calibration)."""
    ratio = np.asarray(errors) / np.maximum(np.asarray(spreads), 1e-12)
    z = scalar_inputs(X6_train)
    return Calibration(k=float(np.quantile(ratio, q)), lo=np.quantile(z, q_edge, axis=0),
                       hi=np.quantile(z, 1 - q_edge, axis=0), q=q, q_edge=q_edge)


def prescreen(models, cases, top=16, unc_limit=0.02, max_reruns=256, chunk=8192, log=print, calib=None):
    """Objective of every variant under each model of an ensemble; returns
    the variants to rerun in PIC (the `top` best by the ensemble mean, then
    every variant whose uncertainty exceeds unc_limit of its mean, most
    uncertain first, up to max_reruns in all: PIC runs are the budget), with
    the screen's timing.  The uncertainty is the ensemble spread, or with a
    Calibration k times the spread, and every variant at the edge of the
    training inputs counts as uncertain (ahead of the rest)."""
    from . import wakeset
    t = time.perf_counter()
    X6 = wakeset.features(cases)
    t_feat = time.perf_counter() - t
    J = []
    sync = torch.cuda.synchronize if torch.cuda.is_available() else (lambda: None)
    sync()
    t = time.perf_counter()
    for m in models:
        X = torch.from_numpy(pad_features(X6)).to(m.net.device).to(torch.bfloat16)
        W = m.net.predict(X, chunk=chunk)[:, :, -1:].cpu().numpy()
        J.append(objective(X6, W * m.scale(X6)[:, None, None]))
    sync()
    t_net = time.perf_counter() - t
    J = np.array(J)
    mean, unc = J.mean(0), J.std(0) / J.mean(0)
    edge = np.zeros(len(cases), dtype=bool)
    if calib is not None:
        unc = calib.k * unc
        edge = calib.edge(X6)
    best = np.argsort(mean)[:top]
    bset = set(best.tolist())
    order = np.lexsort((-unc, ~edge))          # edge cases first, then by uncertainty
    risky = [k for k in order if (unc[k] > unc_limit or edge[k]) and k not in bset]
    rerun = list(best) + risky[:max(0, max_reruns - top)]
    rec = {"variants": len(cases), "models": len(models), "features_s": t_feat, "network_s": t_net,
           "over_unc_limit": int(np.sum(unc > unc_limit)), "at_training_edge": int(edge.sum()),
           "uncertain": int(np.sum((unc > unc_limit) | edge)), "reruns": len(rerun),
           "rerun_budget": max_reruns, "calibrated": calib is not None,
           "unc_median": float(np.median(unc)), "unc_p99": float(np.quantile(unc, 0.99))}
    if log:
        log(json.dumps(rec))
    return np.array(rerun), best, mean, unc, rec


def production_config(nx=16384, ny=2048, h=2.5e-6, width=5e-3, cfl=0.4):
    """The large production mesh: 16384 x 2048 cells of 2.5 um, R = 2 m,
    gamma = 2000, TSC.  At CFL 0.4 a bunch at c crosses 16000 cells in 40000
    steps, which fits the mesh; at CFL 0.5 it would reach the end wall after
    about 32000."""
    from .workloads import bend_config
    return bend_config(nx, ny, h, C5_R, width, C5_GAMMA, shape_order=1, cfl=cfl)


def production_run(case, n=32_000_000, steps=40_000, stations=32, cfg=None, log=print, checkpoint=None,
                   resume=None):
    """The production run for one profile: quiet-start bunch of n particles
    50 cells plus 6 sigma_s from the mesh start, FP32 mode, stepped as a
    one-member ensemble (the batched path, one CUDA graph per step).  Records
    the wake on the 256 bins every steps/stations steps; returns the wakes and
    the timing (device time of the stepping; the station reads excluded).
    checkpoint: a file rewritten at every station; resume: a checkpoint of the
    same run to continue from (its stations before the saved step are left
    out of the returned wakes)."""
    from scipy.special import ndtri
    from . import wakeset
    from .pic import Ensemble, Simulation
    cfg = cfg or production_config()
    sim = Simulation(cfg, fp32=True)
    first, rep, t_poisson = 0, {"solves": None}, 0.0
    if resume:  # the file holds fields, window and bunch: nothing to load or solve
        done, _ = sim.restore(resume)
        first = int(done) // (steps // stations)
        n = sim.n
        if log:
            log("production: resumed at step %d" % done)
    else:
        hx = sim.info()["hx"]
        g = np.random.Generator(np.random.Philox(case.seed))
        x = 50 * hx + 6 * case.sigma_s + wakeset.quiet_offsets(case, n)
        q = np.clip(np.mod(g.uniform() + wakeset.GOLDEN * np.arange(n), 1.0), 0.5 / n, 1 - 0.5 / n)
        y = 0.5 * cfg.width + case.sigma_s / 2.5 * ndtri(q)
        gam = case.gamma * (1.0 + 1e-4 * g.standard_normal(n))
        sim.load(x, y, np.sqrt(gam * gam - 1.0), np.zeros(n), np.full(n, wakeset.CHARGE / n))
        del x, y, gam, q
        t = time.perf_counter()
        rep = sim.initial_fields()
        t_poisson = time.perf_counter() - t
    ens = Ensemble([sim])
    reader = wakeset._WakeReader([sim], [case.sigma_s])
    every = steps // stations
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = torch.cuda.ExternalStream(ens.stream())
    W, dev_ms = [], 0.0
    t = time.perf_counter()
    for j in range(first, stations):
        a.record(st)
        ens.step(every)
        b.record(st)
        ens.sync()
        dev_ms += a.elapsed_time(b)
        w, _ = reader.read()
        W.append(w[0])
        if checkpoint:
            sim.checkpoint(checkpoint, step=(j + 1) * every, time=(j + 1) * every * sim.info()["dt"])
        if log and (j % 8 == 7 or j == stations - 1):
            log("production: %d steps, %.2f ms/step" % ((j + 1) * every, dev_ms / ((j + 1 - first) * every)))
    wall = time.perf_counter() - t
    mom = sim.moments()
    ens.close()
    sim.close()
    ran = every * (stations - first)
    return np.array(W).T, {"particles": n, "steps": ran, "first_step": first * every, "cells": cfg.Nx * cfg.Ny,
                           "ms_per_step": dev_ms / ran, "wall_s": wall,
                           "particle_steps_per_s": n * ran / (dev_ms / 1e3),
                           "poisson_s": t_poisson, "poisson": rep["solves"], "final_moments": mom[:8].tolist()}


def _summary(e):
    e = np.asarray(e, dtype=np.float64)
    e = e[np.isfinite(e)]
    return {"n": int(e.size), "mean": float(e.mean()), "median": float(np.median(e)),
            "p90": float(np.quantile(e, 0.9)), "max": float(e.max()), "frac_le_2pct": float(np.mean(e <= 0.02))}


def study(d, models=4, steps=40000, variants=100000, top=16, out=None, log=print):
    """The whole workflow on a data set: train `models` networks (seeds 0..),
    check each and their mean on the held-out cases against the
    alignment-averaged PIC (with the single PIC runs' own scatter beside it),
    time inference at 65536 profiles, prescreen `variants` production
    profiles, rerun the selected ones in PIC (alignment-averaged) and compare.
    Writes a JSON record to `out` after every stage."""
    from . import wakeset
    R = {}

    def dump():
        if out:
            with open(out, "w") as f:
                json.dump(R, f, indent=1)

    facts = d["facts"]
    R["data"] = {"cases": len(d["cases"]), "skipped": d.get("skipped", 0),
                 "pic_s_per_case_stepping": pic_seconds_per_case(d),
                 "pic_s_per_case_setup": sum(f["setup_s"] for f in facts) / sum(f["members"] for f in facts)}
    nets = []
    for k in range(models):
        m, rec = train(d, steps=steps, seed=k, log=None)
        rec.pop("losses")
        R["train%d" % k] = rec
        nets.append(m)
        dump()
    R["inference"] = time_inference(nets[0], d["X"][:64], n=65536, chunk=8192)
    tr, te = split(len(d["X"]))
    held = [d["cases"][k] for k in te]
    mean, mask, runs = pic_reference(held, log=None)
    R["eval"] = [evaluate(m, d, ref=(mean, mask), log=None)[0] for m in nets]
    R["eval_against_single_pic"] = evaluate(nets[0], d, log=None)[0]
    preds = [m.predict(d["X"][te]) for m in nets]
    P = np.mean(preds, axis=0)
    err = rel_errors(P, mean, mask)
    kinds = np.array([c.kind for c in held])
    R["ensemble_mean_eval"] = {"all": _summary(err), **{n: _summary(err[kinds == i]) for i, n in
                                                        enumerate(("gaussian", "flat_top", "double_horn"))}}
    # the spread calibrated on the held-out cases (the prescreen's uncertainty)
    spread = wake_spread(preds)
    calib = calibrate(err, spread, d["X"][tr])
    R["calibration"] = {"k": calib.k, "quantile": calib.q, "edge_quantile": calib.q_edge,
                        "spread": _summary(spread), "held_out_within_k_spread": float(np.mean(err <= calib.k * spread))}
    dump()
    t = time.perf_counter()
    var = c5_variants(variants)
    t_var = time.perf_counter() - t
    rerun, best, J, unc, rec = prescreen(nets, var, top=top, log=None, calib=calib)
    rec["variants_s"] = t_var
    R["prescreen"] = rec
    dump()
    sel = [var[k] for k in rerun]
    t = time.perf_counter()
    pm, pmask, _ = pic_reference(sel, log=None)
    t_pic = time.perf_counter() - t
    Xs = wakeset.features(sel)
    preds_s = [m.predict(Xs) for m in nets]
    Ps = np.mean(preds_s, axis=0)
    ran = np.all(np.isfinite(pm.reshape(len(sel), -1)), axis=1)     # the reference's geometry asserts for a few
    e_sel = np.full(len(sel), np.nan)
    e_sel[ran] = rel_errors(Ps[ran], pm[ran], pmask[ran])
    Jp, Js = np.full(len(sel), np.nan), objective(Xs, Ps)
    Jp[ran] = objective(Xs[ran], pm[ran])
    rank = lambda a: np.argsort(np.argsort(a))
    istop = np.arange(len(sel)) < len(best)
    b = int(np.argmin(np.where(ran, Jp, np.inf)))
    # how the calibrated wake uncertainty k * spread covers the reruns' actual errors
    u_sel = calib.k * wake_spread(preds_s)
    sel_edge = calib.edge(Xs)
    R["calibration"]["reruns_within_k_spread"] = float(np.mean(e_sel[ran] <= u_sel[ran])) if ran.any() else None
    R["calibration"]["reruns_calibrated_uncertainty"] = _summary(u_sel)
    R["calibration"]["reruns_at_training_edge"] = int(sel_edge.sum())
    R["reruns"] = {"count": len(sel), "ran": int(ran.sum()), "pic_seconds_4_shifts": t_pic,
                   "wake_err": _summary(e_sel), "wake_err_top": _summary(e_sel[istop]),
                   "wake_err_uncertain": _summary(e_sel[~istop]),
                   "objective_err": _summary(np.abs(Js - Jp) / Jp),
                   "objective_err_top": _summary((np.abs(Js - Jp) / Jp)[istop]),
                   "spearman_all": float(np.corrcoef(rank(Jp[ran]), rank(Js[ran]))[0, 1]),
                   "spearman_top": float(np.corrcoef(rank(Jp[ran & istop]), rank(Js[ran & istop]))[0, 1]),
                   "pic_best": {"variant": int(rerun[b]), "in_surrogate_top": bool(istop[b]),
                                "surrogate_rank_among_reruns": int(np.sum(Js[ran] < Js[b])),
                                "J_pic": float(Jp[b]), "J_surrogate": float(Js[b])}}
    dump()
    return R, nets


def pic_seconds_per_case(d):
    f = d["facts"]
    return sum(x["seconds"] for x in f) / sum(x["members"] for x in f)


if __name__ == "__main__":
    import argparse
    from . import wakeset
    ap = argparse.ArgumentParser(description="train / evaluate the wake surrogate")
    ap.add_argument("cmd", choices=["train", "evaluate", "time", "study", "production"])
    ap.add_argument("--variant", type=int, default=0, help="production variant index (production)")
    ap.add_argument("--particles", type=int, default=32_000_000, help="production bunch size (production)")
    ap.add_argument("--checkpoint", default=None, help="checkpoint file rewritten at every station (production)")
    ap.add_argument("--resume", default=None, help="checkpoint to continue from (production)")
    ap.add_argument("--models", type=int, default=4, help="networks in the ensemble (study)")
    ap.add_argument("--variants", type=int, default=100000, help="production variants to screen (study)")
    ap.add_argument("--json", default=None, help="where study writes its record")
    ap.add_argument("--n", type=int, default=65536, help="profiles per inference batch (time)")
    ap.add_argument("--data", default=None, help="data files, comma-separated")
    ap.add_argument("--model", default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    if a.cmd == "production":  # the 16384 x 2048 run of one screened variant (no data needed)
        v = c5_variants(a.variant + 1)[a.variant]
        W, rec = production_run(v, n=a.particles, steps=a.steps, checkpoint=a.checkpoint, resume=a.resume)
        rec["variant"], rec["variant_index"] = v.dict(), a.variant
        if a.json:
            with open(a.json, "w") as f:
                json.dump(rec, f, indent=1)
        if a.out:
            np.savez_compressed(a.out, W=W.astype(np.float32))
        print(json.dumps(rec))
        raise SystemExit(0)
    if a.cmd == "time":  # inference throughput with the weights as initialised (no data needed)
        cases = wakeset.draw_cases(64, seed=99)
        m = WakeModel(FNO(seed=a.seed), np.zeros(7), 1.0)
        print(json.dumps(time_inference(m, wakeset.features(cases), n=a.n, chunk=min(a.n, 8192))))
        raise SystemExit(0)
    d = wakeset.load(*a.data.split(","))
    if a.cmd == "study":
        R, nets = study(d, models=a.models, steps=a.steps, variants=a.variants, out=a.json)
        if a.out:
            nets[0].save(a.out)
        print(json.dumps(R))
        raise SystemExit(0)
    if a.cmd == "train":
        m, rec = train(d, steps=a.steps, batch=a.batch, lr0=a.lr, seed=a.seed)
        print(json.dumps(rec))
        if a.out:
            m.save(a.out)
        evaluate(m, d)
    else:
        evaluate(WakeModel.load(a.model), d)
