"""Wake data set of the surrogate: seeded line-charge profiles with bend
parameters, each run through the batched FP32 PIC (TSC, CFL 0.5, Poisson
initial fields), with the longitudinal wake on the bunch axis recorded at 32
stations along the bend.

A case is a profile family (Gaussian, flat-top, double-horn) with its shape
parameters, an rms length sigma_s log-uniform in [20, 200] um, gamma ~ U[200,
2000], bend radius R ~ U[0.5, 5] m and a pipe width of 64 - 96 sigma_s.  Cells
are sigma_s / 8; the mesh holds a straight section just long enough for the
bunch and its window and a bend long enough for the bunch to travel 1024 cells
(128 sigma_s) in it.  The bunch is a two-dimensional quiet start (profile
quantiles in s paired with a rank-1 lattice of Gaussian quantiles in y, rms
sigma_s / 2.5), with a drawn gamma spread of 1e-4 rms.  The bunch centroid reaches the bend entrance after
ENTRY_STEPS steps; station j is STATION_STEPS (j + 1) steps later.

Inputs of a case (per bin of the 256 bins spanning +-SPAN sigma_s around the
centroid): line density per sigma_s, bin position, and the four scalars;
outputs: E_s [V/m] on the same bins at the 32 stations (the IntegrateElong
diagnostic sampled on window columns, interpolated linearly onto the bins).
"""
import json
import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, asdict

import numpy as np
from scipy.special import erf

from .workloads import C_LIGHT, MASS_EV, RunConfig

NBINS, NSTATIONS = 256, 32
SPAN = 4.0                 # bins cover +-SPAN sigma_s
CELLS_PER_SIGMA = 8
STATION_STEPS = 64         # steps between stations (32 cells of travel at CFL 0.5)
CHARGE = -1e-9


@dataclass
class WakeCase:
    kind: int              # 0 Gaussian, 1 flat-top, 2 double-horn
    edge: float            # flat-top edge width (units of the half length)
    tilt: float            # linear tilt of the flat top
    horn_pos: float        # horn centres at +-horn_pos
    horn_w: float          # horn rms width
    horn_a: float          # horn peak heights relative to the flat top
    horn_b: float
    sigma_s: float         # rms bunch length [m]
    gamma: float
    R: float               # bend radius [m]
    width_sigma: float     # pipe width / sigma_s (target; the mesh rounds it)
    seed: int

    def dict(self):
        return asdict(self)


def draw_cases(n, seed=7):
    """n seeded cases; the families alternate.  Pipes are wide (64 - 96
    sigma_s): at 12 - 40 sigma_s the wake over this travel depends steeply on
    the bend radius through the curved walls' cut cells (a 1 % change of R
    moves it by 5 - 25 %), at 80 sigma_s by 0.05 - 1.5 %."""
    g = np.random.Generator(np.random.Philox(seed))
    out = []
    for k in range(n):
        kind = k % 3
        out.append(WakeCase(kind=kind, edge=float(g.uniform(0.05, 0.3)), tilt=float(g.uniform(-0.3, 0.3)),
                            horn_pos=float(g.uniform(0.7, 0.95)), horn_w=float(g.uniform(0.04, 0.12)),
                            horn_a=float(g.uniform(0.5, 2.5)), horn_b=float(g.uniform(0.5, 2.5)),
                            sigma_s=float(np.exp(g.uniform(np.log(20e-6), np.log(200e-6)))),
                            gamma=float(g.uniform(200.0, 2000.0)), R=float(g.uniform(0.5, 5.0)),
                            width_sigma=float(g.uniform(64.0, 96.0)), seed=int(g.integers(1, 2 ** 31))))
    return out


def shape(case, z):
    """Unnormalised density of the profile family at z (units of the
    family's own length scale)."""
    if case.kind == 0:
        return np.exp(-0.5 * z * z)
    e = case.edge * math.sqrt(2.0)
    ft = 0.5 * (erf((z + 1.0) / e) - erf((z - 1.0) / e)) * (1.0 + case.tilt * z)
    if case.kind == 1:
        return np.maximum(ft, 0.0)
    hw = 2.0 * case.horn_w ** 2
    horns = case.horn_a * np.exp(-(z + case.horn_pos) ** 2 / hw) + case.horn_b * np.exp(-(z - case.horn_pos) ** 2 / hw)
    return np.maximum(ft, 0.0) + horns


def profile(case, fine=8192):
    """(z grid, density, centroid, rms) of the family on a fine grid."""
    z = np.linspace(-6.0, 6.0, fine)
    d = shape(case, z)
    d /= np.trapezoid(d, z)
    mu = np.trapezoid(z * d, z)
    rms = math.sqrt(np.trapezoid((z - mu) ** 2 * d, z))
    return z, d, mu, rms


def line_density(case):
    """Input profile: density per sigma_s at the 256 bin centres, which span
    +-SPAN sigma_s around the centroid (integrates to ~1 over the bins)."""
    z, d, mu, rms = profile(case)
    s = bin_centres()                        # units of sigma_s
    return np.interp(mu + s * rms, z, d, left=0.0, right=0.0) * rms


def bin_centres():
    return (np.arange(NBINS) + 0.5) / NBINS * 2 * SPAN - SPAN


def quiet_offsets(case, n):
    """Longitudinal offsets [m] from the centroid: particle k at the
    (k + 1/2) / n quantile of the profile."""
    z, d, mu, rms = profile(case)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (d[1:] + d[:-1]) * np.diff(z))])
    cdf /= cdf[-1]
    u = np.interp((np.arange(n) + 0.5) / n, cdf, z)
    return (u - mu) / rms * case.sigma_s


def case_config(case):
    """RunConfig for a case: square cells sigma_s / 8; the bend angle gives an
    arc for 1024 cells of travel plus the bunch; the pipe fills the mesh height
    (the reference's domain rule, Bend.cpp:92-105); the drift before the bend
    holds the bunch 6 sigma_s before the entrance and its window."""
    h = case.sigma_s / CELLS_PER_SIGMA
    R = case.R
    la = 50 * h
    travel = NSTATIONS * STATION_STEPS * 0.5 * h
    phi = (travel + 8 * case.sigma_s + 40 * h) / R
    c, sn = math.cos(phi), math.sin(phi)
    w0 = case.width_sigma * case.sigma_s
    height = (R - 0.5 * w0) * (1 - c) + w0 + la * sn
    Ny = int(math.ceil(height / h)) + 2
    dom_w = (Ny - 2) * h
    width = (dom_w - R * (1 - c) - la * sn) / (1 - 0.5 * (1 - c))   # fills the mesh height exactly
    lb_min = 12 * case.sigma_s + 40 * h
    Nx = int(math.ceil((lb_min + (R + 0.5 * width) * sn + la * c) / h)) + 2
    lb = (Nx - 2) * h - la * c - (R + 0.5 * width) * sn
    ekin_mev = (case.gamma - 1.0) * MASS_EV * 1e-6
    ekin = ekin_mev * 1e6
    bz = math.sqrt(ekin * ekin + 2.0 * ekin * MASS_EV) / (C_LIGHT * R)
    cfg = RunConfig(Nx=Nx, Ny=Ny, length_before=lb, length_after=la, width=width, phi_deg=math.degrees(phi),
                    ekin_mev=ekin_mev, bz=bz, shape_order=1, dt=0.5 * h / C_LIGHT)
    return cfg, lb


GOLDEN = 0.6180339887498949


def case_bunch(case, cfg, lb, n, shift=0.0):
    """Two-dimensional quiet start: particle k sits at the (k + 1/2)/n
    quantile of the profile in s and at the quantile frac(u0 + k * 0.618...)
    of the transverse Gaussian (a rank-1 lattice; u0 drawn from the case
    seed, so that seeds give independent realisations); gamma spread drawn.
    shift moves the bunch by that fraction of a cell in s."""
    from scipy.special import ndtri
    g = np.random.Generator(np.random.Philox(case.seed))
    u0 = g.uniform()
    x = lb - 6 * case.sigma_s + shift * case.sigma_s / CELLS_PER_SIGMA + quiet_offsets(case, n)
    q = np.mod(u0 + GOLDEN * np.arange(n), 1.0)
    q = np.clip(q, 0.5 / n, 1.0 - 0.5 / n)
    y = 0.5 * cfg.width + case.sigma_s / 2.5 * ndtri(q)
    gam = case.gamma * (1.0 + 1e-4 * g.standard_normal(n))
    px = np.sqrt(gam * gam - 1.0)
    return x, y, px, np.zeros(n), np.full(n, CHARGE / n)


ENTRY_STEPS = 6 * CELLS_PER_SIGMA * 2      # 6 sigma_s at half a cell per step


def station_steps():
    return [ENTRY_STEPS + STATION_STEPS * (j + 1) for j in range(NSTATIONS)]


NFEATURES = 7


def _params(cases):
    """Shape parameters of many cases as arrays [N, 1]."""
    f = lambda name: np.array([getattr(c, name) for c in cases], dtype=np.float64)[:, None]
    return {k: f(k) for k in ("kind", "edge", "tilt", "horn_pos", "horn_w", "horn_a", "horn_b")}


def shape_batch(P, z, kind):
    """shape() for many cases of one family at once: P from _params, z [N, m]."""
    if kind == 0:
        return np.exp(-0.5 * z * z)
    e = P["edge"] * math.sqrt(2.0)
    ft = np.maximum(0.5 * (erf((z + 1.0) / e) - erf((z - 1.0) / e)) * (1.0 + P["tilt"] * z), 0.0)
    if kind == 1:
        return ft
    hw = 2.0 * P["horn_w"] ** 2
    return ft + P["horn_a"] * np.exp(-(z + P["horn_pos"]) ** 2 / hw) + P["horn_b"] * np.exp(-(z - P["horn_pos"]) ** 2 / hw)


_POOL = None


def _pool():
    """Host threads for the per-chunk feature work (numpy's and scipy's
    element-wise kernels release the GIL); each chunk is computed exactly as
    it would be alone, so the results do not depend on the thread count."""
    global _POOL
    if _POOL is None:
        _POOL = ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)))
    return _POOL


def moments_batch(cases, fine=512):
    """(mass, centroid, rms) of the families' shapes, vectorised per family
    (a Gaussian analytically; the flat-top families, whose support lies
    within +-3 of their scale, by the trapezoid rule on a fine grid), chunks
    of 4096 cases on the host threads."""
    z = np.linspace(-3.0, 3.0, fine)
    dz = z[1] - z[0]
    wq = np.full(fine, dz)
    wq[0] = wq[-1] = 0.5 * dz
    kinds = np.array([c.kind for c in cases])
    mass, mu, rms = np.full(len(cases), math.sqrt(2 * math.pi)), np.zeros(len(cases)), np.ones(len(cases))

    def one(kind, sel, P):
        d = shape_batch(P, z[None, :], kind)
        mass[sel] = d @ wq
        mu[sel] = (d * z) @ wq / mass[sel]
        rms[sel] = np.sqrt((d * (z[None, :] - mu[sel, None]) ** 2) @ wq / mass[sel])

    jobs = []
    for kind in (1, 2):
        idx = np.nonzero(kinds == kind)[0]
        for a in range(0, len(idx), 4096):
            sel = idx[a:a + 4096]
            jobs.append(_pool().submit(one, kind, sel, _params([cases[k] for k in sel])))
    for j in jobs:
        j.result()
    return mass, mu, rms


def features(cases, chunk=1024):
    """[N][256][7] float32: line density per sigma_s, bin position / SPAN,
    log-scaled gamma, R, sigma_s, pipe width / sigma_s (each about [-1, 1]
    over the drawn ranges), and the slope of the line density (per sigma_s^2,
    / 4).  Vectorised per family over chunks of cases: a Gaussian is centred
    with unit rms; the flat-top families (support within +-3 of their scale)
    take centroid and rms from a fine grid; the density at the bins comes
    from the shape itself.  Chunks of cases run on the host threads (the
    values do not depend on the chunking: every step is per case)."""
    N = len(cases)
    out = np.zeros((N, NBINS, NFEATURES), dtype=np.float32)
    sb = bin_centres()
    mass_all, mu_all, rms_all = moments_batch(cases)
    kinds = np.array([c.kind for c in cases])

    def one(kind, sel, P):
        mass, mu, rms = mass_all[sel], mu_all[sel], rms_all[sel]
        lam = shape_batch(P, mu[:, None] + sb[None, :] * rms[:, None], kind) / mass[:, None] * rms[:, None]
        out[sel, :, 0] = lam
        out[sel, :, 6] = np.gradient(lam, 2 * SPAN / NBINS, axis=1) / 4.0

    jobs = []
    for kind in (0, 1, 2):
        idx = np.nonzero(kinds == kind)[0]
        for a in range(0, len(idx), chunk):
            sel = idx[a:a + chunk]
            jobs.append(_pool().submit(one, kind, sel, _params([cases[k] for k in sel])))
    for j in jobs:
        j.result()
    out[:, :, 1] = sb[None, :] / SPAN
    for j, (name, ref) in enumerate((("gamma", 632.5), ("R", 1.581), ("sigma_s", 63.25e-6))):
        out[:, :, 2 + j] = ((np.log([getattr(c, name) for c in cases]) - math.log(ref)) / 1.152)[:, None]
    out[:, :, 5] = ((np.array([case_config(c)[0].width / c.sigma_s for c in cases]) - 80.0) / 16.0)[:, None]
    return out


def sample_wake(sim, sigma_s):
    """E_s of a member on the 256 bins (NaN-free: bins outside the sampled
    columns take the nearest sample) and the mask of sampled bins."""
    w, org, _ = sim.window()
    e = sim.wake()
    mom = sim.moments()
    s = org[0] + np.arange(2, w[2] - 2) * sim.info()["hx"] - mom[0]
    ok = np.isfinite(e)
    s, e = s[ok], e[ok]
    sb = bin_centres() * sigma_s
    out = np.interp(sb, s, e)
    return out, (sb >= s[0]) & (sb <= s[-1])


class _WakeReader:
    """Reads the wake of many members with one wait: every member's
    diagnostic is enqueued on its own stream into one device buffer, then the
    buffer comes back in one copy and is interpolated onto the bins."""

    def __init__(self, sims, sigmas):
        import torch
        from ._lib import lib
        self.sims, self.lib = sims, lib()
        self.n = [s.window()[0][2] - 4 for s in sims]
        self.hx = np.array([s.info()["hx"] for s in sims])
        self.sb = np.outer(np.asarray(sigmas), bin_centres())
        self.ld = max(self.n)
        self.buf = torch.empty(len(sims), self.ld, dtype=torch.float64, device="cuda")
        self.meta = torch.empty(len(sims), 4, dtype=torch.float64, device="cuda")

    def read(self):
        import ctypes as C
        import torch
        from ._lib import check
        for k, s in enumerate(self.sims):
            check(self.lib.csrst_diag_wake_async(s.h, C.c_void_p(self.buf[k].data_ptr()), self.n[k],
                                                 C.c_void_p(self.meta[k].data_ptr())), s.h)
        torch.cuda.synchronize()
        buf, meta = self.buf.cpu().numpy(), self.meta.cpu().numpy()
        out = np.zeros(self.sb.shape)
        ok = np.zeros(self.sb.shape, dtype=bool)
        for k in range(len(self.sims)):
            e = buf[k, :self.n[k]]
            s = meta[k, 0] + np.arange(2, self.n[k] + 2) * self.hx[k] - meta[k, 2]
            f = np.isfinite(e)
            s, e = s[f], e[f]
            out[k] = np.interp(self.sb[k], s, e)
            ok[k] = (self.sb[k] >= s[0]) & (self.sb[k] <= s[-1])
        return out, ok


def run_cases(cases, n_particles=50_000, batch=256, fp32=True, log=None, shift=0.0):
    """Runs every case in batches of `batch` members (one Ensemble each) and
    returns wakes [N][256][32] (float32, V/m), the mask of bins inside the
    sampled window columns (same shape) and per-batch run facts (the stepping
    time includes the station reads)."""
    import time
    from ._lib import CsrstError
    from .pic import Ensemble, Simulation
    N = len(cases)
    wakes = np.zeros((N, NBINS, NSTATIONS), dtype=np.float32)
    mask = np.zeros((N, NBINS, NSTATIONS), dtype=bool)
    facts = []
    st = station_steps()
    for a in range(0, N, batch):
        group = cases[a:a + batch]
        t = time.perf_counter()
        sims, keep = [], []
        for k, c in enumerate(group):
            cfg, lb = case_config(c)
            try:
                s = Simulation(cfg, fp32=fp32)
            except CsrstError as e:  # the reference's geometry asserts for this bend: no PIC wake for the case
                if log:
                    log("case %d skipped: %s" % (a + k, e))
                wakes[a + k] = np.nan
                continue
            s.load(*case_bunch(c, cfg, lb, n_particles, shift))
            s.initial_fields()
            sims.append(s)
            keep.append(k)
        group = [group[k] for k in keep]
        ens = Ensemble(sims)
        ens.sync()
        setup = time.perf_counter() - t
        done, outside = 0, 0
        reader = _WakeReader(sims, [c.sigma_s for c in group])
        t = time.perf_counter()
        for j, target in enumerate(st):
            ens.step(target - done)
            done = target
            ens.sync()
            wk, ok = reader.read()
            wakes[a + np.array(keep), :, j] = wk
            mask[a + np.array(keep), :, j] = ok
            outside += int(np.sum(~ok))
        elapsed = time.perf_counter() - t
        facts.append({"members": len(group), "steps": done, "seconds": elapsed, "setup_s": setup,
                      "bins_outside": outside, "particles": n_particles * len(group),
                      "cells": int(sum(s.Nx * s.Ny for s in sims))})
        if log:
            log("cases %d-%d: set-up %.1f s, %d steps in %.2f s, %d bins outside the window"
                % (a, a + len(group), setup, done, elapsed, outside))
        ens.close()
        for s in sims:
            s.close()
    return wakes, mask, facts


def generate(n, seed=7, n_particles=50_000, batch=256, start=0, count=None, log=print):
    """The data set (cases start .. start + count of the seeded draw of n):
    cases, input features, PIC wakes and masks."""
    cases = draw_cases(n, seed)[start:start + (n if count is None else count)]
    X = features(cases)
    W, M, facts = run_cases(cases, n_particles=n_particles, batch=batch, log=log)
    return dict(cases=cases, X=X, W=W, M=M, facts=facts)


def save(path, d):
    """Compact file: each case's wake in FP16 relative to its own peak (an
    FP32 scale per case; 5e-4 of the peak, far below the PIC's shot noise and
    the surrogate's error), masks bit-packed; the input features are
    recomputed from the cases on load.  Skipped cases are NaN."""
    W = d["W"]
    peak = np.array([np.nanmax(np.abs(w)) if np.any(np.isfinite(w)) else np.nan for w in W], dtype=np.float32)
    rel = W / np.where(peak > 0, peak, 1.0)[:, None, None]
    np.savez_compressed(path, W=rel.astype(np.float16), peak=peak, M=np.packbits(d["M"].reshape(-1)),
                        shape=np.array(W.shape),
                        cases=np.array([[getattr(c, f) for f in WakeCase.__dataclass_fields__] for c in d["cases"]]),
                        facts=np.array(json.dumps(d["facts"])))


def load(*paths):
    """One data set from one or more files (concatenated in order)."""
    names = list(WakeCase.__dataclass_fields__)
    cases, W, M, facts = [], [], [], []
    for path in paths:
        z = np.load(path)
        shape = tuple(int(v) for v in z["shape"])
        cases += [WakeCase(**{f: (int(v) if f in ("kind", "seed") else float(v)) for f, v in zip(names, row)})
                  for row in z["cases"]]
        W.append(z["W"].astype(np.float32) * z["peak"][:, None, None])
        M.append(np.unpackbits(z["M"])[:int(np.prod(shape))].reshape(shape).astype(bool))
        facts += json.loads(str(z["facts"]))
    W, M = np.concatenate(W), np.concatenate(M)
    ok = np.all(np.isfinite(W.reshape(len(W), -1)), axis=1)   # cases the PIC ran
    cases = [c for c, k in zip(cases, ok) if k]
    return dict(cases=cases, X=features(cases), W=W[ok], M=M[ok], facts=facts, skipped=int((~ok).sum()))


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="generate the surrogate's wake data set with the batched PIC")
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--particles", type=int, default=50_000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--start", type=int, default=0)
    ap.add_argument("--count", type=int, default=None)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    save(a.out, generate(a.n, a.seed, a.particles, a.batch, a.start, a.count))
