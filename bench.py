#!/usr/bin/env python
"""Throughput of the CSRST per-time-step PIC loop on B200.

A step is one full time step of the reference's main loop (main.cpp:390-506):
TETMSolver::updateField_firstStep, updateField_secondStep and moveMesh, i.e.
two relativistic pushes with gather and charge-conserving deposit, four
TE/TM field sub-steps on the static mesh, the cut cells and the moving
window, their strip exchanges and the window move.

Default workload: 8192 x 1024 static mesh at 5 um, 4e6 macro-particles,
TSC (IntS1 gather + first-order deposit), CFL 0.5, in FP32 mode (FP32
fields, gather and kick on FP32 offsets from FP64 cell origins, FP64
deposit), with the plain FP64 GPU path timed beside it and the FP32 result
checked against it (CSR wake, energy change per slice, continuity).
Synthetic seeded bunch (Gaussian, sigma_s 50 um, sigma_x 20 um, energy
spread 1e-4, 1 nC); initial fields from the GPU multigrid Poisson solve.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank runs an independent replica (the loop does not
shard; the ensemble members are independent units): value = all ranks'
particle-steps / max-over-ranks time.
"""
import argparse
import json
import math
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s, Yee cell-updates/s; FP32 vs FP64 GPU at ≤1e-3 CSR-wake err"
UNIT = "particle-steps/s"
# algorithmic bytes per unit: the fused Yee update reads and writes Ex, Ey,
# Hzx, Hzy and reads a 1-byte mask per cell-step; a push streams position and
# momentum in and out per particle (FP32 mode: 4-byte cell + two FP32 offsets
# + two FP32 momentum deviations).
YEE_BYTES = {"fp64": 65, "fp32": 33}
PUSH_BYTES = {"fp64": 64, "fp32": 40}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="c2")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"],
                   help="mode of the headline value; the other mode is timed beside it")
    p.add_argument("--no-compare", action="store_true", help="skip the other precision and the accuracy check")
    p.add_argument("--no-ensemble", action="store_true", help="skip the 64-member batched-ensemble workload")
    p.add_argument("--no-surrogate", action="store_true", help="skip the wake-surrogate measurements")
    p.add_argument("--ensemble-only", default=None, choices=["c3", "small"],
                   help="time only the batched FP32 ensemble (c3: 64 uneven members; small: 256 512x104 members)")
    p.add_argument("--shape", default=None, help="push_ctas,tx,ty,parts for --ensemble-only instead of the autotuner")
    return p.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value, world, device="cuda"):
    """The largest of every rank's value (each rank calls this with its own
    measurement): a multi-GPU time is the slowest replica's."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def peaks(bf16=False):
    """HBM GB/s (and, with bf16=True, (hbm, dense BF16 TFLOP/s burst, source))
    from MEASURED_PEAKS.json, else the pool's fallback figures."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        if bf16:
            return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured bf16_tflops"
        return float(d["hbm_gbs"]), "measured"
    if bf16:
        return 6650.0, 1590.0, "fallback bf16 (no MEASURED_PEAKS.json)"
    return 6650.0, "fallback"


# The launches of one time step per kernel group (order 1 = TSC), as the
# profile launch lists name them.
STEP_LAUNCHES = {
    ("push", "fp32", 1): {"k_push32<1, 0>": 1, "k_push32<1, 1>": 1, "k_prep32": 1, "k_after32": 2},
    ("yee", "fp32", 1): {"k_yee_tiles<float>": 1, "k_yee_fixup<float>": 1, "k_window_ey<float>": 1},
    ("push", "fp64", 1): {"k_push<1>": 2, "k_push_prep": 2, "k_push_post": 2, "k_global_bounds": 2},
    ("yee", "fp64", 1): {"k_yee_tiles<double>": 1, "k_yee_fixup<double>": 1, "k_window_ey<double>": 1},
}
LAUNCH_LISTS = {"fp32": "profiles/c2_tsc_fp32_step_launches.txt", "fp64": "profiles/c2_tsc_fp64_step_launches.txt"}


def profile_traffic(group, prec, order):
    """Per-step DRAM bytes (read + write) of a kernel group from the committed
    ncu launch list of the c2 workload (LAUNCH_LISTS: one row per kernel with
    its DRAM MB per launch), summed over the step's launches of that group.
    None when the list is missing or does not name every kernel the step
    launches (e.g. after a kernel was replaced), so the figure never outlives
    the kernels it was measured on.  Returns (bytes, source file)."""
    want = STEP_LAUNCHES.get((group, prec, order))
    f = ROOT / LAUNCH_LISTS[prec]
    if not want or not f.exists():
        return None, None
    rows = {}
    for line in f.read_text().splitlines():
        if line.startswith("#") or "|" not in line:
            continue
        c = [v.strip() for v in line.split("|")]
        rows[c[0]] = (float(c[5]) + float(c[6])) * 1e6
    if any(k not in rows for k in want):
        return None, None
    return sum(n * rows[k] for k, n in want.items()), LAUNCH_LISTS[prec]


class Clocks:
    """nvidia-smi sampler over the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def soak(self, sim, seconds=0.8):
        """Keeps the GPU on this workload until the sampler has produced
        samples under load (the timed region alone is often shorter than the
        sampling period).  Untimed steps, like the warm-up."""
        t = time.perf_counter()
        while time.perf_counter() - t < seconds:
            sim.step(20)
            sim.sync()

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def time_mode(args, cfg, bunch, world, fp32, clocks):
    """One precision mode: initial fields, warm-up, the timed graph-captured
    steps (max over ranks) and a per-group kernel attribution pass."""
    import torch
    from csrst_b200 import Simulation
    sim = Simulation(cfg, fp32=fp32)
    sim.load(*bunch)
    # initial fields of the bunch (PoissonSolver::computeField): one-time set-up, timed on its own
    t_if = time.perf_counter()
    rep = sim.initial_fields(1e-12, 1e-6, 500)
    t_if = time.perf_counter() - t_if
    stream = torch.cuda.ExternalStream(sim.stream())
    sim.step(args.warmup)
    sim.sync()
    if clocks:
        clocks.soak(sim)
    # ---- timed region: graph-captured steps, inputs resident in HBM ----
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    sim.step(args.steps)
    t1.record(stream)
    sim.sync()
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1), world)
    if world > 1:
        torch.distributed.barrier()
    # ---- kernel attribution: the same steps' kernels, eagerly, with CUDA
    # events between the groups on the library's stream (csrst_step_timed) ----
    groups = {"push": 0.0, "yee": 0.0, "move": 0.0}
    ksteps = min(args.steps, 10)
    for _ in range(ksteps):
        t = sim.step_timed()
        groups["push"] += t["push"]
        groups["yee"] += t["fields"]
        groups["move"] += t["move"]
    for k in groups:
        groups[k] /= ksteps
    window = sim.window()[0][2:]
    hx = sim.info()["hx"]
    sim.close()
    return {"ms": ms, "groups": groups, "window": window, "hx": hx,
            "initial_fields": {"ms": round(1e3 * t_if, 2), "levels": rep["levels"],
                               "iterations": [it for it, _ in rep["solves"]],
                               "relres": [float("%.3g" % rr) for _, rr in rep["solves"]]}}


def slice_energy_change(cfg, spec, bunch, steps):
    """Energy change per longitudinal slice (16 slices over +-3 sigma along
    the bunch axis) after `steps` steps, FP64 path and FP32 mode."""
    from csrst_b200 import Simulation
    out = {}
    for fp32 in (False, True):
        s = Simulation(cfg, fp32=fp32)
        s.load(*bunch)
        _, _, px, py = s.particles()
        g0 = np.sqrt(1 + px * px + py * py)
        s.step(steps)
        x, y, px, py = s.particles()
        out[fp32] = (np.sqrt(1 + px * px + py * py) - g0, x, y, s.moments())
        s.close()
    dg64, x, y, m = out[False]
    c, sn = m[2] / math.hypot(m[2], m[3]), m[3] / math.hypot(m[2], m[3])
    sl = (x - m[0]) * c + (y - m[1]) * sn
    idx = np.clip(np.digitize(sl, np.linspace(-3 * spec.sigma_s, 3 * spec.sigma_s, 17)) - 1, 0, 15)
    cnt = np.maximum(np.bincount(idx, minlength=16), 1)
    e64 = 0.511 * np.bincount(idx, dg64, minlength=16) / cnt
    e32 = 0.511 * np.bincount(idx, out[True][0], minlength=16) / cnt
    return e64, e32


def continuity32(sim, sf):
    """Continuity of one FP32-mode push (a keep_old handle): the current of
    its moves from the stand-alone FP32 deposit (csrst_flux32; the push's own
    window current equals it bit for bit, tests/test_gpu_fp32.py), both
    components, against (a) the integer charge it assigns, exactly, and (b)
    the FP64 charge shape (PartBunch's getChargeDensityDiff) in FP64.
    Returns (max |integer residual|, FP64 residual relative to max |rho/dt|)."""
    info = sim.info()
    h, dt, scale = (info["hx"], info["hy"]), info["dt"], info["fixed_scale"]
    sim.push(0)
    c1, b0, b1, _, _, q = sim.bunch32(0)
    c0, a0, a1 = sim.bunch32(1)
    w, org, _ = sim.window()
    P0, P1, L0, L1 = w
    fx, drho = sf.flux32(0, c0, a0, a1, c1, b0, b1, q, scale, P0, P1, L0, L1, with_charge=True)
    fy = sf.flux32(1, c0, a0, a1, c1, b0, b1, q, scale, P0, P1, L0, L1)
    exact = int(np.abs(drho[1:, 1:] + (fx[1:, 1:] - fx[1:, :-1]) + (fy[1:, 1:] - fy[:-1, 1:])).max())
    unpack = lambda c: ((c & 0xFFFF).astype(np.int64), (c.astype(np.uint32) >> 16).astype(np.int64))
    ci, cj = unpack(c0)
    ni, nj = unpack(c1)
    ox, oy = info["ox"] + (ci + a0.astype(np.float64)) * h[0], info["oy"] + (cj + a1.astype(np.float64)) * h[1]
    x, y = info["ox"] + (ni + b0.astype(np.float64)) * h[0], info["oy"] + (nj + b1.astype(np.float64)) * h[1]
    q64 = q.astype(np.float64)
    qs = 2.0 ** np.floor(np.log2(2.0 ** 62 / (4 * np.abs(q64).sum())))
    rho = sf.getChargeDensityDiff(ox, oy, x, y, q64, org, h, 0, 0, L0, L1, qs)
    jx, jy = fx / (scale * dt * h[1]), fy / (scale * dt * h[0])
    r = rho[1:, 1:] / dt + (jx[1:, 1:] - jx[1:, :-1]) / h[0] + (jy[1:, 1:] - jy[:-1, 1:]) / h[1]
    return exact, float(np.abs(r).max() / np.abs(rho / dt).max())


def accuracy(cfg, spec, bunch, steps=50):
    """FP32 mode against the FP64 path on identical inputs: the longitudinal
    wake on the bunch axis, the energy change per slice, and the continuity
    residual of one FP32-mode push.  The energy change per slice is taken
    where it is physical: a bunch entering the dipole (the small bend
    workload, 300 steps); over the workload's own 50 steps in the straight
    section it is ~1e-8 MeV and numerically noise."""
    from csrst_b200 import ShapeFunction, Simulation
    res, sims = {}, {}
    for fp32 in (False, True):
        s = Simulation(cfg, fp32=fp32, keep_old=fp32)
        s.load(*bunch)
        s.initial_fields(1e-12, 1e-6, 500)
        s.step(steps)
        res[fp32] = {"wake": s.wake()}
        sims[fp32] = s
    a, b = res[True], res[False]
    ok = np.isfinite(a["wake"]) & np.isfinite(b["wake"])
    wake_err = float(np.abs(a["wake"][ok] - b["wake"][ok]).max() / np.abs(b["wake"][ok]).max())
    # energy change per slice in the dipole (small bend workload, 300 steps)
    from csrst_b200.workloads import make_bunch, workload
    bcfg, bspec = workload("small-1-bend")
    de64, de32 = slice_energy_change(bcfg, bspec, make_bunch(bspec), 300)
    slice_err = float(np.abs(de32 - de64).max() / np.abs(de64).max())
    exact, cont = continuity32(sims[True], ShapeFunction(cfg.shape_order))
    # through the dipole: the c1 geometry from the dipole entrance, 2000 steps
    from csrst_b200.compare import fp32_vs_fp64
    dip = fp32_vs_fp64("c1-bend", 2000, every=100)
    for v in sims.values():
        v.close()
    return {"steps": steps, "wake_rel_err": float("%.3g" % wake_err),
            "energy_change_per_slice": {"case": "512x104 mesh at 20 um, R = 0.25 m, 4000 particles, TSC, "
                                                "bunch entering the dipole, 300 steps, 16 slices",
                                        "rel_err": float("%.3g" % slice_err),
                                        "fp64_mev": [float("%.4g" % v) for v in de64]},
            "continuity_residual_rel": float("%.3g" % cont),
            "continuity_integer_residual": exact,
            "through_dipole": {"case": "c1 geometry (2048x512, 10 um, R = 1 m, 2e5 particles, CIC), bunch from the "
                                       "dipole entrance, 2000 steps, wake sampled every 100 steps",
                               "wake_rel_err": float("%.3g" % dip["wake_rel_err"]),
                               "integrated_wake_rel_err": float("%.3g" % dip["integrated_rel_err"]),
                               "energy_change_per_slice_rel_err": float("%.3g" % dip["slice_rel_err"]),
                               "fp64_slice_mev": [float("%.4g" % v) for v in dip["slice_mev_fp64"]]},
            "bar": "wake <= 1e-3 of the FP64 path's maximum; continuity <= 1e-10 (FP64 check against the FP64 "
                   "charge shape); the integer residual against the charge the deposit assigns is exactly 0"}


def run_ensemble(args, rank, members=64, ms=None, fields=True):
    """The batched-ensemble workload: `members` independent bunches (uneven
    meshes 1024-8192 x 256-1024, 5e4-1e6 particles, CIC/TSC) stepped as one
    batch in FP32 mode after the autotuner picked the launch shapes, against
    the same members run one after another on the plain FP64 path (each
    member its own handle, stream and CUDA graph) and on FP32 unbatched."""
    import torch
    from csrst_b200 import Ensemble, Simulation
    from csrst_b200.workloads import ensemble_members, make_bunch
    if ms is None:
        ms = ensemble_members(members, seed=2024 + rank)
    members = len(ms)
    total = sum(spec.n for _, spec in ms)
    cells = sum(cfg.Nx * cfg.Ny for cfg, _ in ms)
    K, W = max(args.steps // 2, 5), max(args.warmup, 3)
    out = {"members": members, "particles": total, "cells": cells, "steps": K, "warmup": W}

    def build(fp32):
        sims = []
        t = time.perf_counter()
        for cfg, spec in ms:
            sm = Simulation(cfg, fp32=fp32)
            sm.load(*make_bunch(spec))
            if fields:
                sm.initial_fields(1e-12, 1e-6, 500)
            sims.append(sm)
        return sims, time.perf_counter() - t

    def time_streams(sims):
        # members one after another, each on its own stream, device-timed fork/join
        side = torch.cuda.Stream()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for sm in sims:
            sm.step(W)
            sm.sync()
        torch.cuda.synchronize()
        start.record(side)
        ends = []
        for sm in sims:
            st = torch.cuda.ExternalStream(sm.stream())
            st.wait_event(start)
            sm.step(K)
            e = torch.cuda.Event()
            e.record(st)
            ends.append(e)
        for e in ends:
            side.wait_event(e)
        stop.record(side)
        torch.cuda.synchronize()
        return start.elapsed_time(stop)

    # plain FP64 path, unbatched
    sims, setup = build(False)
    ms64 = time_streams(sims)
    for sm in sims:
        sm.close()
    out["fp64_unbatched"] = {"value": round(total * K / (ms64 * 1e-3), 1), "ms_per_step": round(ms64 / K, 3),
                             "setup_s": round(setup, 1)}
    # FP32 mode, unbatched
    sims, _ = build(True)
    ms32 = time_streams(sims)
    out["fp32_unbatched"] = {"value": round(total * K / (ms32 * 1e-3), 1), "ms_per_step": round(ms32 / K, 3)}
    # FP32 mode, batched + graph, autotuned
    ens = Ensemble(sims)
    rows = ens.tune(steps=2)
    best = min(rows, key=lambda r: r[4])
    ens.step(W)
    ens.sync()
    st = torch.cuda.ExternalStream(ens.stream())
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(st)
    ens.step(K)
    t1.record(st)
    ens.sync()
    torch.cuda.synchronize()
    msb = t0.elapsed_time(t1)
    ens.close()
    for sm in sims:
        sm.close()
    out["fp32_batched"] = {"value": round(total * K / (msb * 1e-3), 1), "ms_per_step": round(msb / K, 3),
                           "launches_per_step": 4 * 2 + 2 * 4 + 2 + 1,
                           "tuned_shape": {"push_ctas": int(best[0]), "tile": [int(best[1]), int(best[2])],
                                           "parts": int(best[3])},
                           "tuning_table_ms": [[int(r[0]), int(r[1]), int(r[2]), int(r[3]), round(r[4], 3)]
                                               for r in rows]}
    out["fp32_batched_over_fp64_unbatched"] = round(ms64 / msb, 2)
    out["fp32_batched_over_fp32_unbatched"] = round(ms32 / msb, 2)
    return out


def small_members():
    """256 members of 512 x 104 meshes at 20 um with 4000 particles each,
    CIC / TSC / cubic in turn."""
    from csrst_b200.workloads import workload as wl
    small = []
    for k in range(256):
        c, sp = wl(f"small-{k % 3}")
        sp.seed = 500 + k
        small.append((c, sp))
    return small


def ensemble_only(args):
    """The batched FP32 ensemble alone (for profiling): build, tune or set
    the launch shape, warm up, time `steps` steps on the device."""
    import torch
    from csrst_b200 import Ensemble, Simulation
    from csrst_b200.workloads import ensemble_members, make_bunch
    ms = small_members() if args.ensemble_only == "small" else ensemble_members(64, seed=2024)
    sims = []
    for cfg, spec in ms:
        sm = Simulation(cfg, fp32=True)
        sm.load(*make_bunch(spec))
        if args.ensemble_only == "c3":
            sm.initial_fields(1e-12, 1e-6, 500)
        sims.append(sm)
    ens = Ensemble(sims)
    if args.shape:
        ens.set_shape(*(int(v) for v in args.shape.split(",")))
    else:
        ens.tune(steps=2)
    ens.step(args.warmup)
    ens.sync()
    st = torch.cuda.ExternalStream(ens.stream())
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(st)
    ens.step(args.steps)
    t1.record(st)
    ens.sync()
    ms_ = t0.elapsed_time(t1) / args.steps
    total = sum(spec.n for _, spec in ms)
    ens.close()
    for sm in sims:
        sm.close()
    return {"ensemble": args.ensemble_only, "members": len(ms), "particles": total, "ms_per_step": round(ms_, 4),
            "particle_steps_per_s": round(total / (ms_ * 1e-3), 1), "shape": args.shape or "tuned"}


def run_surrogate(args):
    """The learned part, measured live.  (1) Inference of the wake surrogate
    (1D FNO: width 128, 32 modes, 4 layers; every product on the tcgen05
    GEMM) at a batch of 65536 profiles resident on the device, with the
    weights as initialised (the time does not depend on their values), and
    its tensor roofline.  (2) Training steps per second (batch 64, the step
    captured as one CUDA graph).  (3) What the surrogate replaces: the batched
    FP32 PIC's cost per data-set case (256 cases stepped as one ensemble for
    256 steps, scaled to a case's 2144 steps; set-up reported apart), and the
    screening speed-up.  Its accuracy against PIC needs the 4096-run data set
    and a trained model: profiles/surrogate_wake.md."""
    import torch
    from csrst_b200 import wakescreen, wakeset
    from csrst_b200.pic import Ensemble, Simulation
    from csrst_b200.surrogate import FNO
    out = {}
    cases = wakeset.draw_cases(256, seed=99)
    X6 = wakeset.features(cases)
    net = FNO(seed=0)
    model = wakescreen.WakeModel(net, np.zeros(7), 1.0)
    inf = wakescreen.time_inference(model, X6, n=65536, chunk=8192)
    hbm, tf_peak, src = peaks(bf16=True)
    variants = wakescreen.c5_variants(20000)
    t0 = time.perf_counter()
    wakeset.features(variants)
    feat_s = (time.perf_counter() - t0) / len(variants)
    # about 65 flop per byte: far below the B200's ridge point, so the bound is HBM
    out["inference"] = dict(inf, roofline={"kernel": "the forward pass (tensor-core GEMMs + transposes)",
                                           "bound": "hbm", "achieved": round(inf["gbs"], 1), "peak": hbm,
                                           "unit": "GB/s", "frac": round(inf["gbs"] / hbm, 4),
                                           "algorithmic_bytes_per_profile": inf["bytes_per_profile"],
                                           "peak_source": src.replace("bf16_tflops", "hbm_gbs")},
                            tensor={"achieved": round(inf["tflops"], 2), "peak": tf_peak, "unit": "TFLOP/s",
                                    "frac": round(inf["tflops"] / tf_peak, 4), "peak_source": src},
                            host_features_s_per_profile=round(feat_s, 7))
    # training steps
    B = 64
    Xs = torch.from_numpy(wakescreen.pad_features(np.repeat(X6[:B], 1, axis=0))).cuda().to(torch.bfloat16)
    Ts = torch.randn(B, wakeset.NBINS, 32, device="cuda")
    Ms = torch.ones_like(Ts)
    net.loss_and_grad(Xs, Ts, Ms)
    net.adam(total=1000)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        net.loss_and_grad(Xs, Ts, Ms)
        net.adam(total=1000)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(200):
        g.replay()
    b.record()
    torch.cuda.synchronize()
    net.check()
    out["training"] = {"batch": B, "ms_per_step": round(a.elapsed_time(b) / 200, 4),
                       "library_calls_per_step": 106,
                       "what": "forward, hand-written backward and Adam, captured as one CUDA graph"}
    del g
    # the PIC it replaces: 256 data-set cases as one ensemble
    t0 = time.perf_counter()
    sims = []
    for c in cases:
        cfg, lb = wakeset.case_config(c)
        try:
            s = Simulation(cfg, fp32=True)
        except Exception:
            continue
        s.load(*wakeset.case_bunch(c, cfg, lb, 50_000))
        s.initial_fields()
        sims.append(s)
    ens = Ensemble(sims)
    ens.sync()
    setup = (time.perf_counter() - t0) / len(sims)
    ens.step(8)
    ens.sync()
    st = torch.cuda.ExternalStream(ens.stream())
    a.record(st)
    ens.step(256)
    b.record(st)
    ens.sync()
    ms = a.elapsed_time(b) / 256
    ens.close()
    for s in sims:
        s.close()
    per_case = ms * 1e-3 * wakeset.station_steps()[-1] / len(sims)
    sur = inf["seconds"] / inf["profiles"]
    out["pic_per_case"] = {"members": len(sims), "ms_per_ensemble_step": round(ms, 3),
                           "stepping_s_per_case": round(per_case, 5), "setup_s_per_case": round(setup, 4),
                           "what": "50k-particle TSC cases, 2144 steps, FP32 batched ensemble of 256"}
    out["screening_speedup"] = {"network_only": round(per_case / sur), "with_host_features": round(per_case / (sur + feat_s)),
                                "bar": ">= 1000x faster than PIC"}
    return out


DATA = "synthetic (seeded Gaussian bunch; initial fields from the GPU multigrid Poisson solve)"


def run_config(args, cfg, spec, world, window, h):
    """The workload as both arms name it (the precision is the line's dtype)."""
    return {"workload": f"{args.workload}: {cfg.Nx}x{cfg.Ny} static mesh, h={1e6 * h:.3g}um, "
                        f"{spec.n} particles, shape order {cfg.shape_order}, CFL 0.5",
            "Nx": cfg.Nx, "Ny": cfg.Ny, "particles": spec.n, "shape_order": cfg.shape_order,
            "window": [int(v) for v in window], "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (126 MB): 4 static planes of %.3g M cells, %.3g M particles" % (
                cfg.Nx * cfg.Ny / 1e6, spec.n / 1e6)}


def run_b200(args, world, rank, local):
    import torch
    from csrst_b200.workloads import make_bunch, workload

    torch.cuda.set_device(local)
    cfg, spec = workload(args.workload)
    spec.seed += rank
    bunch = make_bunch(spec)
    n = spec.n
    cells = cfg.Nx * cfg.Ny
    head = args.precision
    # clocks are sampled from before the first warm-up to the end of the last
    # attribution pass: the GPU runs this workload the whole time
    clocks = Clocks(local) if rank == 0 else None
    runs = {head: time_mode(args, cfg, bunch, world, head == "fp32", clocks)}
    other = "fp64" if head == "fp32" else "fp32"
    if not args.no_compare:
        runs[other] = time_mode(args, cfg, bunch, world, other == "fp32", clocks)
    clk = clocks.stop() if clocks else None
    hbm, src = peaks()

    def roof(key, prec, bytes_step, ms_):
        ach = bytes_step / (ms_ * 1e-3) / 1e9
        tr, tsrc = profile_traffic(key, prec, cfg.shape_order) if args.workload == "c2" else (None, None)
        return {"kernel": key, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(ach / hbm, 4), "traffic": tr, "traffic_source": tsrc,
                "peak_source": f"{src} hbm_gbs",
                "algorithmic_bytes_per_step": bytes_step, "ms_per_step": round(ms_, 4)}

    def summary(prec):
        r = runs[prec]
        g = r["groups"]
        r_yee = roof("yee", prec, YEE_BYTES[prec] * cells, g["yee"])
        r_push = roof("push", prec, 2 * PUSH_BYTES[prec] * n, g["push"])
        dom, oth = (r_yee, r_push) if g["yee"] >= g["push"] else (r_push, r_yee)
        return {"value": round(world * n * args.steps / (r["ms"] * 1e-3), 1),
                "ms_per_step": round(r["ms"] / args.steps, 4),
                "cell_updates_per_s": round(world * cells * args.steps / (r["ms"] * 1e-3), 1),
                "roofline": dom, "roofline_other": oth,
                "kernel_ms_per_step": {k: round(v, 4) for k, v in g.items()},
                "initial_fields": dict(r["initial_fields"],
                                       what="one-time set-up, not in the timed steps: 3 MG-PCG solves on the "
                                            f"{cfg.Nx}x{cfg.Ny} mesh incl. charge deposits and host round trips")}

    hs = summary(head)
    dtype = ("f32 (fields, gather, kick, drifts, positions, current path integral) + f64 (bend frame, end-point "
             "charge weights) + i64 (fixed-point current)") if head == "fp32" else "f64"
    out = {"metric": METRIC, "value": hs["value"], "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": hs["ms_per_step"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
           "data": DATA,
           "config": run_config(args, cfg, spec, world, runs[head]["window"], runs[head]["hx"]),
           "cell_updates_per_s": hs["cell_updates_per_s"],
           "roofline": hs["roofline"], "roofline_other": hs["roofline_other"],
           "kernel_ms_per_step": hs["kernel_ms_per_step"], "initial_fields": hs["initial_fields"],
           "clocks": clk}
    if other in runs:
        out[other] = summary(other)
        out[f"{head}_over_{other}"] = round(hs["value"] / out[other]["value"], 3)
    # launches per FP32 step: the first push (prep, push, closing kernel that
    # also sets up the second), the second push (push, closing kernel), the
    # fused field sweep (tiles, window fix-up), the window's Ey, and the move
    # (two copy stages, finish)
    out["gpu_launches"] = args.steps * (3 + 2 + 2 + 1 + 3)
    if rank == 0 and not args.no_compare:
        out["accuracy_fp32_vs_fp64"] = accuracy(cfg, spec, bunch)
    if not args.no_ensemble:
        out["batched_ensemble"] = run_ensemble(args, rank)
        # many small members: the regime where the batch's few launches per step matter
        small = small_members()
        out["batched_ensemble_small"] = dict(run_ensemble(args, rank, ms=small, fields=False),
                                             what="256 members of 512x104 meshes at 20 um with 4000 particles "
                                                  "each, CIC/TSC/cubic, zero initial fields")
    if rank == 0 and not args.no_surrogate:
        out["surrogate"] = run_surrogate(args)
    if not args.no_e2e:
        out["e2e"] = run_e2e(args, cfg, spec, bunch, rank, world, head == "fp32")
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(cfg, spec, bunch)
    return out if rank == 0 else None


def run_e2e(args, cfg, spec, bunch, rank, world, fp32):
    """The same metric through the C ABI with host buffers: the bunch goes
    up from pinned host memory, every step returns the beam moments to the
    host, and the bunch comes back at the end."""
    import torch
    from csrst_b200 import Simulation
    n = spec.n
    pinned = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in bunch]
    outp = [torch.empty(n, dtype=torch.float64).pin_memory().numpy() for _ in range(4)]
    sim = Simulation(cfg, fp32=fp32)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t = time.perf_counter()
    sim.load(*pinned)
    for _ in range(args.warmup + args.steps):
        sim.step(1)
        sim.moments()
    from csrst_b200._lib import lib, ptr
    lib().csrst_get_particles(sim.h, *map(ptr, outp))
    torch.cuda.synchronize()
    el = max_over_ranks(time.perf_counter() - t, world)
    k = args.warmup + args.steps
    sim.close()
    return {"value": round(world * n * k / el, 1), "unit": UNIT,
            "h2d_bytes_per_step": int(5 * 8 * n / k), "d2h_bytes_per_step": int(18 * 8 + 4 * 8 * n / k),
            "steps": k, "includes": "bunch upload, window set-up and sort, steps, per-step moments, bunch download "
                                    "(zero initial fields: the solve is reported under initial_fields)"}


def oracle_steps(cfg, bunch, warmup, steps):
    """The oracle (the CPU restatement of the reference loop, plain FP64 sums
    in the reference's order) on the full workload: load, `warmup` untimed
    steps, then `steps` timed steps.  Returns (seconds per step, window size,
    mesh spacing hx)."""
    from oracle import oracle as O
    d = cfg.dict()
    d["order"] = cfg.shape_order
    s = O.Sim(d)
    s.load(*bunch)
    s.step(warmup)
    t = time.perf_counter()
    s.step(steps)
    el = time.perf_counter() - t
    hx = O.bend(cfg.Nx, cfg.Ny, cfg.length_before, cfg.length_after, cfg.width, cfg.phi_deg, cfg.ekin_mev,
                cfg.bz)["hx"]
    return el / max(steps, 1), list(s.window()[0][2:]), hx


def cpu_baseline(cfg, spec, bunch, steps=2):
    sec, _, _ = oracle_steps(cfg, bunch, 0, steps)
    return {"value": round(spec.n / sec, 1), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"oracle (C++ restatement of the reference loop, -O2 -ffp-contract=off), 1 thread: "
                      f"{steps} full steps of the whole workload ({cfg.Nx}x{cfg.Ny} mesh, {spec.n} particles), "
                      f"{sec:.2f} s per step, nothing extrapolated"}


def _ref_worker(args):
    name, seed, warmup, steps = args
    from csrst_b200.workloads import make_bunch, workload
    cfg, spec = workload(name)
    spec.seed = seed
    return oracle_steps(cfg, make_bunch(spec), warmup, steps)


def ref_cores():
    """Host cores the reference arm uses: all it may run on, capped by the
    memory one full-workload replica needs (about 0.8 GB)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
        n = min(n, max(1, int(avail * 0.5 / 0.8e9)))
    except (ValueError, OSError):
        pass
    return max(1, min(n, 64))


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of the reference loop on the
    box's host cores, one full-workload replica per core (the loop does not
    shard; replicas are its only parallelism on the host), each running the
    declared warm-up and timed steps in full.  value = all replicas'
    particle-steps / the slowest replica's timed seconds."""
    if rank != 0:
        return None
    import multiprocessing as mp
    from csrst_b200.workloads import workload
    cfg, spec = workload(args.workload)
    cores = ref_cores()
    t = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_ref_worker, [(args.workload, spec.seed + k, args.warmup, args.steps) for k in range(cores)])
    wall = time.perf_counter() - t
    sec = max(r[0] for r in res)
    value = cores * spec.n / sec
    return {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sec, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the same seeded Gaussian bunch generator; zero initial fields: a step's work does "
                    "not depend on the field values)",
            "config": run_config(args, cfg, spec, world, res[0][1], res[0][2]),
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{cores} replica processes of the oracle (C++ restatement of the reference "
                                       f"loop), each the whole workload for {args.warmup} warm-up + {args.steps} "
                                       f"timed steps; slowest replica {sec:.2f} s per step; wall {wall:.1f} s"},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        # CPU work of rank 0 alone: no process group and no GPU; the other
        # ranks leave at once with status 0
        out = run_reference(args, world, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import torch
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.ensemble_only and args.impl != "reference":
            import torch
            torch.cuda.set_device(local)
            out = ensemble_only(args) if rank == 0 else None
        else:
            out = run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
