"""The surrogate's wake data set on the CPU: profile families, the
two-dimensional quiet start, the mesh each case gets (the geometry builds in
the CPU oracle), input features and the compact file format."""
import dataclasses
import os
import tempfile

import numpy as np
import pytest

from csrst_b200 import wakeset as ws


def test_profiles_normalised_and_centred():
    for c in ws.draw_cases(9):
        z, d, mu, rms = ws.profile(c)
        assert abs(np.trapezoid(d, z) - 1) < 1e-9
        lam = ws.line_density(c)
        assert abs(lam.sum() * 2 * ws.SPAN / ws.NBINS - 1) < 2e-3      # mass inside +-4 sigma_s
        u = ws.quiet_offsets(c, 40_000) / c.sigma_s
        assert abs(u.mean()) < 1e-3 and abs(u.std() - 1) < 2e-3
        assert np.all(np.diff(u) >= 0)                                   # quantiles in order


def test_quiet_start_is_quiet_and_seeded():
    c = ws.draw_cases(1)[0]
    cfg, lb = ws.case_config(c)
    x, y, px, py, q = ws.case_bunch(c, cfg, lb, 20_000)
    assert abs(q.sum() - ws.CHARGE) < 1e-18 and np.all(py == 0)
    assert abs((y - 0.5 * cfg.width).std() / (c.sigma_s / 2.5) - 1) < 5e-3
    # line density of the loaded bunch equals the profile (no shot noise in s)
    h = (2 * ws.SPAN / ws.NBINS) * c.sigma_s
    xc = x - x.mean()
    hist, _ = np.histogram(xc, bins=ws.NBINS, range=(-ws.SPAN * c.sigma_s, ws.SPAN * c.sigma_s))
    lam = ws.line_density(c) * len(x) * h / c.sigma_s
    assert np.abs(hist - lam).max() <= 0.02 * lam.max() + 2
    # another seed moves the transverse lattice, not the longitudinal quantiles
    x2, y2, *_ = ws.case_bunch(dataclasses.replace(c, seed=c.seed + 1), cfg, lb, 20_000)
    assert np.array_equal(np.sort(x), np.sort(x2)) and not np.array_equal(y, y2)


def test_case_meshes():
    for c in ws.draw_cases(60)[::7]:
        cfg, lb = ws.case_config(c)
        h = c.sigma_s / ws.CELLS_PER_SIGMA
        assert cfg.dt == pytest.approx(0.5 * h / 299792458.0)
        # the reference's domain rule gives square cells of h
        phi = np.radians(cfg.phi_deg)
        box_l = cfg.length_before + cfg.length_after * np.cos(phi) + (c.R + 0.5 * cfg.width) * np.sin(phi)
        box_w = (c.R - 0.5 * cfg.width) * (1 - np.cos(phi)) + cfg.width + cfg.length_after * np.sin(phi)
        assert box_l / (cfg.Nx - 2) == pytest.approx(h, rel=1e-9)
        assert box_w / (cfg.Ny - 2) == pytest.approx(h, rel=1e-9)
        # the bunch starts in the straight section with room for its window behind it
        assert lb - 6 * c.sigma_s - 4.5 * c.sigma_s > 20 * h
        # the bend holds the whole travel of the stations
        assert c.R * phi >= ws.NSTATIONS * ws.STATION_STEPS * 0.5 * h + 5 * c.sigma_s


def test_case_geometry_builds_in_the_oracle():
    from oracle.oracle import Sim
    for c in ws.draw_cases(40)[::13]:
        cfg, _ = ws.case_config(c)
        d = cfg.dict()
        d["order"] = d.pop("shape_order")
        Sim(d)


def test_features_ranges():
    X = ws.features(ws.draw_cases(300))
    assert X.shape == (300, ws.NBINS, ws.NFEATURES)
    assert np.all(np.abs(X[:, :, 1:6]) <= 1.05)
    assert np.all(X[:, :, 0] >= 0)


def test_file_round_trip_and_skipped_cases():
    cs = ws.draw_cases(5)
    w = np.random.default_rng(0).standard_normal((5, ws.NBINS, ws.NSTATIONS)).astype(np.float32) * 2e5
    w[3] = np.nan
    m = np.random.default_rng(1).random((5, ws.NBINS, ws.NSTATIONS)) < 0.8
    p = tempfile.mktemp(suffix=".npz")
    try:
        ws.save(p, dict(cases=cs, X=ws.features(cs), W=w, M=m, facts=[{"members": 5}]))
        d = ws.load(p)
    finally:
        os.remove(p)
    keep = [0, 1, 2, 4]
    assert d["skipped"] == 1 and d["cases"] == [cs[k] for k in keep]
    assert np.array_equal(d["M"], m[keep])
    peak = np.abs(w[keep]).max(axis=(1, 2))
    assert np.all(np.abs(d["W"] - w[keep]).max(axis=(1, 2)) <= 6e-4 * peak)
