"""FP32 mode (CSRST_FLAG_FP32) against the FP64 GPU path, which is itself
bit-exact to the oracle.

FP32 mode has no reference counterpart.  Its bar: the longitudinal wake on
the bunch within 1e-3 of the FP64 path's (relative to the wake's maximum);
the current it deposits equal to the FP64 deposit of the same moves to 1e-6;
the discrete continuity equation satisfied exactly in integers for the
charge the deposit assigns and to 1e-10 relative against the FP64 charge
shape."""
import numpy as np
import pytest

from csrst_b200 import ShapeFunction, Simulation, TETMSolver, moveMesh
from csrst_b200.workloads import make_bunch, workload

pytestmark = pytest.mark.gpu

WAKE_TOL = 1e-3


def run(name, fp32, steps, fields=True):
    cfg, spec = workload(name)
    s = Simulation(cfg, fp32=fp32)
    s.load(*make_bunch(spec))
    if fields:
        s.initial_fields()
    s.step(steps)
    return s


def wake_err(a, b):
    ok = np.isfinite(a) & np.isfinite(b)
    assert ok.sum() > 10
    return np.abs(a[ok] - b[ok]).max() / np.abs(b[ok]).max()


@pytest.mark.parametrize("name", ["small-0", "small-1", "small-2", "small-1-bend"])
def test_fp32_wake_and_bunch_vs_fp64(gpu_lib, name):
    steps = 60
    # the initial-field solve covers the straight section before the bend
    # (PoissonSolver::cutoffStencil): a bunch that starts in the dipole runs
    # from zero fields
    fields = "bend" not in name
    s64, s32 = run(name, False, steps, fields), run(name, True, steps, fields)
    assert s64.window()[0] == s32.window()[0]
    err = wake_err(s32.wake(), s64.wake())
    assert err <= WAKE_TOL, err
    h = s64.info()["hx"]
    p64, p32 = s64.particles(), s32.particles()
    assert np.abs(p32[0] - p64[0]).max() < 1e-3 * h     # positions within 1e-3 cells
    assert np.abs(p32[1] - p64[1]).max() < 1e-3 * h
    m64, m32 = s64.moments(), s32.moments()
    assert m32[14] == pytest.approx(m64[14], rel=1e-9)  # kinetic energy
    assert abs(m32[15] - m64[15]) <= 1e-3 * abs(m64[15])  # energy spread
    s64.close(); s32.close()


def test_fp32_initial_fields_match_fp64(gpu_lib):
    """FP32 mode solves in FP64 for its FP32-stored bunch and rounds the
    fields once: they agree with the FP64 path's to FP32 precision."""
    s64, s32 = run("small-1", False, 0), run("small-1", True, 0)
    for a, b in zip(s32.get_static(), s64.get_static()):
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()
    s64.close(); s32.close()


def unpack(cell):
    return (cell & 0xFFFF).astype(np.int64), (cell.astype(np.uint32) >> 16).astype(np.int64)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_fp32_push_current_conserves_charge_exactly(gpu_lib, order):
    """FP32-mode pushes (keep_old) after 3 steps in the dipole: each push's
    window current is, bit for bit, the stand-alone FP32 deposit
    (csrst_flux32) of the moves it made; those moves satisfy
    drho + div F = 0 exactly in integers; the current equals the FP64
    path-integral deposit of the same moves (read back as FP64 positions) to
    1e-6 of its maximum and the charge change the FP64 charge shape to 1e-10,
    so that rho/dt + div J <= 1e-10 holds against the FP64 charge too."""
    cfg, spec = workload(f"small-{order}-bend")
    s = Simulation(cfg, fp32=True, keep_old=True)
    s.load(*make_bunch(spec))
    s.step(3)
    info = s.info()
    h, dt, scale = (info["hx"], info["hy"]), info["dt"], info["fixed_scale"]
    sf = ShapeFunction(order)
    for comp in (0, 1):
        xo, yo, _, _ = s.particles()
        s.push(comp)
        c1, b0, b1, _, _, q = s.bunch32(0)
        c0, a0, a1 = s.bunch32(1)
        xn, yn, _, _ = s.particles()
        w, org, _ = s.window()
        P0, P1, L0, L1 = w
        jwin = s.window_field(4 + comp)[1:L1 + 1, 1:L0 + 1]
        F = [None, None]
        F[0], drho = sf.flux32(0, c0, a0, a1, c1, b0, b1, q, scale, P0, P1, L0, L1, with_charge=True)
        F[1] = sf.flux32(1, c0, a0, a1, c1, b0, b1, q, scale, P0, P1, L0, L1)
        inv = 1.0 / (scale * dt * h[1 - comp])
        assert np.array_equal(jwin, F[comp].astype(np.float64) * inv)
        res = drho[1:, 1:] + (F[0][1:, 1:] - F[0][1:, :-1]) + (F[1][1:, 1:] - F[1][:-1, 1:])
        assert np.abs(drho).max() > 0 and (res == 0).all()
        # against the FP64 reference deposit of the same moves
        ci, cj = unpack(c0)
        ox = info["ox"] + (ci + a0.astype(np.float64)) * h[0]
        oy = info["oy"] + (cj + a1.astype(np.float64)) * h[1]
        assert np.abs(ox - xo).max() < 1e-12 and np.abs(oy - yo).max() < 1e-12  # the start is the bunch as read
        q64 = q.astype(np.float64)
        jscale = 2.0 ** np.floor(np.log2(2.0 ** 62 / (4.0 * len(q64) * np.abs(q64).max() * 299792458.0
                                                      / (h[0] * h[1]))))
        ref = sf.getCurrentDensityBase(comp, ox, oy, xn, yn, q64, org, h, dt, 0, 0, L0, L1, jscale)
        assert np.abs(jwin - ref).max() <= 1e-6 * np.abs(ref).max()
        qs = 2.0 ** np.floor(np.log2(2.0 ** 62 / (4 * np.abs(q64).sum())))
        rho = sf.getChargeDensityDiff(ox, oy, xn, yn, q64, org, h, 0, 0, L0, L1, qs)
        jx = F[0] / (scale * dt * h[1])
        jy = F[1] / (scale * dt * h[0])
        r64 = rho[1:, 1:] / dt + (jx[1:, 1:] - jx[1:, :-1]) / h[0] + (jy[1:, 1:] - jy[:-1, 1:]) / h[1]
        assert np.abs(r64).max() <= 1e-10 * np.abs(rho / dt).max()
        s.update_e(comp)
        s.drift(-0.5 * dt)
    s.close()


def test_fp32_graph_matches_eager_and_reruns(gpu_lib):
    cfg, spec = workload("small-1")
    b = make_bunch(spec)
    out = []
    for eager in (False, True, False):
        s = Simulation(cfg, fp32=True)
        s.load(*b)
        if eager:
            solver = TETMSolver(s)
            for _ in range(6):
                solver.updateField_firstStep()
                solver.updateField_secondStep()
                moveMesh(s)
        else:
            s.step(6)
        out.append(s.particles() + [s.window_field(k) for k in range(6)])
        s.close()
    for a, c, d in zip(*out):
        assert np.array_equal(a, c) and np.array_equal(a, d)


def test_fp32_full_size_c2(gpu_lib):
    """The 8192 x 1024 / 4e6-particle TSC workload: FP32 wake within 1e-3 of
    FP64 after 20 steps."""
    s64, s32 = run("c2", False, 20), run("c2", True, 20)
    assert wake_err(s32.wake(), s64.wake()) <= WAKE_TOL
    s64.close(); s32.close()


def test_fp32_rejects_large_meshes(gpu_lib):
    big = workload("small-0")[0]
    big.Nx = 40000
    with pytest.raises(Exception):
        Simulation(big, fp32=True)


def test_fp32_energy_change_per_slice_in_the_dipole(gpu_lib):
    """A bunch entering the dipole loses energy to CSR; FP32 mode's energy
    change per slice stays within 1e-3 of the FP64 path's after 200 steps."""
    cfg, spec = workload("small-1-bend")
    b = make_bunch(spec)
    dg, pos = {}, None
    for fp32 in (False, True):
        s = Simulation(cfg, fp32=fp32)
        s.load(*b)
        _, _, px, py = s.particles()
        g0 = np.sqrt(1 + px * px + py * py)
        s.step(200)
        x, y, px, py = s.particles()
        dg[fp32] = np.sqrt(1 + px * px + py * py) - g0
        if not fp32:
            pos = (x, s.moments())
        s.close()
    x, m = pos
    edges = np.linspace(m[0] - 3 * spec.sigma_s, m[0] + 3 * spec.sigma_s, 17)
    idx = np.clip(np.digitize(x, edges) - 1, 0, 15)
    cnt = np.maximum(np.bincount(idx, minlength=16), 1)
    e64 = np.bincount(idx, dg[False], minlength=16) / cnt
    e32 = np.bincount(idx, dg[True], minlength=16) / cnt
    assert np.abs(e64).max() > 0
    assert np.abs(e32 - e64).max() <= 1e-3 * np.abs(e64).max()


def test_fp32_csr_wake_through_the_dipole_c1(gpu_lib):
    """The c1 geometry (2048 x 512 at 10 um, R = 1 m, 5 mm pipe, 2e5
    particles, CIC) with the bunch starting at the dipole entrance, 2000 steps
    (1000 cells of the 1440-cell arc): FP32 mode's wake on the bunch axis and
    its time integral (the reference's energy change, sampled every 100
    steps) stay within 1e-3 of the FP64 path's maxima (measured 1.0e-4 and
    2.3e-5); the energy change of 16 slices, from every particle's gamma,
    within 3e-3 (measured 1.5e-3: the FP32 momentum deviations accumulate
    4000 rounded kicks)."""
    from csrst_b200.compare import fp32_vs_fp64
    r = fp32_vs_fp64("c1-bend", 2000, every=100)
    assert r["wake_samples"] >= 50 and r["integrated_columns"] > 500
    assert r["wake_rel_err"] <= WAKE_TOL, r
    assert r["integrated_rel_err"] <= WAKE_TOL, r
    assert r["slice_rel_err"] <= 3e-3, r
    assert max(abs(v) for v in r["slice_mev_fp64"]) > 0
