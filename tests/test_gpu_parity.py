"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Bar: bit-exact (array_equal) for geometry, gathers, particle positions and
momenta, cell indices, window position and all fields when the oracle
accumulates the current in the same 64-bit fixed point as the GPU; within a
stated relative tolerance against the oracle's plain FP64 current sums
(the reference's order of summation).
"""
import numpy as np
import pytest

from csrst_b200 import CsrstError, ScatterGatherImpl, ShapeFunction, Simulation, TETMSolver
from csrst_b200.workloads import make_bunch, workload

pytestmark = pytest.mark.gpu

C_LIGHT = 299792458.0


def smooth_fields(cfg, seed, amp=2e5):
    """Smooth random fields on the static mesh (V/m, A/m)."""
    rng = np.random.default_rng(seed)
    j, i = np.mgrid[0:cfg.Ny, 0:cfg.Nx]
    out = []
    for k in range(4):
        f = np.zeros((cfg.Ny, cfg.Nx))
        for _ in range(3):
            kx, ky = rng.uniform(0.01, 0.2, 2)
            ph = rng.uniform(0, 6.3, 2)
            f += rng.uniform(-1, 1) * np.sin(kx * i + ph[0]) * np.cos(ky * j + ph[1])
        out.append(f * (amp if k < 2 else amp / 376.73))
    return out


def pair(name, oracle, fixed=True, fields=True, keep_old=False, seed=0):
    cfg, spec = workload(name)
    g = Simulation(cfg, keep_old=keep_old)
    bunch = make_bunch(spec)
    d = cfg.dict()
    d["order"] = cfg.shape_order
    if fields:
        f = smooth_fields(cfg, seed)
        g.set_static(*f)
    g.load(*bunch)
    if fixed:
        d["fixed_scale"] = g.info()["fixed_scale"]
    o = oracle.Sim(d)
    if fields:
        o.set_static(*f)
    o.load(*bunch)
    return cfg, g, o


def assert_same_state(g, o, fields=True):
    for a, b in zip(g.particles(), o.particles()):
        assert np.array_equal(a, b)
    wg, og, bg = g.window()
    wo, oo, bo = o.window()
    assert wg == wo and np.array_equal(og, oo)
    if fields:
        for a, b in zip(g.get_static(), o.get_static()):
            assert np.array_equal(a, b)
        for k in range(4):
            assert np.array_equal(g.window_field(k), o.window_field(k)), k


def test_geometry_bit_exact(gpu_lib, oracle):
    for name in ("small-0", "c1"):
        cfg, _ = workload(name)
        g = Simulation(cfg)
        gi, gc = g.geometry()
        oi, oc = oracle.geometry(cfg.Nx, cfg.Ny, cfg.length_before, cfg.length_after, cfg.width,
                                 cfg.phi_deg, cfg.ekin_mev, cfg.bz)
        assert np.array_equal(gi, oi)
        assert np.array_equal(gc, oc)
        g.close()


@pytest.mark.parametrize("order", [0, 1, 2])
def test_gather_golden_and_random(gpu_lib, oracle, order):
    sg = ScatterGatherImpl(order)
    x, y = np.array([3.3]), np.array([3.2])
    for comp in (0, 1, 2):
        w = oracle.scatter(order, comp, (21, 21), (0, 0), (1, 1), x, y, [1.0])
        v = sg.gather((w != 0).astype(float), (0, 0), (1, 1), x, y, comp)[0]
        assert abs(v - 1.0) < 1e-12   # test/scattergather.cpp:133-166, :218-269, :344-416
    rng = np.random.default_rng(order)
    patch = rng.standard_normal((40, 50))
    xs = rng.uniform(4, 44, 2000) * 1e-5 + 1e-3
    ys = rng.uniform(4, 34, 2000) * 2e-5 - 2e-3
    for comp in (0, 1, 2):
        a = sg.gather(patch, (1e-3, -2e-3), (1e-5, 2e-5), xs, ys, comp)
        b = oracle.gather(order, comp, patch, (1e-3, -2e-3), (1e-5, 2e-5), xs, ys)
        assert np.array_equal(a, b)


def charge_scale(q):
    """Fixed-point scale for a charge sum: a power of two with 4 sum|q| below 2^62."""
    return 2.0 ** np.floor(np.log2(2.0 ** 62 / (4.0 * np.abs(q).sum())))


def random_moves(n, h, seed, cfl=0.5):
    rng = np.random.default_rng(seed)
    ox = rng.uniform(6, 14, n) * h[0]
    oy = rng.uniform(6, 14, n) * h[1]
    ang = rng.uniform(0, 2 * np.pi, n)
    r = rng.uniform(0, cfl, n) * min(h)
    return ox, oy, ox + r * np.cos(ang), oy + r * np.sin(ang), rng.uniform(-2e-15, 2e-15, n)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_deposit_parity_and_continuity(gpu_lib, oracle, order):
    h = (1e-5, 1.2e-5)
    dt = 0.5 * h[0] / C_LIGHT
    ox, oy, x, y, q = random_moves(20000, h, order)
    bound = 4.0 * len(q) * np.abs(q).max() * C_LIGHT / (h[0] * h[1])
    scale = 2.0 ** np.floor(np.log2(2.0 ** 62 / bound))
    sf = ShapeFunction(order)
    J = {}
    for comp in (0, 1):
        a = sf.getCurrentDensityBase(comp, ox, oy, x, y, q, (0, 0), h, dt, 0, 0, 24, 24, scale)
        b = oracle.deposit(order, comp, ox, oy, x, y, q, (0, 0), h, dt, 0, 0, 24, 24, fixed_scale=scale)
        c = oracle.deposit(order, comp, ox, oy, x, y, q, (0, 0), h, dt, 0, 0, 24, 24)
        assert np.array_equal(a, b)                                   # same fixed point: bit-exact
        assert np.abs(a - c).max() <= 1e-12 * np.abs(c).max()         # reference FP64 order: 1e-12
        J[comp] = a
    rho = sf.getChargeDensityDiff(ox, oy, x, y, q, (0, 0), h, 0, 0, 24, 24, charge_scale(q))
    res = rho[1:, 1:] / dt + (J[0][1:, 1:] - J[0][1:, :-1]) / h[0] + (J[1][1:, 1:] - J[1][:-1, 1:]) / h[1]
    assert np.abs(res).max() <= 1e-10 * np.abs(rho / dt).max()


@pytest.mark.parametrize("name", ["small-0", "small-1", "small-2", "small-1-bend"])
def test_push_bit_exact(gpu_lib, oracle, name):
    cfg, g, o = pair(name, oracle, keep_old=True)
    g.push(0)
    o.push(0)
    assert_same_state(g, o, fields=False)
    for a, b in zip(g.old_positions(), o.old_positions()):
        assert np.array_equal(a, b)
    assert g.window()[2] == o.window()[2]               # PartBunch::getGlobalBounds
    assert np.array_equal(g.window_field(4), o.window_field(4))   # J_x of the window


@pytest.mark.parametrize("name", ["small-0", "small-1"])
def test_field_substeps_bit_exact(gpu_lib, oracle, name):
    cfg, g, o = pair(name, oracle)
    for s in (g, o):
        s.push(0)
        s.half_h()
    assert_same_state(g, o)
    for s in (g, o):
        s.update_e(0)
        s.half_h()
    assert_same_state(g, o)
    for s in (g, o):
        s.drift(-0.5 * s.dt if s is o else -0.5 * g.info()["dt"])
        s.push(1)
        s.update_e(1)
    assert_same_state(g, o)


@pytest.mark.parametrize("name", ["small-0", "small-1", "small-2", "small-1-bend"])
def test_steps_bit_exact_fixed_point(gpu_lib, oracle, name):
    cfg, g, o = pair(name, oracle)
    g.step(12)       # graph-captured steps
    o.step(12)
    assert_same_state(g, o)
    assert np.array_equal(g.window_field(4), o.window_field(4))
    assert np.array_equal(g.window_field(5), o.window_field(5))


def test_tetm_solver_api_matches_graph_path(gpu_lib):
    cfg, spec = workload("small-1")
    b = make_bunch(spec)
    a, c = Simulation(cfg), Simulation(cfg)
    for s in (a, c):
        s.load(*b)
    solver = TETMSolver(a)
    for _ in range(5):
        solver.updateField_firstStep()
        solver.updateField_secondStep()
        a.move()
    c.step(5)
    for u, v in zip(a.particles(), c.particles()):
        assert np.array_equal(u, v)
    for u, v in zip(a.get_static(), c.get_static()):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("name", ["small-0", "small-1-bend"])
def test_steps_vs_reference_summation(gpu_lib, oracle, name):
    """Against the oracle's FP64 current sums (the reference's order)."""
    cfg, g, o = pair(name, oracle, fixed=False)
    g.step(12)
    o.step(12)
    h = g.info()["hx"]
    gx, gy, gpx, gpy = g.particles()
    ox, oy, opx, opy = o.particles()
    assert np.abs(gx - ox).max() <= 1e-9 * h and np.abs(gy - oy).max() <= 1e-9 * h
    assert np.abs(gpx - opx).max() <= 1e-12 * np.abs(opx).max()
    assert np.abs(gpy - opy).max() <= 1e-12 * np.abs(opx).max()
    # cell indices of the window (bit-exact)
    w, org, _ = g.window()
    assert np.array_equal(np.floor((gx - org[0]) / h), np.floor((ox - org[0]) / h))
    for a, b in zip(g.get_static(), o.get_static()):
        assert np.abs(a - b).max() <= 1e-9 * max(np.abs(b).max(), 1e-300)


def test_moments_and_wake(gpu_lib, oracle):
    cfg, g, o = pair("small-1", oracle)
    g.step(6)
    o.step(6)
    mg, mo = g.moments(), o.moments()
    # groups: rmean, pmean, rrms, prms, eps, rmin, rmax, (Ekin, dE); each
    # within 1e-9 of the group's magnitude.  The momentum spread follows the
    # reference's formula sum(p'^2) - N |<p>|^2 with <p> rounded to double
    # (PartBunch.cpp:620-628): for |<p>| ~ 1e3 and spread ~ 1e-1 that
    # formula itself carries ~1e-8 relative error, which bounds prms, eps
    # and dE; the GPU centres p' first and is the more accurate of the two.
    for a, b, tol in ((0, 2, 1e-9), (2, 4, 1e-9), (4, 6, 1e-9), (6, 8, 1e-7), (8, 10, 1e-7),
                      (10, 12, 1e-9), (12, 14, 1e-9), (14, 15, 1e-9), (15, 16, 1e-7)):
        scale = np.abs(mo[a:b]).max()
        assert np.abs(mg[a:b] - mo[a:b]).max() <= tol * scale, (a, mg[a:b], mo[a:b])
    # dispersion terms Dy, DDy (PartBunch.cpp:643-644): the reference pairs y' and py'
    # with the uncentred px' ~ |<p>|; the GPU with the centred one plus |<p>| sum(y')
    scale = np.abs(mo[16:18]).max()
    assert scale > 0 and np.abs(mg[16:18] - mo[16:18]).max() <= 1e-6 * scale, (mg[16:18], mo[16:18])
    # field energy sums (CalcEnergy.cpp:41-120), static mesh alone and with the window
    for win in (False, True):
        eg, eo = g.field_energy(win), o.field_energy(win)
        assert np.all(eo > 0) and np.all(np.abs(eg - eo) <= 1e-12 * np.abs(eo)), (win, eg, eo)
    wg = g.wake()
    wo = o.wake(mo[:2], mo[2:4])
    assert np.array_equal(np.isnan(wg), np.isnan(wo))
    ok = ~np.isnan(wo)
    assert np.abs(wg[ok] - wo[ok]).max() <= 1e-9 * np.abs(wo[ok]).max()


def test_c1_full_size_bit_exact(gpu_lib, oracle):
    """The 2048 x 512 / 2e5-particle workload, 4 steps, against the oracle."""
    cfg, g, o = pair("c1", oracle, fields=False)
    g.step(4)
    o.step(4)
    assert_same_state(g, o)


def test_c2_full_size_bit_exact(gpu_lib, oracle):
    """The headline workload on the FP64 path: 8192 x 1024 static mesh at
    5 um, the full 4e6-particle TSC bunch, smooth random static fields so that
    every gather reads non-zero values, 2 steps (4 pushes, 8 field sub-steps,
    2 window moves) against the oracle: particles, window, static and window
    fields bit-identical."""
    cfg, g, o = pair("c2", oracle, fields=True, seed=11)
    assert len(g.particles()[0]) == 4_000_000
    g.step(2)
    o.step(2)
    assert_same_state(g, o)
    g.close()


def test_continuity_full_size(gpu_lib):
    """Deposit + charge difference of 4e6 particles (the TSC workload's
    bunch) moving for one step: residual <= 1e-10 relative."""
    cfg, spec = workload("c2")
    x, y, px, py, q = make_bunch(spec)
    h = (5e-6, 5e-6)
    dt = 0.5 * h[0] / C_LIGHT
    gam = np.sqrt(1 + px * px + py * py)
    nx, ny = x + C_LIGHT * dt * px / gam, y + 1e-3 * h[1] * np.sin(x / h[0])
    org = (x.min() - 10 * h[0], y.min() - 10 * h[1])
    ni = int((x.max() - org[0]) / h[0]) + 20
    nj = int((y.max() - org[1]) / h[1]) + 20
    bound = 4.0 * len(q) * np.abs(q).max() * C_LIGHT / (h[0] * h[1])
    scale = 2.0 ** np.floor(np.log2(2.0 ** 62 / bound))
    sf = ShapeFunction(1)
    jx = sf.getCurrentDensityBase(0, x, y, nx, ny, q, org, h, dt, 0, 0, ni, nj, scale)
    jy = sf.getCurrentDensityBase(1, x, y, nx, ny, q, org, h, dt, 0, 0, ni, nj, scale)
    rho = sf.getChargeDensityDiff(x, y, nx, ny, q, org, h, 0, 0, ni, nj, charge_scale(q))
    res = rho[1:, 1:] / dt + (jx[1:, 1:] - jx[1:, :-1]) / h[0] + (jy[1:, 1:] - jy[:-1, 1:]) / h[1]
    assert np.abs(res).max() <= 1e-10 * np.abs(rho / dt).max()


def test_deterministic_rerun(gpu_lib):
    cfg, spec = workload("small-2")
    b = make_bunch(spec)
    runs = []
    for _ in range(2):
        s = Simulation(cfg)
        s.load(*b)
        s.step(8)
        runs.append(s.particles() + s.get_static())
        s.close()
    for a, c in zip(*runs):
        assert np.array_equal(a, c)


def test_error_paths(gpu_lib):
    cfg, spec = workload("small-0")
    s = Simulation(cfg)
    with pytest.raises(CsrstError) as e:
        s.push(0)
    assert e.value.code == -4
    x, y, px, py, q = make_bunch(spec)
    x = x.copy()
    x[17] = np.nan
    with pytest.raises(CsrstError) as e:
        s.load(x, y, px, py, q)
    assert e.value.code == -1


@pytest.mark.parametrize("fp32", [False, True])
def test_rejected_bunch_keeps_the_loaded_one(gpu_lib, fp32):
    """The bunch is checked on the device after the upload: the error names
    the first rejected particle and why (non-finite values; in FP32 mode also
    a position off the static mesh), and the bunch already loaded stays in
    place and keeps stepping."""
    cfg, spec = workload("small-1")
    s = Simulation(cfg, fp32=fp32)
    bunch = make_bunch(spec)
    s.load(*bunch)
    s.step(2)
    before = s.particles()
    x, y, px, py, q = (a.copy() for a in bunch)
    q[40] = np.inf
    py[11] = np.nan
    x[25] = -1.0                      # off the static mesh
    with pytest.raises(CsrstError) as e:
        s.load(x, y, px, py, q)
    assert e.value.code == -1 and "non-finite particle data at index 11" in str(e.value)
    py[11] = 0.0
    with pytest.raises(CsrstError) as e:
        s.load(x, y, px, py, q)
    assert e.value.code == -1
    if fp32:
        assert "outside the static mesh at index 25" in str(e.value)
    else:
        assert "non-finite particle data at index 40" in str(e.value)
    for a, b in zip(s.particles(), before):
        assert np.array_equal(a, b)
    s.step(1)
    s.sync()
    s.close()


@pytest.mark.parametrize("name", ["small-0", "small-1", "small-2", "small-1-bend"])
def test_line_fields(gpu_lib, oracle, name):
    """SaveEMFieldsCommand's line samples (SaveEMFields.cpp:34-189) on the
    overlaid static mesh, for every shape order, with and without the window's
    current: positions (built from the centroid and mean momentum, whose FP64
    and long-double Kahan sums round differently) within 1e-12, fields within
    1e-12 of their magnitude."""
    cfg, g, o = pair(name, oracle)
    g.step(5)
    o.step(5)
    for cur in (False, True):
        lg, lo = g.line_fields(cur), o.line_fields(cur)
        assert lg.shape == lo.shape and lg.shape[0] > 10
        for c in (0, 5, 6):
            assert np.abs(lg[:, c] - lo[:, c]).max() <= 1e-12 * np.abs(lo[:, c]).max(), c
        for c in (1, 2, 3, 4):
            scale = np.abs(lo[:, c]).max()
            if c == 4 and not cur:
                assert scale == 0 and np.all(lg[:, c] == 0)
                continue
            assert scale > 0 and np.abs(lg[:, c] - lo[:, c]).max() <= 1e-12 * scale, (cur, c)


def test_halton_bunch_steps(gpu_lib, oracle):
    """The reference's command-line bunch (Distribution.cpp:55-163, the Halton
    round Gaussian), placed and sized for the 512 x 104 mesh, runs through the
    loop bit-identically to the oracle."""
    from csrst_b200.workloads import halton_bunch
    cfg, spec = workload("small-1")
    g = Simulation(cfg)
    info = g.info()
    bunch = halton_bunch(3000, mean_rx=spec.x0, mean_ry=spec.y0, sigma_x=40e-6, ekin_mev=cfg.ekin_mev,
                         sigma_p=1.0, qtotal_nc=1.0, origin=(info["ox"], info["oy"]), spacing=(info["hx"], info["hy"]))
    f = smooth_fields(cfg, 3)
    g.set_static(*f)
    g.load(*bunch)
    d = cfg.dict()
    d["order"] = cfg.shape_order
    d["fixed_scale"] = g.info()["fixed_scale"]
    o = oracle.Sim(d)
    o.set_static(*f)
    o.load(*bunch)
    g.step(6)
    o.step(6)
    assert_same_state(g, o)


def test_vtk_fields_match_oracle(gpu_lib, oracle, tmp_path):
    """PlotBinaryVTKCommand's two series (main.cpp:358-365) from a GPU run:
    the static piece holds the oracle's overlaid fields rounded to Float32
    (the current, whose FP64 sums may differ in the last bits, within one
    Float32 step), the window piece the oracle's window interior."""
    from csrst_b200.diagnostics import VtkSink, overlaid_fields, read_vtr, window_fields
    cfg, g, o = pair("small-1", oracle)
    g.step(5)
    o.step(5)
    d = str(tmp_path / "Data")
    a = read_vtr(VtkSink(g, directory=d).execute(1.0))
    w = read_vtr(VtkSink(g, base="mm", directory=d, source="window").execute(1.0))
    ex, ey, hz, jx, jy = overlaid_fields(o)
    (wx, wy, wh, wjx, wjy), _ = window_fields(o)
    f32 = lambda v: np.asarray(v, dtype=np.float32)
    E = a["E-Field"].reshape(cfg.Ny, cfg.Nx, 3)
    J = a["J-Field"].reshape(cfg.Ny, cfg.Nx, 3)
    assert np.array_equal(E[..., 0], f32(ex)) and np.array_equal(E[..., 1], f32(ey))
    for got, ref in ((J[..., 0], jx), (J[..., 1], jy)):         # the current: one Float32 rounding step
        assert np.abs(got - ref).max() <= 2.4e-7 * np.abs(ref).max()
    assert np.array_equal(a["H-Field"].reshape(cfg.Ny, cfg.Nx), f32(hz))
    assert np.abs(jx).max() > 0
    L1, L0 = wx.shape
    assert np.array_equal(w["E-Field"].reshape(L1, L0, 3)[..., 0], f32(wx))
    assert np.array_equal(w["H-Field"].reshape(L1, L0), f32(wh))


def test_large_window_global_accumulator(gpu_lib, oracle):
    """A window too large for the push's accumulator in shared memory (162 x
    181 cells: 235 KB of fixed-point current) takes the push variants that add
    into the window accumulator in global memory, keeping only the warp
    tiles in shared memory: the FP64 path stays bit-identical to the oracle,
    and FP32 mode (its split move + deposit launches) follows it to within
    1e-3 cells."""
    from csrst_b200.workloads import BunchSpec, bend_config
    h = 20e-6
    cfg = bend_config(2048, 512, h, 0.1, 8e-3, 1000.0, shape_order=1, cfl=0.5)
    spec = BunchSpec(n=4000, gamma=1000.0, sigma_s=400e-6, sigma_x=500e-6, energy_spread=1e-4,
                     charge=-1e-9, x0=60 * h + 5 * 400e-6, y0=0.5 * 8e-3, seed=5)
    bunch = make_bunch(spec)
    f = smooth_fields(cfg, 7)
    g = Simulation(cfg)
    g.set_static(*f)
    g.load(*bunch)
    w = g.window()[0]
    assert w[2] * w[3] * 8 > 227 * 1024
    d = cfg.dict()
    d["order"] = cfg.shape_order
    d["fixed_scale"] = g.info()["fixed_scale"]
    o = oracle.Sim(d)
    o.set_static(*f)
    o.load(*bunch)
    g.step(5)
    o.step(5)
    assert_same_state(g, o)
    s32 = Simulation(cfg, fp32=True)
    s32.set_static(*f)
    s32.load(*bunch)
    s32.step(5)
    assert s32.window()[0] == g.window()[0]
    for a, b in zip(s32.particles()[:2], g.particles()[:2]):
        assert np.abs(a - b).max() < 1e-3 * h
    s32.close()
    g.close()
