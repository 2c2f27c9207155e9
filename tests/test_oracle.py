"""CPU checks of the oracle against the reference's own known answers.

test/scattergather.cpp tabulates the IntCIC / IntS1 / IntS2 scatter weights
of one particle at (3.3, 3.2) (golden file tests/golden/scattergather.json);
test/calcCurrent.cpp and test/calcCurrentS1.cpp check that the deposited
current satisfies the discrete continuity equation against the matching
charge shape.  These pin the oracle before the GPU is checked against it.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = json.loads((Path(__file__).parent / "golden" / "scattergather.json").read_text())


@pytest.mark.parametrize("name", ["CIC", "S1", "S2"])
def test_scatter_tables(oracle, name):
    t = GOLDEN["tables"][name]
    x, y = [3.3], [3.2]
    ex = oracle.scatter(t["order"], 0, (21, 21), (0, 0), (1, 1), x, y, [1.0])
    ey = oracle.scatter(t["order"], 1, (21, 21), (0, 0), (1, 1), x, y, [1.0])
    bz = oracle.scatter(t["order"], 2, (21, 21), (0, 0), (1, 1), x, y, [1.0])
    tol = GOLDEN["tolerance"]
    for i, j, a, b in t["edge"]:
        assert abs(ex[j, i] - a) < tol and abs(ey[j, i] - b) < tol, (name, i, j)
    for i, j, v in t["cell"]:
        assert abs(bz[j, i] - v) < tol, (name, i, j)
    # every listed nonzero is the whole support (weights sum to 1)
    assert abs(ex.sum() - 1) < 1e-12 and abs(ey.sum() - 1) < 1e-12 and abs(bz.sum() - 1) < 1e-12


@pytest.mark.parametrize("order", [0, 1, 2])
def test_gather_of_unit_support_is_one(oracle, order):
    # scattergather.cpp:133-166 / :218-269 / :344-416
    x, y = [3.3], [3.2]
    for comp in (0, 1, 2):
        w = oracle.scatter(order, comp, (21, 21), (0, 0), (1, 1), x, y, [1.0])
        v = oracle.gather(order, comp, (w != 0).astype(float), (0, 0), (1, 1), x, y)[0]
        assert abs(v - 1.0) < 1e-12


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("h", [(1.0, 0.5), (0.04, 0.05)])
def test_continuity(oracle, order, h):
    # calcCurrent.cpp:47-104 (dx = {1, 0.5}); calcCurrentS1.cpp:42-112 (dx = {0.04, 0.05})
    rng = np.random.default_rng(order + 7)
    n = 200
    ox = rng.uniform(5, 9, n) * h[0]
    oy = rng.uniform(5, 9, n) * h[1]
    x = ox + rng.uniform(-0.95, 0.95, n) * h[0]
    y = oy + rng.uniform(-0.95, 0.95, n) * h[1]
    q = rng.uniform(-1, 1, n)
    dt = 1.0
    jx = oracle.deposit(order, 0, ox, oy, x, y, q, (0, 0), h, dt, 0, 0, 20, 20)
    jy = oracle.deposit(order, 1, ox, oy, x, y, q, (0, 0), h, dt, 0, 0, 20, 20)
    rho = oracle.charge_diff(order, ox, oy, x, y, q, (0, 0), h, 0, 0, 20, 20)
    res = rho[1:, 1:] / dt + (jx[1:, 1:] - jx[1:, :-1]) / h[0] + (jy[1:, 1:] - jy[:-1, 1:]) / h[1]
    assert np.abs(res).max() <= 1e-10 * np.abs(rho / dt).max()


def test_reference_single_particle_continuity(oracle):
    # The exact particles of test/calcCurrent.cpp:61-66 (charge +1 moving from
    # (3.3, 3.2) to (4.2, 3.3), dx = {1, 0.5}) for the zeroth-order pair.
    h = (1.0, 0.5)
    ox, oy, x, y, q = [3.3], [3.2], [4.2], [3.3], [1.0]
    jx = oracle.deposit(0, 0, ox, oy, x, y, q, (0, 0), h, 1.0, 0, 0, 20, 20)
    jy = oracle.deposit(0, 1, ox, oy, x, y, q, (0, 0), h, 1.0, 0, 0, 20, 20)
    rho = oracle.charge_diff(0, ox, oy, x, y, q, (0, 0), h, 0, 0, 20, 20)
    res = rho[1:, 1:] + (jx[1:, 1:] - jx[1:, :-1]) / h[0] + (jy[1:, 1:] - jy[:-1, 1:]) / h[1]
    assert np.abs(res).max() < 1e-10  # SPACE_EPS, calcCurrent.cpp:90


def test_fixed_point_deposit_close_to_double(oracle):
    rng = np.random.default_rng(5)
    n = 500
    h = (1e-5, 1e-5)
    ox = rng.uniform(5, 9, n) * h[0]
    oy = rng.uniform(5, 9, n) * h[1]
    x, y = ox + 0.5 * h[0], oy + 0.1 * h[1]
    q = np.full(n, -1e-15)
    # the library's scale rule: a power of two with 4 N |q| c / (hx hy) below 2^62
    bound = 4.0 * n * 1e-15 * 299792458.0 / (h[0] * h[1])
    scale = 2.0 ** np.floor(np.log2(2.0 ** 62 / bound))
    a = oracle.deposit(1, 0, ox, oy, x, y, q, (0, 0), h, 1e-14, 0, 0, 20, 20)
    b = oracle.deposit(1, 0, ox, oy, x, y, q, (0, 0), h, 1e-14, 0, 0, 20, 20, fixed_scale=scale)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()


def test_q_rsqrt_matches_float32_restatement(oracle):
    # src/utils.hh:491-504 in numpy float32 arithmetic
    def q(x):
        x = np.float32(x)
        xh, xq = np.float32(0.5) * x, np.float32(0.5010936) * x
        i = np.array([x], np.float32).view(np.uint32)[0]
        i = np.uint32(0x5f3759df) - (i >> np.uint32(1))
        x = np.array([i], np.uint32).view(np.float32)[0]
        x = x * (np.float32(1.5) - xh * x * x)
        x = x * (np.float32(1.5010936) - xq * x * x)
        return float(x)
    for v in (1.0, 2.0, 1e6 + 1, 4e6, 123.456, 1e-3):
        assert oracle.q_rsqrt(v) == q(v)
        assert abs(oracle.q_rsqrt(v) * np.sqrt(v) - 1) < 2e-3


def test_geometry_cut_cells_are_consistent(oracle):
    from csrst_b200.workloads import workload
    cfg, _ = workload("small-0")
    inside, cells = oracle.geometry(cfg.Nx, cfg.Ny, cfg.length_before, cfg.length_after, cfg.width,
                                    cfg.phi_deg, cfg.ekin_mev, cfg.bz)
    assert inside.sum() > 0.9 * (cfg.Nx - 4) * 100  # a 2 mm pipe at 20 um is ~100 cells tall
    assert len(cells) > 2 * cfg.Nx * 0.9
    i, j = cells[:, 0].astype(int), cells[:, 1].astype(int)
    assert not inside[j, i].any()                 # cut cells are never regular cells
    assert (cells[:, 4] >= 0.5 * cells[:, 2:].max(axis=1) - 1e-15).all()  # limitArea
    # Bend::crossBoundary returns its "no crossing" value 99.9 for edges that
    # cross the wall where the straight section meets the bend; the reference
    # keeps those cells, so areas above 1 occur exactly there.
    big = cells[:, 4] > 1 + 1e-10
    assert (cells[big][:, [2, 3, 5, 6]] == 99.9).any(axis=1).all()
    order = j * cfg.Nx + i
    assert (np.diff(order) > 0).all()             # row-major, like bCellNrToLocal


def test_oracle_loop_moves_window(oracle):
    from csrst_b200.workloads import make_bunch, workload
    cfg, spec = workload("small-1")
    d = cfg.dict()
    d["order"] = cfg.shape_order
    s = oracle.Sim(d)
    s.load(*make_bunch(spec))
    w0 = s.window()[0]
    s.step(20)
    w1 = s.window()[0]
    # CFL 0.5 at beta ~ 1: the bunch moves half a cell per step
    assert w1[0] - w0[0] in (9, 10, 11)
    assert w1[2:] == w0[2:]
    x, y, px, py = s.particles()
    assert np.isfinite(x).all() and np.isfinite(px).all()


@pytest.mark.parametrize("order", [0, 1, 2])
def test_oracle_initial_fields(oracle, order):
    """The oracle's boosted electrostatic solve (PoissonSolver::computeField):
    converges on the reference's matrix, gives a relativistic field
    (Ey ~ Z0 Hz), leaves no field beyond the straight section it solves on
    and zeroes E outside the pipe (resetOutsideDomain)."""
    from csrst_b200.workloads import make_bunch, workload
    cfg, spec = workload(f"small-{order}")
    d = cfg.dict()
    d["order"] = order
    s = oracle.Sim(d)
    s.load(*make_bunch(spec))
    gamma, solves = s.initial_fields(1e-13, 1e-13, 2000)
    assert gamma == pytest.approx(1000.0, rel=1e-5)
    for it, rr in solves:
        assert rr <= 1e-13 and it < 50
    ex, ey, hx, hy = s.get_static()
    assert np.array_equal(hx, hy)                 # fillFields writes both split halves
    # Hz is solved for the bunch shifted by half a cell, so compare norms
    assert np.linalg.norm(ey) / np.linalg.norm(hx + hy) == pytest.approx(376.73, rel=0.02)
    assert np.abs(ex).max() < 1e-3 * np.abs(ey).max()   # longitudinal field suppressed by 1/gamma^2
    b = oracle.bend(cfg.Nx, cfg.Ny, cfg.length_before, cfg.length_after, cfg.width, cfg.phi_deg,
                    cfg.ekin_mev, cfg.bz)
    max_x = int(cfg.length_before / b["hx"])    # Bend::getLengthStraightSection
    for f in (ex, ey, hx):                       # no charge and no unknowns past the straight section
        assert not f[:, max_x + 1:].any()
    inside, cells = oracle.geometry(cfg.Nx, cfg.Ny, cfg.length_before, cfg.length_after, cfg.width,
                                    cfg.phi_deg, cfg.ekin_mev, cfg.bz)
    cut = np.zeros_like(inside)
    cut[cells[:, 1].astype(int), cells[:, 0].astype(int)] = 1
    outside = (inside == 0) & (cut == 0)
    assert not ex[outside].any() and not ey[outside].any()
