"""Run configurations and seeded synthetic bunches.

The reference reads its run set-up from the command line (src/main.cpp:111-136)
and builds its bunch from GSL Halton sequences (src/Distribution.cpp:55-130).
Here a configuration is derived from physical targets (grid, cell size, bend
radius, pipe width, beam energy) and the bunch comes from a seeded numpy
Philox generator; both sides of every parity check read the same arrays.
"""
import math
from dataclasses import dataclass, asdict

import numpy as np

C_LIGHT = 299792458.0
MASS_EV = 0.511e6                 # rest mass used by Bend (src/Bend.cpp:66)
M_E_GEV = 0.51099906e-03          # Physics::m_e (src/Physics.cpp:54)
CHARGE_MASS = -1e-9 / M_E_GEV     # PartBunch charge-to-mass ratio (src/main.cpp:223)


@dataclass
class RunConfig:
    Nx: int
    Ny: int
    length_before: float
    length_after: float
    width: float
    phi_deg: float
    ekin_mev: float
    bz: float
    shape_order: int = 0
    dt: float = 0.0               # <= 0: hx / c, the reference's fixed choice (main.cpp:187)
    charge_mass: float = CHARGE_MASS
    flags: int = 0

    def dict(self):
        return asdict(self)


@dataclass
class BunchSpec:
    n: int
    gamma: float
    sigma_s: float                # rms length (x) [m]
    sigma_x: float                # rms width (y) [m]
    energy_spread: float          # relative rms of gamma
    charge: float                 # total charge [C], negative for electrons
    x0: float                     # centroid x [m]
    y0: float                     # centroid y [m]
    seed: int = 1


def bend_config(Nx, Ny, h, R, width, gamma, shape_order=0, cfl=None, length_after=None):
    """Chooses the bend angle and the drift before the bend so that the
    reference's domain rule (Bend::Init, src/Bend.cpp:92-105) gives cells of
    size h on an Nx x Ny mesh.  The drift after the bend defaults to 50
    cells: the reference's wall crossing (Bend::crossBoundary) finds the end
    wall only in the straight section after the bend, so a zero-length drift
    there makes its cut-cell areas assert."""
    if length_after is None:
        length_after = 50 * h
    ekin_mev = (gamma - 1.0) * MASS_EV * 1e-6
    ekin = ekin_mev * 1e6
    p_ev = math.sqrt(ekin * ekin + 2.0 * ekin * MASS_EV)
    bz = p_ev / (C_LIGHT * R)
    dom_w = (Ny - 2) * h
    if dom_w <= width:
        raise ValueError("the mesh must be taller than the pipe")

    def width_of(phi):
        return (R - 0.5 * width) * (1 - math.cos(phi)) + width + length_after * math.sin(phi)

    lo, hi = 0.0, 0.5 * math.pi
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if width_of(mid) < dom_w else (lo, mid)
    phi = 0.5 * (lo + hi)
    lb = (Nx - 2) * h - length_after * math.cos(phi) - (R + 0.5 * width) * math.sin(phi)
    if lb <= 0:
        raise ValueError("mesh too short for this bend")
    dt = 0.0 if cfl is None else cfl * h / C_LIGHT
    return RunConfig(Nx=Nx, Ny=Ny, length_before=lb, length_after=length_after, width=width,
                     phi_deg=math.degrees(phi), ekin_mev=ekin_mev, bz=bz,
                     shape_order=shape_order, dt=dt)


def make_bunch(spec: BunchSpec):
    """Gaussian bunch: x ~ N(x0, sigma_s), y ~ N(y0, sigma_x),
    gamma_i = gamma (1 + N(0, spread)), P = (beta gamma, 0)."""
    g = np.random.Generator(np.random.Philox(spec.seed))
    x = spec.x0 + spec.sigma_s * g.standard_normal(spec.n)
    y = spec.y0 + spec.sigma_x * g.standard_normal(spec.n)
    gam = spec.gamma * (1.0 + spec.energy_spread * g.standard_normal(spec.n))
    px = np.sqrt(gam * gam - 1.0)
    py = np.zeros(spec.n)
    q = np.full(spec.n, spec.charge / spec.n)
    return x, y, px, py, q


# Named workloads.  C1/C2 follow the reference's headline configurations;
# the "small" ones are the same physics on meshes the CPU oracle runs in
# seconds.
def workload(name):
    if name in ("c1", "c1-bend"):  # 2048 x 512, h = 10 um, R = 1 m, 5 mm pipe, CIC, CFL 0.5, 2e5 particles
        # "-bend": the bunch starts at the dipole entrance (6 sigma_s into the
        # arc), so that its steps run through the dipole
        h = 10e-6
        cfg = bend_config(2048, 512, h, 1.0, 5e-3, 1000.0, shape_order=0, cfl=0.5)
        x0 = cfg.length_before + 6 * 50e-6 if name == "c1-bend" else 50 * h + 6 * 50e-6
        spec = BunchSpec(n=200_000, gamma=1000.0, sigma_s=50e-6, sigma_x=20e-6,
                         energy_spread=1e-4, charge=-1e-9, x0=x0,
                         y0=0.5 * 5e-3, seed=11)
    elif name == "c2":    # 8192 x 1024, h = 5 um, TSC, 4e6 particles
        h = 5e-6
        cfg = bend_config(8192, 1024, h, 1.0, 5e-3, 1000.0, shape_order=1, cfl=0.5)
        spec = BunchSpec(n=4_000_000, gamma=1000.0, sigma_s=50e-6, sigma_x=20e-6,
                         energy_spread=1e-4, charge=-1e-9, x0=50 * h + 6 * 50e-6,
                         y0=0.5 * 5e-3, seed=12)
    elif name.startswith("small"):
        # small-<order>[-bend]: 512 x 104 mesh at 20 um, 2 mm pipe, R = 0.25 m,
        # 4000 particles; "-bend" starts the bunch at the dipole entrance.
        parts = name.split("-")
        order = int(parts[1]) if len(parts) > 1 else 0
        h = 20e-6
        cfg = bend_config(512, 104, h, 0.25, 2e-3, 1000.0, shape_order=order, cfl=0.5)
        x0 = 40 * h + 6 * 60e-6
        if "bend" in parts:
            x0 = cfg.length_before + 6 * 60e-6
        spec = BunchSpec(n=4000, gamma=1000.0, sigma_s=60e-6, sigma_x=40e-6,
                         energy_spread=1e-4, charge=-1e-9, x0=x0, y0=0.5 * 2e-3, seed=3)
    else:
        raise KeyError(name)
    return cfg, spec


def bend_config_fit(Nx, Ny, h, R, width, gamma, lb_min, shape_order=0, cfl=0.5, length_after=None):
    """A bend on an Nx x Ny mesh of square cells h with a drift of at least
    lb_min before it: the bend angle is the largest that fits both the mesh
    height with a pipe of `width` and the mesh length; when the length limits
    it, the pipe is widened until the bend fills the mesh height again."""
    if length_after is None:
        length_after = 50 * h
    ekin_mev = (gamma - 1.0) * MASS_EV * 1e-6
    ekin = ekin_mev * 1e6
    bz = math.sqrt(ekin * ekin + 2.0 * ekin * MASS_EV) / (C_LIGHT * R)
    dom_l, dom_w = (Nx - 2) * h, (Ny - 2) * h
    if dom_w <= width or dom_l <= lb_min + length_after:
        raise ValueError("mesh too small for this bend")

    def width_of(phi, w):
        return (R - 0.5 * w) * (1 - math.cos(phi)) + w + length_after * math.sin(phi)

    def length_of(phi, w):
        return lb_min + length_after * math.cos(phi) + (R + 0.5 * w) * math.sin(phi)

    def fill(phi):  # pipe width that makes the bounding box exactly (Ny - 2) h tall
        c, sn = math.cos(phi), math.sin(phi)
        return (dom_w - R * (1 - c) - length_after * sn) / (1 - 0.5 * (1 - c))

    lo, hi = 0.0, 0.5 * math.pi
    for _ in range(200):  # largest angle the height allows with the narrowest pipe
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if width_of(mid, width) < dom_w else (lo, mid)
    lo, hi = 0.0, lo
    for _ in range(200):  # then the largest that also fits the length with the filling pipe
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if length_of(mid, fill(mid)) < dom_l else (lo, mid)
    phi = lo
    c, sn = math.cos(phi), math.sin(phi)
    width = fill(phi)
    lb = dom_l - length_after * c - (R + 0.5 * width) * sn
    if lb < lb_min or width > 0.75 * dom_w:
        raise ValueError("mesh too small for this bend")
    return RunConfig(Nx=Nx, Ny=Ny, length_before=lb, length_after=length_after, width=width,
                     phi_deg=math.degrees(phi), ekin_mev=ekin_mev, bz=bz, shape_order=shape_order,
                     dt=cfl * h / C_LIGHT)


def ensemble_members(m=64, seed=2024):
    """The batched-ensemble workload: m independent bunches with uneven
    meshes and bunch sizes.  Nx ~ U[1024, 8192], Ny ~ U[256, 1024],
    sigma_s log-uniform in [20, 200] um, sigma_x = sigma_s / 2.5, gamma ~
    U[200, 2000], bend radius ~ U[0.5, 5] m, 5e4 - 1e6 particles, CIC and TSC
    alternating, CFL 0.5.  Cells are sigma_s / 10, made coarser in steps of
    1.25 until the bend fits the drawn mesh (bend_config_fit; the pipe is 60 -
    85 % of the mesh height)."""
    g = np.random.Generator(np.random.Philox(seed))
    out = []
    while len(out) < m:
        k = len(out)
        Nx = int(g.integers(1024, 8193))
        Ny = int(g.integers(256, 1025))
        sigma_s = float(np.exp(g.uniform(np.log(20e-6), np.log(200e-6))))
        gamma = float(g.uniform(200.0, 2000.0))
        R = float(g.uniform(0.5, 5.0))
        n = int(g.integers(50_000, 1_000_001))
        cfg = None
        for t in range(12):  # cells of sigma_s / 10, coarser until the bend fits the mesh
            h = sigma_s / 10 * 1.25 ** t
            width = 0.6 * (Ny - 2) * h
            x0 = 50 * h + 6 * sigma_s
            try:
                cfg = bend_config_fit(Nx, Ny, h, R, width, gamma, x0 + 30 * sigma_s, shape_order=k % 2)
                break
            except ValueError:
                continue
        if cfg is None:
            continue
        spec = BunchSpec(n=n, gamma=gamma, sigma_s=sigma_s, sigma_x=sigma_s / 2.5, energy_spread=1e-4,
                         charge=-1e-9, x0=x0, y0=0.5 * width, seed=1000 + k)
        out.append((cfg, spec))
    return out


# ---- the reference's own initial distribution (src/Distribution.cpp:55-163) ----

M_E_MEV = M_E_GEV * 1e3       # Distribution.cpp:26: MASS = Physics::m_e * 1e3


def radical_inverse(n, base):
    """Van der Corput radical inverse of the integers n in `base` (the
    published Halton construction): digits of n mirrored about the point,
    accumulated most significant first as v /= base; r += v * digit."""
    x = np.asarray(n, dtype=np.int64).copy()
    r = np.zeros(x.shape)
    v = np.ones(x.shape)
    while np.any(x > 0):
        m = x > 0
        v[m] /= base
        r[m] += v[m] * (x[m] % base)
        x[m] //= base
    return r


def halton_bunch(n=50000, mean_rx=0.05, mean_ry=0.0, sigma_x=0.01, ekin_mev=250.0, sigma_p=1.0, qtotal_nc=-1.0,
                 origin=(0.0, 0.0), spacing=(1.0, 1.0)):
    """The bunch the reference builds from its command line (Distribution.cpp:55-131 and gaussian2DSample :145-153;
    defaults from main.cpp:126-133): point k (k = 1 .. n) of the 2D Halton
    sequence (bases 2, 3) becomes a round Gaussian sample by Box-Muller,
    sigma sqrt(-2 ln v0) (cos, sin)(2 pi v1).  Positions and momentum offsets
    come from two generators of the same sequence, so they are proportional
    point by point; momenta are (sqrt(gamma^2 - 1), 0) + offset with gamma =
    Ekin / m_e + 1; charges -Qtotal 1e-9 / n each.  Then the positions alone
    are sorted by mesh row (truncated, Utils::XFirst, utils.hh:116-142) and x
    — which, as in the reference, unpairs them from the momenta.  Returns
    (x, y, px, py, q).  GSL is not available here: the sequence is the
    published construction, checked against scipy's, not against GSL itself."""
    k = np.arange(1, n + 1)
    v0, v1 = radical_inverse(k, 2), radical_inverse(k, 3)
    r = np.sqrt(-2.0 * np.log(v0))
    a = 2.0 * math.pi * v1
    c, s_ = np.cos(a), np.sin(a)
    x, y = mean_rx + sigma_x * r * c, mean_ry + sigma_x * r * s_
    gamma = ekin_mev / M_E_MEV + 1.0
    px, py = math.sqrt(gamma * gamma - 1.0) + sigma_p * r * c, sigma_p * r * s_
    row = np.trunc((y - origin[1]) / spacing[1]).astype(np.int64)
    order = np.lexsort((x, row))
    q = np.full(n, -qtotal_nc * 1e-9 / n)
    return x[order], y[order], px, py, q
