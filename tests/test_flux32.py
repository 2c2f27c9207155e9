"""FP32 mode's charge-conserving deposit (csrst_b200/csrc/flux32.cuh) on the
CPU: the same header compiled for the host (tests/cpp/flux32_host.cpp).

For random moves of up to one cell per axis (start offsets outside the start
cell included, as after the pending -dt/2 drift), every shape order:
 * continuity holds exactly in integers: drho + div F = 0 at every vertex;
 * the current equals the oracle's FP64 restatement of the reference's path
   integral (ShapeFunction getCurrentDensityBase) to FP32 accuracy:
   Jx within 1e-7 and Jy within 2e-6 of their maxima;
 * the charge each particle carries equals the oracle's FP64 charge shape
   (getChargeDensityDiff) to 1e-12 of its maximum."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
C_LIGHT = 299792458.0


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    so = tmp_path_factory.mktemp("flux32") / "flux32_host.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC",
                    str(ROOT / "tests/cpp/flux32_host.cpp"), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    I, F, Q = C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_longlong)
    L.flux32_host.argtypes = [C.c_int, C.c_int, I, F, F, I, F, F, F, C.c_long, C.c_double, C.c_int, C.c_int,
                              C.c_int, C.c_int, Q, Q, C.c_int]
    L.flux32_host.restype = C.c_int
    return L


def random_moves(n, seed, cfl=0.9):
    """Start cell + offset (offsets in [-0.3, 1): a pending drift can put the
    start in the cell before), a move of up to `cfl` cells along x and 0.3
    across, end stored as cell + FP32 offset in [0, 1)."""
    rng = np.random.default_rng(seed)
    ci = rng.integers(10, 30, n)
    cj = rng.integers(10, 30, n)
    a0 = rng.uniform(-0.3, 1.0, n).astype(np.float32)
    a1 = rng.uniform(0.0, 1.0, n).astype(np.float32)
    ang = rng.uniform(-np.pi, np.pi, n)
    r = rng.uniform(0, 1, n)
    d0 = (cfl * r * np.cos(ang)).astype(np.float32)
    d1 = (0.3 * r * np.sin(ang)).astype(np.float32)
    d1[: n // 4] = 0.0                       # straight along x
    d0[n // 4: n // 3] = 0.0                 # straight along y
    e0 = (a0 + d0).astype(np.float32)
    e1 = (a1 + d1).astype(np.float32)
    f0, f1 = np.floor(e0), np.floor(e1)
    b0 = (e0 - f0).astype(np.float32)
    b1 = (e1 - f1).astype(np.float32)
    up0, up1 = b0 >= 1.0, b1 >= 1.0
    b0[up0] = 0.0
    b1[up1] = 0.0
    ni = ci + f0.astype(np.int64) + up0
    nj = cj + f1.astype(np.int64) + up1
    q = rng.uniform(-2e-15, -1e-15, n).astype(np.float32)
    pack = lambda i, j: (i | (j << 16)).astype(np.int32)
    return pack(ci, cj), a0, a1, pack(ni, nj), b0, b1, q, (ci, cj, ni, nj)


def flux(host, order, comp, mv, scale, ni=48, nj=48, drho=False, fast=True):
    c0, a0, a1, c1, b0, b1, q, _ = mv
    F = np.zeros((nj, ni), dtype=np.int64)
    R = np.zeros((nj, ni), dtype=np.int64) if drho else None
    P = lambda a, t: np.ascontiguousarray(a).ctypes.data_as(C.POINTER(t))
    rc = host.flux32_host(order, comp, P(c0, C.c_int), P(a0, C.c_float), P(a1, C.c_float), P(c1, C.c_int),
                          P(b0, C.c_float), P(b1, C.c_float), P(q, C.c_float), len(q), scale, 0, 0, ni, nj,
                          F.ctypes.data_as(C.POINTER(C.c_longlong)),
                          R.ctypes.data_as(C.POINTER(C.c_longlong)) if drho else None, 1 if fast else 0)
    assert rc == 0
    return F, R


def flux_scale(q):
    return 2.0 ** np.floor(np.log2(2.0 ** 62 / (4.0 * len(q) * np.abs(q.astype(np.float64)).max())))


@pytest.mark.parametrize("order", [0, 1, 2])
def test_flux32_exact_continuity(host, order):
    mv = random_moves(20000, 5 + order)
    scale = flux_scale(mv[6])
    fx, rho = flux(host, order, 0, mv, scale, drho=True)
    fy, _ = flux(host, order, 1, mv, scale)
    res = rho[1:, 1:] + (fx[1:, 1:] - fx[1:, :-1]) + (fy[1:, 1:] - fy[:-1, 1:])
    assert np.abs(rho).max() > 0 and np.abs(fx).max() > 0 and np.abs(fy).max() > 0
    assert (res == 0).all()
    # nothing outside the region the moves reach (no current leaks past a stencil box)
    assert (fx[:, :6] == 0).all() and (fx[:, 34:] == 0).all()


@pytest.mark.parametrize("order", [0, 1, 2])
def test_flux32_matches_fp64_reference_current(host, oracle, order):
    h = (1e-5, 1.2e-5)
    dt = 0.5 * h[0] / C_LIGHT
    mv = random_moves(20000, 17 + order)
    c0, a0, a1, c1, b0, b1, q, (ci, cj, ni, nj) = mv
    scale = flux_scale(q)
    fx, rho = flux(host, order, 0, mv, scale, drho=True)
    fy, _ = flux(host, order, 1, mv, scale)
    ox = (ci + a0.astype(np.float64)) * h[0]
    oy = (cj + a1.astype(np.float64)) * h[1]
    x = (ni + b0.astype(np.float64)) * h[0]
    y = (nj + b1.astype(np.float64)) * h[1]
    q64 = q.astype(np.float64)
    jx = oracle.deposit(order, 0, ox, oy, x, y, q64, (0, 0), h, dt, 0, 0, 48, 48)
    jy = oracle.deposit(order, 1, ox, oy, x, y, q64, (0, 0), h, dt, 0, 0, 48, 48)
    ref_rho = oracle.charge_diff(order, ox, oy, x, y, q64, (0, 0), h, 0, 0, 48, 48)
    # flux units -> current density and charge density
    jx32 = fx / (scale * dt * h[1])
    jy32 = fy / (scale * dt * h[0])
    rho32 = rho / (scale * h[0] * h[1])
    assert np.abs(jx32 - jx).max() <= 1e-7 * np.abs(jx).max()
    assert np.abs(jy32 - jy).max() <= 2e-6 * np.abs(jy).max()
    assert np.abs(rho32 - ref_rho).max() <= 1e-12 * np.abs(ref_rho).max()


@pytest.mark.parametrize("order", [0, 1, 2])
def test_flux32_compact_form_is_bit_identical(host, order):
    """The compact form the push takes for moves that keep their y base index
    and advance x by at most one gives the same integers as the general form."""
    mv = random_moves(20000, 31 + order, cfl=0.6)
    scale = flux_scale(mv[6])
    for comp in (0, 1):
        a, ra = flux(host, order, comp, mv, scale, drho=True, fast=True)
        b, rb = flux(host, order, comp, mv, scale, drho=True, fast=False)
        assert np.array_equal(a, b) and np.array_equal(ra, rb)


def test_flux32_rejects_moves_of_more_than_one_cell(host):
    mv = list(random_moves(100, 3))
    c0, c1 = mv[0].copy(), mv[3].copy()
    c1[7] = c0[7] + 2                        # two cells along x
    mv[3] = c1
    F = np.zeros((48, 48), dtype=np.int64)
    P = lambda a, t: np.ascontiguousarray(a).ctypes.data_as(C.POINTER(t))
    rc = host.flux32_host(1, 0, P(mv[0], C.c_int), P(mv[1], C.c_float), P(mv[2], C.c_float), P(mv[3], C.c_int),
                          P(mv[4], C.c_float), P(mv[5], C.c_float), P(mv[6], C.c_float), 100, 2.0 ** 40, 0, 0, 48,
                          48, F.ctypes.data_as(C.POINTER(C.c_longlong)), None, 0)
    assert rc & 1
