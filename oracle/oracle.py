"""ctypes binding of the CPU oracle (oracle/csrst_oracle.cpp).

Test infrastructure only: tests/, __graft_entry__.smoke() and the CPU legs of
bench.py use it as the checker.  The product package never imports it.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None

D = C.POINTER(C.c_double)
U8 = C.POINTER(C.c_uint8)
I = C.POINTER(C.c_int)


class OrcConfig(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("order", C.c_int), ("fixed_point", C.c_int),
                ("length_before", C.c_double), ("length_after", C.c_double),
                ("width", C.c_double), ("phi_deg", C.c_double), ("ekin_mev", C.c_double),
                ("bz", C.c_double), ("dt", C.c_double), ("charge_mass", C.c_double),
                ("fixed_scale", C.c_double)]


def build():
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _LIB
    if _LIB is None:
        so = _HERE / "libcsrst_oracle.so"
        if not so.exists():
            build()
        L = C.CDLL(str(so))
        L.orc_q_rsqrt.restype = C.c_float
        L.orc_q_rsqrt.argtypes = [C.c_float]
        L.orc_bend.argtypes = [C.c_int, C.c_int] + [C.c_double] * 6 + [D]
        L.orc_crossings.restype = C.c_long
        L.orc_crossings.argtypes = [C.c_int] + [C.c_double] * 8 + [D, D, D]
        L.orc_geometry.restype = C.c_long
        L.orc_geometry.argtypes = [C.c_int, C.c_int] + [C.c_double] * 6 + [U8, D, C.c_long]
        L.orc_gather.argtypes = [C.c_int, C.c_int, D, C.c_int, C.c_int] + [C.c_double] * 4 + [D, D, C.c_long, D]
        L.orc_scatter.argtypes = [C.c_int, C.c_int, D, C.c_int, C.c_int] + [C.c_double] * 4 + [D, D, D, C.c_long]
        L.orc_deposit.argtypes = ([C.c_int, C.c_int, D, D, D, D, D, C.c_long] + [C.c_double] * 5 +
                                  [C.c_int] * 4 + [D, C.c_int, C.c_double])
        L.orc_charge_diff.argtypes = ([C.c_int, D, D, D, D, D, C.c_long] + [C.c_double] * 4 +
                                      [C.c_int] * 4 + [D])
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcConfig)]
        for f in ("orc_destroy",):
            getattr(L, f).argtypes = [C.c_void_p]
        L.orc_error.argtypes = [C.c_void_p]
        L.orc_dt.restype = C.c_double
        L.orc_dt.argtypes = [C.c_void_p]
        L.orc_set_static.argtypes = [C.c_void_p, D, D, D, D]
        L.orc_get_static.argtypes = [C.c_void_p, D, D, D, D]
        L.orc_reset_outside.argtypes = [C.c_void_p]
        L.orc_load.argtypes = [C.c_void_p, D, D, D, D, D, C.c_long]
        L.orc_get_particles.argtypes = [C.c_void_p, D, D, D, D]
        L.orc_get_old.argtypes = [C.c_void_p, D, D]
        L.orc_get_window.argtypes = [C.c_void_p, I, D, I]
        L.orc_get_window_field.argtypes = [C.c_void_p, C.c_int, D]
        L.orc_push.argtypes = [C.c_void_p, C.c_int]
        L.orc_drift.argtypes = [C.c_void_p, C.c_double]
        L.orc_half_h.argtypes = [C.c_void_p]
        L.orc_set_pml.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
        L.orc_pml_cells.argtypes = [C.c_void_p]
        L.orc_update_e.argtypes = [C.c_void_p, C.c_int]
        L.orc_move.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_wake.argtypes = [C.c_void_p] + [C.c_double] * 4 + [D]
        L.orc_moments.argtypes = [C.c_void_p, D]
        L.orc_field_energy.argtypes = [C.c_void_p, C.c_int, D]
        L.orc_line_fields.argtypes = [C.c_void_p, C.c_int, D, C.c_int, C.POINTER(C.c_int)]
        L.orc_initial_fields.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, D]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(D)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def q_rsqrt(x):
    return lib().orc_q_rsqrt(float(x))


def crossings(dual, old, new, spacing, origin):
    """(fractions, points[n][2]) of the crossing split of one move."""
    fr, s0, s1 = np.zeros(32), np.zeros(32), np.zeros(32)
    n = lib().orc_crossings(1 if dual else 0, old[0], old[1], new[0], new[1], spacing[0], spacing[1], origin[0],
                            origin[1], _p(fr), _p(s0), _p(s1))
    return fr[:n], np.stack([s0[:n], s1[:n]], axis=1)


def bend(Nx, Ny, Lb, La, w, phi_deg, ekin, bz):
    out = np.zeros(8)
    lib().orc_bend(Nx, Ny, Lb, La, w, phi_deg, ekin, bz, _p(out))
    return dict(zip(("hx", "hy", "ox", "oy", "cx", "cy", "R", "phi"), out.tolist()))


def geometry(Nx, Ny, Lb, La, w, phi_deg, ekin, bz, max_cells=None):
    inside = np.zeros(Nx * Ny, np.uint8)
    max_cells = max_cells or 8 * (Nx + Ny) + 64
    cells = np.zeros((max_cells, 7))
    n = lib().orc_geometry(Nx, Ny, Lb, La, w, phi_deg, ekin, bz,
                           inside.ctypes.data_as(U8), _p(cells), max_cells)
    if n < 0:
        raise RuntimeError(f"geometry aborted ({n})")
    return inside.reshape(Ny, Nx), cells[:n].copy()


def gather(order, comp, patch, origin, spacing, x, y):
    patch = f64(patch)
    x, y = f64(x), f64(y)
    out = np.zeros(len(x))
    ny, nx = patch.shape
    lib().orc_gather(order, comp, _p(patch), nx, ny, origin[0], origin[1], spacing[0], spacing[1],
                     _p(x), _p(y), len(x), _p(out))
    return out


def scatter(order, comp, shape, origin, spacing, x, y, val):
    patch = np.zeros(shape)
    x, y, val = f64(x), f64(y), f64(val)
    lib().orc_scatter(order, comp, _p(patch), shape[1], shape[0], origin[0], origin[1],
                      spacing[0], spacing[1], _p(x), _p(y), _p(val), len(x))
    return patch


def deposit(order, comp, ox, oy, x, y, q, origin, spacing, dt, i0, j0, ni, nj,
            fixed_scale=0.0):
    J = np.zeros((nj, ni))
    ox, oy, x, y, q = map(f64, (ox, oy, x, y, q))
    lib().orc_deposit(order, comp, _p(ox), _p(oy), _p(x), _p(y), _p(q), len(x), origin[0],
                      origin[1], spacing[0], spacing[1], dt, i0, j0, ni, nj, _p(J),
                      1 if fixed_scale else 0, float(fixed_scale))
    return J


def charge_diff(order, ox, oy, x, y, q, origin, spacing, i0, j0, ni, nj):
    r = np.zeros((nj, ni))
    ox, oy, x, y, q = map(f64, (ox, oy, x, y, q))
    lib().orc_charge_diff(order, _p(ox), _p(oy), _p(x), _p(y), _p(q), len(x), origin[0],
                          origin[1], spacing[0], spacing[1], i0, j0, ni, nj, _p(r))
    return r


class Sim:
    """Whole-loop oracle: static mesh + moving window + bunch."""

    def __init__(self, cfg):
        c = OrcConfig()
        c.Nx, c.Ny, c.order = cfg["Nx"], cfg["Ny"], cfg.get("order", 0)
        c.fixed_point = 1 if cfg.get("fixed_scale") else 0
        c.fixed_scale = float(cfg.get("fixed_scale") or 0.0)
        c.length_before, c.length_after = cfg["length_before"], cfg["length_after"]
        c.width, c.phi_deg, c.ekin_mev, c.bz = cfg["width"], cfg["phi_deg"], cfg["ekin_mev"], cfg["bz"]
        c.dt = cfg.get("dt", 0.0)
        c.charge_mass = cfg["charge_mass"]
        self.cfg = cfg
        self.Nx, self.Ny = c.Nx, c.Ny
        self.h = lib().orc_create(C.byref(c))
        if lib().orc_error(self.h):
            raise RuntimeError(f"oracle geometry error {lib().orc_error(self.h)}")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    @property
    def dt(self):
        return lib().orc_dt(self.h)

    def set_static(self, ex, ey, hx, hy):
        a = [f64(v).reshape(-1) for v in (ex, ey, hx, hy)]
        lib().orc_set_static(self.h, *map(_p, a))

    def get_static(self):
        a = [np.zeros(self.Nx * self.Ny) for _ in range(4)]
        lib().orc_get_static(self.h, *map(_p, a))
        return [v.reshape(self.Ny, self.Nx) for v in a]

    def reset_outside(self):
        lib().orc_reset_outside(self.h)

    def load(self, x, y, px, py, q):
        a = list(map(f64, (x, y, px, py, q)))
        self.n = len(a[0])
        rc = lib().orc_load(self.h, *map(_p, a), self.n)
        if rc:
            raise RuntimeError(f"oracle load error {rc}")

    def particles(self):
        a = [np.zeros(self.n) for _ in range(4)]
        lib().orc_get_particles(self.h, *map(_p, a))
        return a

    def old_positions(self):
        a = [np.zeros(self.n) for _ in range(2)]
        lib().orc_get_old(self.h, *map(_p, a))
        return a

    def window(self):
        w = (C.c_int * 4)()
        o = np.zeros(2)
        gb = (C.c_int * 4)()
        lib().orc_get_window(self.h, w, _p(o), gb)
        return list(w), o, list(gb)

    def window_field(self, which):
        w, _, _ = self.window()
        out = np.zeros((w[3] + 2) * (w[2] + 2))
        lib().orc_get_window_field(self.h, which, _p(out))
        return out.reshape(w[3] + 2, w[2] + 2)

    def push(self, jcomp):
        lib().orc_push(self.h, jcomp)

    def drift(self, dt):
        lib().orc_drift(self.h, dt)

    def set_pml(self, width=10, order=4, reflection=float(np.exp(-16.0))):
        lib().orc_set_pml(self.h, int(width), int(order), float(reflection))

    def pml_cells(self):
        return int(lib().orc_pml_cells(self.h))

    def half_h(self):
        lib().orc_half_h(self.h)

    def update_e(self, comp):
        lib().orc_update_e(self.h, comp)

    def move(self):
        return lib().orc_move(self.h)

    def step(self, n=1):
        rc = lib().orc_step(self.h, n)
        if rc:
            raise RuntimeError(f"oracle step error {rc}")

    def moments(self):
        out = np.zeros(18)
        lib().orc_moments(self.h, _p(out))
        return out

    def line_fields(self, with_current=False):
        cnt = C.c_int()
        lib().orc_line_fields(self.h, 1 if with_current else 0, None, 0, C.byref(cnt))
        out = np.zeros((cnt.value, 7))
        lib().orc_line_fields(self.h, 1 if with_current else 0, _p(out), cnt.value, C.byref(cnt))
        return out

    def field_energy(self, with_window=True):
        out = np.zeros(2)
        lib().orc_field_energy(self.h, 1 if with_window else 0, _p(out))
        return out

    def wake(self, rmean, pmean):
        w, _, _ = self.window()
        out = np.zeros(max(w[2] - 4, 0))
        lib().orc_wake(self.h, rmean[0], rmean[1], pmean[0], pmean[1], _p(out))
        return out

    def initial_fields(self, tol_first=1e-12, tol_rest=1e-6, maxit=500):
        """Boosted electrostatic initial fields of the loaded bunch; returns
        (gamma, [(iterations, relative residual)] * 3)."""
        st = np.zeros(7)
        rc = lib().orc_initial_fields(self.h, tol_first, tol_rest, maxit, _p(st))
        if rc:
            raise RuntimeError(f"oracle initial fields error {rc}")
        return st[0], [(int(st[1 + 2 * k]), st[2 + 2 * k]) for k in range(3)]
