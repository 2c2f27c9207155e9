"""Host-side mirror of the reference's PIC-loop interfaces over the C ABI.

Class and method names follow the reference so that a caller of TETMSolver,
PartBunch and ScatterGatherImpl finds the same operations:

  TETMSolver.updateField_firstStep / updateField_secondStep   (TETMSolver.hh:50-70)
  PartBunch.push_particles / drift_particles / calcBeamParameters /
            getGlobalBounds                                   (PartBunch.hh:46-112)
  ScatterGatherImpl.gather                                    (ScatterGatherImpl.hh:27-64)
  ShapeFunction.getCurrentDensityBase / getChargeDensityDiff  (ShapeFunction.hh:141-508)
  moveMesh                                                    (main.cpp:562-652)
  IntegrateElong (per-step E_s samples)                       (IntegrateElong.cpp:38-89)

All state lives on the GPU in one csrst handle; nothing here computes physics.
"""
import ctypes as C

import numpy as np

from ._lib import Config, CsrstError, check, f64, lib, ptr, D

IntCIC, IntS1, IntS2 = 0, 1, 2


class Simulation:
    """Owns one csrst handle: static mesh, moving window and bunch."""

    FLAG_KEEP_OLD = 1
    FLAG_FP32 = 2
    FLAG_SUBSTEP_FIELDS = 4

    def __init__(self, cfg, keep_old=False, fp32=False, substep_fields=False):
        """fp32: FP32 mode (FP32 fields, gather, kick and positions, the
        positions as FP32 offsets from FP64 cell origins; FP32 current path
        integral with exact integer charge conservation, csrst_flux32).
        keep_old: keep the start of every particle's last move.
        substep_fields: one launch per field sub-step instead of the fused
        static sweep (the same results, bit for bit)."""
        c = Config()
        for k, v in cfg.dict().items():
            setattr(c, k, v)
        if keep_old:
            c.flags |= self.FLAG_KEEP_OLD
        if fp32:
            c.flags |= self.FLAG_FP32
        if substep_fields:
            c.flags |= self.FLAG_SUBSTEP_FIELDS
        self.fp32 = bool(c.flags & self.FLAG_FP32)
        self.cfg = cfg
        h = C.c_void_p()
        check(lib().csrst_create(C.byref(c), C.byref(h)))
        self._h = h
        self.Nx, self.Ny = cfg.Nx, cfg.Ny
        self.n = 0

    @property
    def h(self):
        if self._h is None:
            raise RuntimeError("handle destroyed")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().csrst_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, code):
        check(code, self.h)

    # -- set-up ---------------------------------------------------------------
    def info(self):
        out = np.zeros(8)
        self._ck(lib().csrst_get_info(self.h, ptr(out)))
        return dict(zip(("hx", "hy", "ox", "oy", "dt", "fixed_scale", "ncells", "wpitch"), out.tolist()))

    def geometry(self):
        inside = np.zeros(self.Nx * self.Ny, np.uint8)
        n = C.c_long()
        self._ck(lib().csrst_get_geometry(self.h, inside.ctypes.data_as(C.POINTER(C.c_uint8)), None, 0,
                                          C.byref(n)))
        cells = np.zeros((max(n.value, 1), 7))
        self._ck(lib().csrst_get_geometry(self.h, None, ptr(cells), n.value, C.byref(n)))
        return inside.reshape(self.Ny, self.Nx), cells[:n.value]

    def set_static(self, ex, ey, hzx, hzy):
        a = [f64(v).reshape(-1) for v in (ex, ey, hzx, hzy)]
        self._ck(lib().csrst_set_static_fields(self.h, *map(ptr, a)))

    def get_static(self):
        a = [np.zeros(self.Nx * self.Ny) for _ in range(4)]
        self._ck(lib().csrst_get_static_fields(self.h, *map(ptr, a)))
        return [v.reshape(self.Ny, self.Nx) for v in a]

    def reset_outside(self):
        self._ck(lib().csrst_reset_outside(self.h))

    def set_pml(self, width=10, order=4, reflection=float(np.exp(-16.0))):
        """Absorbing layers at the pipe's open ends (csrst_set_pml; the
        reference's PML_WIDTH, PML_ORD, PML_RED by default); width 0 = off,
        the reference's PEC ends."""
        self._ck(lib().csrst_set_pml(self.h, int(width), int(order), float(reflection)))

    def pml(self):
        """(number of layer cells, per row the regular sweep's columns [lo, hi))."""
        n = C.c_int()
        rows = np.zeros(2 * self.Ny, np.int32)
        self._ck(lib().csrst_get_pml(self.h, C.byref(n), rows.ctypes.data_as(C.POINTER(C.c_int))))
        return n.value, rows.reshape(self.Ny, 2)

    def load(self, x, y, px, py, q):
        a = list(map(f64, (x, y, px, py, q)))
        self.n = len(a[0])
        self._ck(lib().csrst_load_particles(self.h, *map(ptr, a), self.n))

    def initial_fields(self, tol_first=1e-12, tol_rest=1e-6, max_iter=500):
        """PoissonSolver::computeField for the loaded bunch (PoissonSolver.cpp:85-201):
        writes Ey, Hz, Ex of the static mesh and refills the window.  Returns
        {"gamma", "solves": [(iterations, relative residual)] * 3, "levels"}."""
        r = np.zeros(8)
        self._ck(lib().csrst_initial_fields(self.h, tol_first, tol_rest, int(max_iter), ptr(r)))
        return {"gamma": r[0], "solves": [(int(r[1 + 2 * k]), r[2 + 2 * k]) for k in range(3)],
                "levels": int(r[7])}

    # -- state ----------------------------------------------------------------
    def particles(self):
        a = [np.zeros(self.n) for _ in range(4)]
        self._ck(lib().csrst_get_particles(self.h, *map(ptr, a)))
        return a

    def old_positions(self):
        a = [np.zeros(self.n) for _ in range(2)]
        self._ck(lib().csrst_get_old_positions(self.h, *map(ptr, a)))
        return a

    def bunch32(self, which=0):
        """FP32 mode's bunch as stored: which=0 -> (cell, ox, oy, dpx, dpy, q),
        cells packed as i | j << 16; which=1 -> (cell, o0, o1) of the start of
        every particle's last move (keep_old)."""
        F = C.POINTER(C.c_float)
        cell = np.zeros(self.n, np.int32)
        f = [np.zeros(self.n, np.float32) for _ in range(5 if which == 0 else 2)]
        args = [cell.ctypes.data_as(C.POINTER(C.c_int))] + [v.ctypes.data_as(F) for v in f]
        args += [None] * (6 - len(args))
        self._ck(lib().csrst_get_bunch32(self.h, which, *args))
        return [cell] + f

    def window(self):
        w = (C.c_int * 4)()
        o = np.zeros(2)
        gb = (C.c_int * 4)()
        self._ck(lib().csrst_get_window(self.h, w, ptr(o), gb))
        return list(w), o, list(gb)

    def window_field(self, which):
        w, _, _ = self.window()
        out = np.zeros((w[3] + 2) * (w[2] + 2))
        self._ck(lib().csrst_get_window_field(self.h, which, ptr(out)))
        return out.reshape(w[3] + 2, w[2] + 2)

    # -- loop pieces ----------------------------------------------------------
    def push(self, jcomp):
        self._ck(lib().csrst_push(self.h, jcomp))

    def drift(self, dt):
        self._ck(lib().csrst_drift(self.h, dt))

    def half_h(self):
        self._ck(lib().csrst_half_h(self.h))

    def update_e(self, comp):
        self._ck(lib().csrst_update_e(self.h, comp))

    def move(self):
        self._ck(lib().csrst_move_window(self.h))

    def step_first(self):
        """TETMSolver::updateField_firstStep: push(Jx), half H, Ex, half H, back drift."""
        self._ck(lib().csrst_step_first(self.h))

    def step_second(self):
        """TETMSolver::updateField_secondStep: push(Jy), Ey, back drift."""
        self._ck(lib().csrst_step_second(self.h))

    def step(self, n=1):
        self._ck(lib().csrst_step(self.h, n))

    def step_timed(self):
        """One step with device times of its kernel groups (ms): push,
        fields, move, total."""
        out = np.zeros(4)
        self._ck(lib().csrst_step_timed(self.h, ptr(out)))
        return dict(zip(("push", "fields", "move", "total"), out.tolist()))

    def sync(self):
        self._ck(lib().csrst_sync(self.h))

    def stream(self):
        return lib().csrst_stream(self.h)

    # -- checkpoint / restart (the restart dump of LoadH5Part, LoadH5Part.cpp:60-321) --
    def checkpoint(self, path, step=0, time=0.0):
        """Writes everything a time step reads (fields, window, bunch) with the
        step count and time; a handle of the same configuration restored from
        the file continues bit for bit."""
        self._ck(lib().csrst_checkpoint_write(self.h, str(path).encode(), int(step), float(time)))

    def restore(self, path):
        """Replaces the state with a checkpoint written for this configuration;
        returns (step, time)."""
        st, tm = C.c_longlong(), C.c_double()
        self._ck(lib().csrst_checkpoint_read(self.h, str(path).encode(), C.byref(st), C.byref(tm)))
        n = C.c_longlong()
        self._ck(lib().csrst_get_num_particles(self.h, C.byref(n)))
        self.n = n.value
        return st.value, tm.value

    def moments(self):
        out = np.zeros(18)
        self._ck(lib().csrst_diag_moments(self.h, ptr(out)))
        return out

    def line_fields(self, with_current=False):
        """[n][7] samples along the centroid line (SaveEMFields.cpp:34-189):
        signed distance, E along / across the momentum, Hz, J along, x, y."""
        cnt = C.c_int()
        self._ck(lib().csrst_diag_line_fields(self.h, 1 if with_current else 0, None, 0, C.byref(cnt)))
        out = np.zeros((cnt.value, 7))
        self._ck(lib().csrst_diag_line_fields(self.h, 1 if with_current else 0, ptr(out), cnt.value, C.byref(cnt)))
        return out

    def field_energy(self, with_window=True):
        """{sum(Ex^2 + Ey^2), sum((Hzx + Hzy)^2)} x cell area over the static
        mesh, the window replacing the points it covers (CalcEnergy.cpp:41-120)."""
        out = np.zeros(2)
        self._ck(lib().csrst_diag_field_energy(self.h, 1 if with_window else 0, ptr(out)))
        return out

    def wake(self):
        w, _, _ = self.window()
        out = np.zeros(max(w[2] - 4, 0))
        self._ck(lib().csrst_diag_wake(self.h, ptr(out), len(out)))
        return out


class Ensemble:
    """Independent members stepped together: one launch per phase of the time
    step for all members, the step captured as one CUDA graph.  Members are
    loaded Simulations in one precision mode; each ends every step bitwise in
    the state its own step() would give."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (C.c_void_p * len(self.sims))(*[s.h.value for s in self.sims])
        e = C.c_void_p()
        rc = lib().csrst_ensemble_create(arr, len(self.sims), C.byref(e))
        if rc:
            buf = C.create_string_buffer(512)
            lib().csrst_ensemble_get_error(None, buf, 512)
            raise CsrstError(rc, buf.value.decode(errors="replace"))
        self._e = e

    def _ck(self, rc):
        if rc:
            buf = C.create_string_buffer(512)
            lib().csrst_ensemble_get_error(self._e, buf, 512)
            raise CsrstError(rc, buf.value.decode(errors="replace"))

    def step(self, n=1):
        self._ck(lib().csrst_ensemble_step(self._e, int(n)))

    def sync(self):
        bad = C.c_int(-1)
        self._ck(lib().csrst_ensemble_sync(self._e, C.byref(bad)))

    def stream(self):
        return lib().csrst_ensemble_stream(self._e)

    def set_shape(self, push_ctas, tx=0, ty=0, parts=1):
        """Launch shapes: push CTAs, field path (tx = ty = 0: the fused
        sweep; else sub-step tiles of tx x ty), parts."""
        self._ck(lib().csrst_ensemble_set_shape(self._e, int(push_ctas), int(tx), int(ty), int(parts)))

    def tune(self, steps=3):
        """Autotunes the launch shapes on real steps; returns the timing table
        [(push_ctas, tx, ty, parts, ms_per_step)] and leaves the fastest selected."""
        rows = np.zeros(5 * 64)
        n = C.c_int(0)
        self._ck(lib().csrst_ensemble_tune(self._e, int(steps), ptr(rows), 64, C.byref(n)))
        return [tuple(rows[5 * k:5 * k + 5]) for k in range(n.value)]

    def close(self):
        if getattr(self, "_e", None) is not None:
            lib().csrst_ensemble_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PartBunch:
    """PartBunch (PartBunch.hh:35-206) over a Simulation's bunch."""

    def __init__(self, sim: Simulation):
        self.sim = sim

    def push_particles(self, jcomp):
        self.sim.push(jcomp)

    def drift_particles(self, dt):
        self.sim.drift(dt)

    def getGlobalBounds(self):
        return self.sim.window()[2]

    def calcBeamParameters(self):
        m = self.sim.moments()
        keys = ("rmean", "pmean", "rrms", "prms", "eps_norm", "rmin", "rmax")
        out = {k: m[2 * i:2 * i + 2] for i, k in enumerate(keys)}
        out["Ekin"], out["dE"] = m[14], m[15]
        return out


class TETMSolver:
    """TETMSolver (TETMSolver.hh:38-103): the two half steps of one time step."""

    def __init__(self, sim: Simulation):
        self.sim = sim

    def getDT(self):
        return self.sim.info()["dt"]

    def updateField_firstStep(self):
        self.sim.step_first()

    def updateField_secondStep(self):
        self.sim.step_second()


def moveMesh(sim: Simulation):
    sim.move()


class PoissonSolver:
    """PoissonSolver (PoissonSolver.hh:47-125) over a Simulation's loaded bunch."""

    def __init__(self, sim: Simulation):
        self.sim = sim

    def computeField(self, tol=1e-12, maxIterations=500):
        """The three solves of PoissonSolver::computeField (PoissonSolver.cpp:85-201),
        the first to tol, the others to 1e-6 as the reference does (:172), then
        SCBoundaryCondition::resetOutsideDomain (main.cpp:248)."""
        return self.sim.initial_fields(tol, 1e-6, maxIterations)


class ScatterGatherImpl:
    """ScatterGatherImpl<IntOp, double> (ScatterGatherImpl.hh:27-644)."""

    def __init__(self, order):
        self.order = order

    def gather(self, patch, origin, spacing, x, y, comp):
        """comp 0/1: edge-centred component; comp 2: cell-centred field."""
        patch = f64(patch)
        x, y = f64(x), f64(y)
        out = np.zeros(len(x))
        o, hh = f64(origin), f64(spacing)
        ny, nx = patch.shape
        check(lib().csrst_gather(self.order, comp, ptr(patch), nx, ny, ptr(o), ptr(hh), ptr(x), ptr(y),
                                 len(x), ptr(out)))
        return out


class ShapeFunction:
    """ShapeFunction<IntOp> current and charge kernels (ShapeFunction.hh:141-508)."""

    def __init__(self, order):
        self.order = order

    def getCurrentDensityBase(self, comp, ox, oy, x, y, q, origin, spacing, dt, i0, j0, ni, nj, scale):
        J = np.zeros((nj, ni))
        a = list(map(f64, (ox, oy, x, y, q)))
        o, hh = f64(origin), f64(spacing)   # keep the arrays alive across the call
        check(lib().csrst_deposit(self.order, comp, *map(ptr, a), len(a[0]), ptr(o), ptr(hh), dt, i0,
                                  j0, ni, nj, scale, ptr(J)))
        return J

    def flux32(self, comp, cell0, a0, a1, cell1, b0, b1, q, scale, i0, j0, ni, nj, with_charge=False):
        """FP32 mode's deposit (csrst_flux32) of moves cell0 + a -> cell1 + b:
        the integer flux of component comp on a dense (nj, ni) patch at mesh
        index (i0, j0) and, with_charge, the integer charge change, for which
        drho + div F = 0 holds exactly."""
        I, F, Q = C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_longlong)
        i32 = lambda v: np.ascontiguousarray(v, dtype=np.int32)
        f32 = lambda v: np.ascontiguousarray(v, dtype=np.float32)
        a = [i32(cell0), f32(a0), f32(a1), i32(cell1), f32(b0), f32(b1), f32(q)]
        out = np.zeros((nj, ni), np.int64)
        rho = np.zeros((nj, ni), np.int64) if with_charge else None
        tp = [I, F, F, I, F, F, F]
        check(lib().csrst_flux32(self.order, comp, *[v.ctypes.data_as(t) for v, t in zip(a, tp)], len(a[0]),
                                 float(scale), int(i0), int(j0), int(ni), int(nj), out.ctypes.data_as(Q),
                                 rho.ctypes.data_as(Q) if with_charge else None))
        return (out, rho) if with_charge else out

    def getChargeDensityDiff(self, ox, oy, x, y, q, origin, spacing, i0, j0, ni, nj, scale):
        r = np.zeros((nj, ni))
        a = list(map(f64, (ox, oy, x, y, q)))
        o, hh = f64(origin), f64(spacing)
        check(lib().csrst_charge_diff(self.order, *map(ptr, a), len(a[0]), ptr(o), ptr(hh), i0, j0, ni,
                                      nj, scale, ptr(r)))
        return r
