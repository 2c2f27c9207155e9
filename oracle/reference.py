"""ctypes binding of the reference's own code compiled here (oracle/_ref,
`make -C oracle ref`): the crossing split and Q_rsqrt of src/utils.hh, the
current deposits of src/*OrderShapeFunction.cpp and the gathers of
src/FieldPatch.hh + src/ScatterGatherImpl.hh (see oracle/ref_driver.cpp).

Test infrastructure: it checks the oracle against the reference and makes
the committed golden vectors (tests/golden/make_reference_vectors.py).
available() is False when neither a built library nor the reference
sources are present (the GPU box has only what was built here)."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
SO = _HERE / "_ref" / "libcsrst_ref.so"
REF = Path("/root/reference")
_LIB = None
D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int)


def available():
    return SO.exists() or (REF / "src" / "FirstOrderShapeFunction.cpp").exists()


def lib():
    global _LIB
    if _LIB is None:
        if not SO.exists():
            subprocess.run(["make", "-s", "-C", str(_HERE), "ref", f"REF={REF}"], check=True)
        L = C.CDLL(str(SO))
        L.ref_q_rsqrt.restype = C.c_float
        L.ref_q_rsqrt.argtypes = [C.c_float]
        L.ref_crossings.restype = C.c_long
        L.ref_crossings.argtypes = [C.c_int] + [C.c_double] * 8 + [D, D, D]
        L.ref_deposit.restype = C.c_int
        L.ref_deposit.argtypes = [C.c_int, C.c_int, D, D, D, D, D, C.c_long] + [C.c_double] * 5 + [C.c_int] * 4 + [D, I]
        L.ref_gather.restype = C.c_int
        L.ref_gather.argtypes = [C.c_int, C.c_int, D, C.c_int, C.c_int] + [C.c_double] * 4 + [D, D, C.c_long, D]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(D)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def q_rsqrt(x):
    return float(lib().ref_q_rsqrt(float(x)))


def crossings(dual, old, new, spacing, origin):
    """(fractions, points[n][2]) of Utils::calc(Dual)CellBorderCrossings."""
    fr, s0, s1 = np.zeros(32), np.zeros(32), np.zeros(32)
    n = lib().ref_crossings(1 if dual else 0, old[0], old[1], new[0], new[1], spacing[0], spacing[1], origin[0],
                            origin[1], _p(fr), _p(s0), _p(s1))
    return fr[:n], np.stack([s0[:n], s1[:n]], axis=1)


def deposit(order, comp, ox, oy, x, y, q, origin, spacing, dt, i0, j0, ni, nj):
    """getCurrentDensityBaseImplX/Y on a dense (nj, ni) patch at (i0, j0);
    returns (J, the reference's own patch domain (i_first, i_last, j_first,
    j_last), whether its patch index check failed)."""
    J = np.zeros((nj, ni))
    dom = np.zeros(4, np.int32)
    a = list(map(f64, (ox, oy, x, y, q)))
    rc = lib().ref_deposit(order, comp, *map(_p, a), len(a[0]), origin[0], origin[1], spacing[0], spacing[1], dt,
                           i0, j0, ni, nj, _p(J), dom.ctypes.data_as(I))
    return J, tuple(int(v) for v in dom), rc != 0


def gather(order, comp, patch, origin, spacing, x, y):
    patch = f64(patch)
    ny, nx = patch.shape
    x, y = f64(x), f64(y)
    out = np.zeros(len(x))
    rc = lib().ref_gather(order, comp, _p(patch), nx, ny, origin[0], origin[1], spacing[0], spacing[1], _p(x),
                          _p(y), len(x), _p(out))
    if rc:
        raise RuntimeError("the reference's patch index check failed")
    return out
