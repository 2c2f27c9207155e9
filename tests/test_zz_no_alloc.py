"""csrst_deposit_noalloc: the deposit for callers that cannot let a library
allocate device memory (their framework owns every allocation, or their time
loop must not stall the device).  The caller -- here torch -- owns the input
and output buffers; the library's only scratch is a fixed device array.

Checked against csrst_deposit (the allocating entry point) on two calls in a
row, so the second call shows that the shared array starts from zero again,
and bit for bit against the oracle's fixed-point deposit on a patch that is
offset from the mesh origin and smaller than the particles' footprint, on a
non-default stream.  This file sorts last so a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from csrst_b200 import ShapeFunction
from csrst_b200._lib import lib

pytestmark = pytest.mark.gpu

C_LIGHT = 299792458.0
CSRST_W_OUTSIDE = 1
CSRST_E_CROSSINGS = -7


def moves(n, h, seed):
    rng = np.random.default_rng(seed)
    ox = rng.uniform(6, 40, n) * h[0]
    oy = rng.uniform(6, 30, n) * h[1]
    ang = rng.uniform(0, 2 * np.pi, n)
    r = rng.uniform(0, 0.5, n) * min(h)
    return ox, oy, ox + r * np.cos(ang), oy + r * np.sin(ang), rng.uniform(-2e-15, 2e-15, n)


def fixed_scale(q, h):
    return 2.0 ** np.floor(np.log2(2.0 ** 62 / (4.0 * len(q) * np.abs(q).max() * C_LIGHT / (h[0] * h[1]))))


def noalloc(order, comp, arrays, origin, spacing, dt, i0, j0, ni, nj, scale, stream=None):
    """Calls the entry point on device copies of `arrays`; returns (status, J)."""
    import torch
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]
    out = torch.full((nj, ni), np.nan, dtype=torch.float64, device="cuda")
    o = np.ascontiguousarray(origin, dtype=np.float64)
    hh = np.ascontiguousarray(spacing, dtype=np.float64)
    torch.cuda.synchronize()
    dp = C.POINTER(C.c_double)
    rc = lib().csrst_deposit_noalloc(order, comp, *[C.c_void_p(t.data_ptr()) for t in dev], len(arrays[0]),
                                     o.ctypes.data_as(dp), hh.ctypes.data_as(dp), dt, i0, j0, ni, nj, scale,
                                     C.c_void_p(out.data_ptr()),
                                     None if stream is None else C.c_void_p(stream.cuda_stream))
    return rc, out.cpu().numpy()


@pytest.mark.parametrize("order", [0, 1, 2])
def test_noalloc_matches_deposit_twice(gpu_lib, order):
    h = (1e-5, 1.2e-5)
    dt = 0.5 * h[0] / C_LIGHT
    sf = ShapeFunction(order)
    for call, (comp, seed) in enumerate(((0, 1), (1, 2))):   # two calls in a row
        arrays = moves(30000, h, seed + 10 * order)
        scale = fixed_scale(arrays[4], h)
        ref = sf.getCurrentDensityBase(comp, *arrays, (0.0, 0.0), h, dt, 0, 0, 48, 40, scale)
        rc, got = noalloc(order, comp, arrays, (0.0, 0.0), h, dt, 0, 0, 48, 40, scale)
        assert rc == 0
        assert np.abs(ref).max() > 0
        assert np.array_equal(got, ref), call


@pytest.mark.parametrize("order", [0, 1, 2])
def test_noalloc_offset_patch_on_a_stream_matches_oracle(gpu_lib, oracle, order):
    """A patch at mesh index (5, 4) that is smaller than the particles'
    footprint, on a torch stream: the contributions inside equal the oracle's
    fixed-point deposit bit for bit, the ones outside are dropped and the call
    says so (CSRST_W_OUTSIDE)."""
    import torch
    h = (1e-5, 1.2e-5)
    dt = 0.5 * h[0] / C_LIGHT
    org = (-3e-5, 2e-5)
    ox, oy, x, y, q = moves(20000, h, 7 + order)
    arrays = (ox + org[0], oy + org[1], x + org[0], y + org[1], q)
    scale = fixed_scale(q, h)
    st = torch.cuda.Stream()
    for comp in (0, 1):
        rc, got = noalloc(order, comp, arrays, org, h, dt, 5, 4, 30, 20, scale, stream=st)
        assert rc == CSRST_W_OUTSIDE
        ref = oracle.deposit(order, comp, *arrays, org, h, dt, 5, 4, 30, 20, fixed_scale=scale)
        assert np.abs(ref).max() > 0
        assert np.array_equal(got, ref), comp


def test_noalloc_crossing_overflow_is_reported(gpu_lib):
    """A particle that crosses more cell borders than one push allows (7 cells
    in x and y) is refused with CSRST_E_CROSSINGS; the others are deposited
    and the next call starts clean."""
    h = (1e-5, 1e-5)
    dt = 0.5 * h[0] / C_LIGHT
    ox, oy, x, y, q = moves(1000, h, 3)
    x[17] = ox[17] + 7 * h[0]
    y[17] = oy[17] + 7 * h[1]
    scale = fixed_scale(q, h)
    rc, _ = noalloc(1, 0, (ox, oy, x, y, q), (0.0, 0.0), h, dt, 0, 0, 64, 64, scale)
    assert rc == CSRST_E_CROSSINGS
    buf = C.create_string_buffer(256)
    lib().csrst_get_error(None, buf, 256)
    assert b"crossings" in buf.value
    x[17], y[17] = ox[17], oy[17]
    rc, got = noalloc(1, 0, (ox, oy, x, y, q), (0.0, 0.0), h, dt, 0, 0, 64, 64, scale)
    assert rc == 0 and np.isfinite(got).all()


def test_noalloc_rejects_oversized_patch(gpu_lib):
    import torch
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    o = np.zeros(2)
    hh = np.ones(2)
    dp = C.POINTER(C.c_double)
    p = C.c_void_p(t.data_ptr())
    rc = lib().csrst_deposit_noalloc(0, 0, p, p, p, p, p, 1, o.ctypes.data_as(dp), hh.ctypes.data_as(dp), 1.0,
                                     0, 0, 1025, 1024, 1.0, p, None)
    assert rc == -1
