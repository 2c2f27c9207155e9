"""The GEMM epilogue's store-order choice (csrst_b200/csrc/gemm_maps.h) on
the CPU: the header compiled for the host (tests/cpp/gemm_maps_host.cpp).

For the output maps the surrogate uses, the vector form (16-byte runs of 8
BF16 or 4 FP32 values) is the expected shape with the lane order that keeps
a warp's stores on whole lines; maps that are not a sum of row and column
offsets over a 32 x 32 piece, maps whose runs are not contiguous and outputs
that are not 16-byte aligned have none (the kernel then stores element by
element); and the element-wise path sweeps by rows only where that touches
fewer sectors."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
W, NB, B = 128, 256, 8192          # width, bins, members of the surrogate's inference batch


@pytest.fixture(scope="module")
def gm(tmp_path_factory):
    so = tmp_path_factory.mktemp("gemm_maps") / "gemm_maps_host.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", str(ROOT / "tests/cpp/gemm_maps_host.cpp"),
                    "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    ll, Q = C.c_longlong, C.POINTER(C.c_longlong)
    L.gm_run_shape.argtypes = [C.c_int, C.c_int, ll, ll, ll, ll, C.c_int, C.POINTER(C.c_int), Q, Q]
    L.gm_bases_aligned.argtypes = [C.c_int, C.c_int, ll, ll, ll, ll, ll, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                   C.c_int]
    L.gm_rows_fast.argtypes = [C.c_int, C.c_int, ll, ll, ll, ll, C.c_int]
    return L


def shape(gm, md, nd, s0, s1, t0, t1, L):
    f = C.c_int(-1)
    r, c = np.zeros(32, dtype=np.int64), np.zeros(32, dtype=np.int64)
    k = gm.gm_run_shape(md, nd, s0, s1, t0, t1, L, C.byref(f), r.ctypes.data_as(C.POINTER(C.c_longlong)),
                        c.ctypes.data_as(C.POINTER(C.c_longlong)))
    return k, f.value, r, c


@pytest.mark.parametrize("name,m,L,want,fast_j", [
    ("rows, BF16 (lift, mode mixing, Q1)", (1, 1, W, 0, 1, 0), 8, 0, 1),
    ("rows, FP32 (Q2, 32 outputs)", (1, 1, 32, 0, 1, 0), 4, 0, 1),
    ("columns: V[b][n][c] from the inverse DFT", (1, 1, 1, 0, W, 0), 8, 1, 0),
    ("spectra U[k][b][2c + ri] from the forward DFT", (1, 2, 2, 0, 2 * W * B, 1), 8, 2, 0),
    ("per-member columns, row divisor 256", (NB, 1, W * NB, 1, NB, 0), 8, 1, 0),
])
def test_vector_forms_of_the_surrogate_maps(gm, name, m, L, want, fast_j):
    k, f, r, c = shape(gm, *m, L)
    assert (k, f) == (want, fast_j), name
    # every run of the chosen shape covers L consecutive indices from a multiple of L
    di = {0: lambda t: 0, 1: lambda t: t, 2: lambda t: t // 2, 3: lambda t: t % 2}[k]
    dj = {0: lambda t: t, 1: lambda t: 0, 2: lambda t: t % 2, 3: lambda t: t // 2}[k]
    ri = {0: 1, 1: L, 2: L // 2, 3: 2}[k]
    rj = {0: L, 1: 1, 2: 2, 3: L // 2}[k]
    for oi in range(0, 32, ri):
        for oj in range(0, 32, rj):
            o = r[oi] + c[oj]
            assert o % L == 0
            assert [r[oi + di(t)] + c[oj + dj(t)] for t in range(L)] == list(range(o, o + L))


def test_maps_without_a_vector_form(gm):
    assert shape(gm, 24, 1, 5000, 1, 24, 0, 8)[0] == -2        # row divisor neither divides 32 nor is a multiple
    assert shape(gm, 1, 1, 1000, 0, 3, 0, 8)[0] == -1          # columns 3 apart: no run of 8 consecutive indices
    assert shape(gm, 1, 1, 1000, 0, 1, 0, 8)[:2] == (0, 1)     # rows 1000 apart: runs along a row
    assert shape(gm, 1, 1, 1004, 0, 1, 0, 8)[0] == -1          # rows 1004 apart: odd rows start off 16 bytes
    assert shape(gm, 1, 1, 1004, 0, 1, 0, 4)[:2] == (0, 1)     # ... which FP32 runs of 4 still allow


def test_alignment_of_every_piece(gm):
    ok = dict(md=1, nd=1, sb=W * NB, s0=W, s1=0, t0=1, t1=0, M=NB * B, N=W, batch=1)
    assert gm.gm_bases_aligned(*ok.values(), 0x10000, 8) == 1
    assert gm.gm_bases_aligned(*ok.values(), 0x10008, 8) == 0   # output not 16-byte aligned
    # batches 4 BF16 values off 16 bytes
    assert gm.gm_bases_aligned(*dict(ok, batch=3, sb=W * NB + 4).values(), 0x10000, 8) == 0
    # blocks of 64 rows (divisor 64) whose block stride is 4 values off: the piece at row 64 starts off 16 bytes
    blk = dict(ok, md=64, s0=64 * W + 4, s1=W)
    assert gm.gm_bases_aligned(*blk.values(), 0x10000, 8) == 0
    assert gm.gm_bases_aligned(*dict(blk, M=64).values(), 0x10000, 8) == 1   # one block only: no such piece


def test_element_wise_sweep_order(gm):
    assert gm.gm_rows_fast(1, 1, 1, 0, W, 0, 2) == 1             # columns contiguous: lanes on consecutive rows
    assert gm.gm_rows_fast(1, 1, W, 0, 1, 0, 2) == 0             # rows contiguous: lanes on consecutive columns
