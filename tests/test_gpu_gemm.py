"""The surrogate's BF16 tensor-core GEMM (tcgen05, FP32 accumulation) against
an FP64 product of the same BF16 values on the CPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16(rng, shape):
    import torch
    return torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(torch.bfloat16)


def ref(a, b):
    return a.float().double().numpy() @ b.float().double().numpy().T


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 128, 192), (200, 64, 64), (130, 48, 128), (384, 256, 256)])
def test_gemm_matches_cpu(gpu_lib, M, N, K):
    import torch
    from csrst_b200.tensor import check_errors, gemm
    rng = np.random.default_rng(M * 7 + N + K)
    a, b = bf16(rng, (M, K)), bf16(rng, (N, K))
    out = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    gemm(a.cuda(), b.cuda(), M, N, K, out32=out)
    torch.cuda.synchronize()
    check_errors()
    r = ref(a, b)
    assert np.abs(out.cpu().numpy() - r).max() <= 1e-4 * np.abs(r).max()


def test_gemm_epilogue_and_batches(gpu_lib):
    """bias, residual, GELU, pre-activation, BF16 copy in a transposed layout,
    accumulation, and a batch of three products."""
    import torch
    from csrst_b200.tensor import check_errors, gemm
    rng = np.random.default_rng(5)
    M, N, K, Z = 256, 64, 128, 3
    a, b = bf16(rng, (Z, M, K)), bf16(rng, (Z, N, K))
    bias = torch.from_numpy(rng.standard_normal(N).astype(np.float32))
    res = torch.from_numpy(rng.standard_normal((Z, M, N)).astype(np.float32))
    pre = torch.zeros(Z, M, N, device="cuda")
    o32 = torch.full((Z, M, N), 2.0, device="cuda")
    o16t = torch.zeros(Z, N, M, dtype=torch.bfloat16, device="cuda")
    gemm(a.cuda(), b.cuda(), M, N, K, batch=Z, stride_a=M * K, stride_b=N * K, alpha=0.5, bias=bias.cuda(),
         res=res.cuda(), pre=pre, out32=o32, act=1, accumulate=True, sb=M * N, out16t=o16t,
         tmap=dict(md=1, nd=1, sm0=1, sm1=0, sn0=M, sn1=0), tb=N * M)
    torch.cuda.synchronize()
    check_errors()
    for z in range(Z):
        h = 0.5 * ref(a[z], b[z]) + bias.double().numpy() + res[z].double().numpy()
        g = 0.5 * h * (1 + np.vectorize(__import__("math").erf)(h / np.sqrt(2)))
        assert np.abs(pre[z].cpu().numpy() - h).max() <= 1e-4 * np.abs(h).max()
        assert np.abs(o32[z].cpu().numpy() - (2.0 + g)).max() <= 1e-4 * np.abs(g).max()
        t = o16t[z].float().cpu().numpy()
        assert np.abs(t - g.T).max() <= 1e-2 * np.abs(g).max()


def test_gemm_dual_segments_and_row_bias(gpu_lib):
    """C_z = A1_z B1^T + A2 B2_z^T + bias_m[m]: two K segments in one
    accumulator, each with its own strides (B1 and A2 shared by the batch)."""
    import torch
    from csrst_b200.tensor import check_errors, gemm_dual
    rng = np.random.default_rng(11)
    M, N, K1, K2, Z = 128, 256, 64, 128, 3
    a1, b1 = bf16(rng, (Z, M, K1)), bf16(rng, (N, K1))
    a2, b2 = bf16(rng, (M, K2)), bf16(rng, (Z, N, K2))
    bm = torch.from_numpy(rng.standard_normal(M).astype(np.float32))
    out = torch.zeros(Z, M, N, device="cuda")
    gemm_dual(a1.cuda(), b1.cuda(), K1, a2.cuda(), b2.cuda(), K2, M, N, stride_a1=M * K1, stride_b2=N * K2,
              batch=Z, bias_m=bm.cuda(), out32=out, sb=M * N)
    torch.cuda.synchronize()
    check_errors()
    for z in range(Z):
        r = ref(a1[z], b1) + ref(a2, b2[z]) + bm.double().numpy()[:, None]
        assert np.abs(out[z].cpu().numpy() - r).max() <= 1e-4 * np.abs(r).max()


def test_gemm_wait_that_gives_up_reports_and_recovers(gpu_lib):
    """The GEMM's mbarrier waits are bounded.  With the stuck-wait hook (a
    negative limit: the epilogue's first wait is on a barrier nothing
    completes, 1000 polls) the wait gives up: the GEMM reports it through its
    error word (1: a wait gave up, and the clean-up waits for the copies and
    products already issued succeeded), writes nothing, and returns; with the
    default limit restored the same GEMM is correct again, so the context and
    the TMEM allocator are intact."""
    import torch
    from csrst_b200._lib import lib
    from csrst_b200.tensor import _err, gemm
    rng = np.random.default_rng(3)
    M, N, K = 256, 128, 512            # 8 K tiles per output tile, two output tiles
    a, b = bf16(rng, (M, K)), bf16(rng, (N, K))
    out = torch.full((M, N), 7.0, dtype=torch.float32, device="cuda")
    err = _err(torch.device("cuda", torch.cuda.current_device()))
    err.zero_()
    try:
        lib().csrst_gemm_set_wait_limit(-1000)
        gemm(a.cuda(), b.cuda(), M, N, K, out32=out)
        torch.cuda.synchronize()
    finally:
        lib().csrst_gemm_set_wait_limit(0)
    assert int(err.item()) == 1
    assert bool((out == 7.0).all())    # the epilogue was skipped
    err.zero_()
    gemm(a.cuda(), b.cuda(), M, N, K, out32=out)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    r = ref(a, b)
    assert np.abs(out.cpu().numpy() - r).max() <= 1e-4 * np.abs(r).max()


def _gelu(h):
    import math
    return 0.5 * h * (1 + np.vectorize(math.erf)(h / np.sqrt(2)))


def _scatter(h, M, N, Z, md, nd, sm0, sm1, sn0, sn1, sb):
    """Element (z, m, n) of h at its index under an output map."""
    m = np.arange(M)[:, None]
    n = np.arange(N)[None, :]
    idx = (m // md) * sm0 + (m % md) * sm1 + (n // nd) * sn0 + (n % nd) * sn1
    return [(z * sb + idx, h[z]) for z in range(Z)]


@pytest.mark.parametrize("case", ["rows_and_member_columns", "spectra_pairs", "dual_both_orders", "ragged"])
def test_gemm_vector_epilogue_maps(gpu_lib, case):
    """The epilogue's 16-byte runs (rows, columns, the spectra's interleaved
    pairs) and the element-wise path of the pieces at ragged edges, against
    an FP64 product of the same BF16 values: pre-activation (FP32), GELU,
    FP32 and BF16 outputs under both maps."""
    import torch
    from csrst_b200.tensor import check_errors, gemm, gemm_dual
    rng = np.random.default_rng(hash(case) % 1000)
    dev = "cuda"
    if case == "rows_and_member_columns":   # the lift's maps: rows, and per member (128 rows) columns
        Z, M, N, K = 1, 384, 128, 64
        om = dict(md=1, nd=1, sm0=N, sm1=0, sn0=1, sn1=0)
        tm = dict(md=128, nd=1, sm0=N * 128, sm1=1, sn0=128, sn1=0)
    elif case == "spectra_pairs":             # the forward DFT's map: U[k][b][2c + ri]
        Z, M, N, K = 1, 256, 64, 256
        om = dict(md=128, nd=2, sm0=256, sm1=2, sn0=512, sn1=1)
        tm = None
    elif case == "dual_both_orders":          # the inverse DFT's maps: V[b][n][o] and Tv[b][o][n]
        Z, M, N, K = 3, 128, 256, 128
        om = dict(md=1, nd=1, sm0=1, sm1=0, sn0=M, sn1=0)
        tm = dict(md=1, nd=1, sm0=N, sm1=0, sn0=1, sn1=0)
    else:                                     # edge pieces (rows past 200, columns past 80) element-wise
        Z, M, N, K = 2, 200, 80, 128
        om = dict(md=1, nd=1, sm0=N, sm1=0, sn0=1, sn1=0)
        tm = dict(md=1, nd=1, sm0=1, sm1=0, sn0=M, sn1=0)
    a, b = bf16(rng, (Z, M, K)), bf16(rng, (Z, N, K))
    bias = torch.from_numpy(rng.standard_normal(N).astype(np.float32))
    size = Z * M * N
    pre = torch.zeros(size, device=dev)
    o32 = torch.zeros(size, device=dev)
    o16 = torch.zeros(size, dtype=torch.bfloat16, device=dev)
    o16t = torch.zeros(size, dtype=torch.bfloat16, device=dev) if tm else None
    gemm(a.cuda(), b.cuda(), M, N, K, batch=Z, stride_a=M * K, stride_b=N * K, alpha=0.75, bias=bias.cuda(),
         pre=pre, out32=o32, out16=o16, act=1, omap=om, sb=M * N, out16t=o16t, tmap=tm, tb=M * N)
    torch.cuda.synchronize()
    check_errors()
    h = np.stack([0.75 * ref(a[z], b[z]) + bias.double().numpy() for z in range(Z)])
    g = _gelu(h)
    P, O32, O16 = pre.cpu().numpy(), o32.cpu().numpy(), o16.float().cpu().numpy()
    for (idx, hz), gz in zip(_scatter(h, M, N, Z, sb=M * N, **om), g):
        assert np.abs(P[idx] - hz).max() <= 1e-4 * np.abs(h).max()
        assert np.abs(O32[idx] - gz).max() <= 1e-4 * np.abs(g).max()
        assert np.abs(O16[idx] - gz).max() <= 1e-2 * np.abs(g).max()
    if tm:
        T = o16t.float().cpu().numpy()
        for idx, gz in _scatter(g, M, N, Z, sb=M * N, **tm):
            assert np.abs(T[idx] - gz).max() <= 1e-2 * np.abs(g).max()


@pytest.mark.parametrize("M,N,K,Z", [(128, 64, 256, 3), (200, 48, 128, 2), (384, 128, 64, 1)])
def test_gemm_mn_major_a(gpu_lib, M, N, K, Z):
    """A read MN-major (K rows of M contiguous values, as the forward DFT reads
    the activations V[b][n][c]): against the FP64 product of the same BF16
    values, with ragged M (the second 64-row box of a tile past the matrix)."""
    import torch
    from csrst_b200.tensor import check_errors, gemm
    rng = np.random.default_rng(M + N + K + Z)
    at, b = bf16(rng, (Z, K, M)), bf16(rng, (Z, N, K))   # at[z][k][m] = A_z[m][k]
    out = torch.zeros(Z, M, N, dtype=torch.float32, device="cuda")
    gemm(at.cuda(), b.cuda(), M, N, K, a_mn=True, lda=M, batch=Z, stride_a=K * M, stride_b=N * K, out32=out,
         sb=M * N)
    torch.cuda.synchronize()
    check_errors()
    for z in range(Z):
        r = ref(at[z].transpose(0, 1).contiguous(), b[z])
        assert np.abs(out[z].cpu().numpy() - r).max() <= 1e-4 * np.abs(r).max()
