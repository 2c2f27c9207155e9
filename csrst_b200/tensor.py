"""Device-side building blocks of the wake surrogate: the BF16 tensor-core
GEMM of libcsrst_gpu.so (tcgen05, FP32 accumulation) behind a small Python
interface over torch device tensors.  torch only provides the device memory
and the stream; the arithmetic is the library's."""
import ctypes as C

import torch

from ._lib import CsrstError, lib

_ERR = {}


class Epilogue(C.Structure):
    """csrst_gemm_epilogue (include/csrst.h)."""
    _fields_ = [("alpha", C.c_float), ("act", C.c_int), ("accumulate", C.c_int), ("md", C.c_int), ("nd", C.c_int),
                ("sb", C.c_longlong), ("sm0", C.c_longlong), ("sm1", C.c_longlong), ("sn0", C.c_longlong),
                ("sn1", C.c_longlong), ("bias", C.c_void_p), ("res", C.c_void_p), ("pre", C.c_void_p),
                ("out32", C.c_void_p), ("out16", C.c_void_p), ("out16t", C.c_void_p), ("tmd", C.c_int),
                ("tnd", C.c_int), ("tb", C.c_longlong), ("tm0", C.c_longlong), ("tm1", C.c_longlong),
                ("tn0", C.c_longlong), ("tn1", C.c_longlong), ("bias_m", C.c_void_p)]


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _err(device):
    """The device's error word of the tensor-core waits ("cuda" and "cuda:0"
    name the same one)."""
    device = torch.device(device)
    if device.type == "cuda" and device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    if device not in _ERR:
        _ERR[device] = torch.zeros(1, dtype=torch.int32, device=device)
    return _ERR[device]


def rowmap(ld):
    """Index map of a plain row-major output with leading dimension ld."""
    return dict(md=1, nd=1, sm0=ld, sm1=0, sn0=1, sn1=0)


def _epilogue(N, alpha, bias, bias_m, res, pre, out32, out16, out16t, act, accumulate, omap, tmap, sb, tb):
    omap = omap or rowmap(N)
    ep = Epilogue()
    ep.alpha, ep.act, ep.accumulate = alpha, act, 1 if accumulate else 0
    ep.md, ep.nd, ep.sm0, ep.sm1, ep.sn0, ep.sn1 = (omap[k] for k in ("md", "nd", "sm0", "sm1", "sn0", "sn1"))
    ep.sb = sb
    ep.bias, ep.res, ep.pre, ep.out32, ep.out16 = _ptr(bias), _ptr(res), _ptr(pre), _ptr(out32), _ptr(out16)
    ep.bias_m = _ptr(bias_m)
    if out16t is not None:
        ep.out16t = _ptr(out16t)
        ep.tmd, ep.tnd, ep.tm0, ep.tm1, ep.tn0, ep.tn1 = (tmap[k] for k in ("md", "nd", "sm0", "sm1", "sn0", "sn1"))
        ep.tb = tb
    return ep


def gemm(A, B, M, N, K, *, lda=None, ldb=None, batch=1, stride_a=0, stride_b=0, alpha=1.0, bias=None, bias_m=None,
         res=None, pre=None, out32=None, out16=None, out16t=None, act=0, accumulate=False, omap=None, tmap=None, sb=0,
         tb=0, a_mn=False):
    """C[M, N] = alpha A[M, K] B[N, K]^T (+ bias[n] + bias_m[m] + res) on the
    tensor cores, batched over `batch`; outputs through the index maps omap /
    tmap (dicts of md, nd, sm0, sm1, sn0, sn1, default row-major N).  a_mn:
    A is MN-major (K rows of M elements, lda apart, default M)."""
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16
    ep = _epilogue(N, alpha, bias, bias_m, res, pre, out32, out16, out16t, act, accumulate, omap, tmap, sb, tb)
    err = _err(A.device)
    rc = lib().csrst_gemm_bf16_ex(_ptr(A), lda or (M if a_mn else K), stride_a, 1 if a_mn else 0, _ptr(B),
                                  ldb or K, stride_b, M, N, K, batch, C.byref(ep), _ptr(err),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc:
        raise CsrstError(rc, "csrst_gemm_bf16: invalid arguments or launch failure")


def gemm_dual(A1, B1, K1, A2, B2, K2, M, N, *, lda1=None, ldb1=None, stride_a1=0, stride_b1=0, lda2=None,
              ldb2=None, stride_a2=0, stride_b2=0, batch=1, alpha=1.0, bias=None, bias_m=None, res=None, pre=None,
              out32=None, out16=None, out16t=None, act=0, accumulate=False, omap=None, tmap=None, sb=0, tb=0):
    """C = alpha (A1[M, K1] B1[N, K1]^T + A2[M, K2] B2[N, K2]^T) (+ epilogue
    terms as in gemm) in one accumulator; each segment has its own leading
    dimensions and batch strides (0: the operand is shared by the batch)."""
    for t in (A1, B1, A2, B2):
        assert t.dtype == torch.bfloat16
    ep = _epilogue(N, alpha, bias, bias_m, res, pre, out32, out16, out16t, act, accumulate, omap, tmap, sb, tb)
    err = _err(A1.device)
    rc = lib().csrst_gemm_bf16_dual(_ptr(A1), lda1 or K1, stride_a1, _ptr(B1), ldb1 or K1, stride_b1, K1, _ptr(A2),
                                    lda2 or K2, stride_a2, _ptr(B2), ldb2 or K2, stride_b2, K2, M, N, batch,
                                    C.byref(ep), _ptr(err), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc:
        raise CsrstError(rc, "csrst_gemm_bf16_dual: invalid arguments or launch failure")


def check_errors(device="cuda"):
    """Raises if a tensor-core wait gave up since the last check."""
    err = _err(torch.device(device))
    if int(err.item()):
        err.zero_()
        raise CsrstError(-2, "tensor-core GEMM: an mbarrier wait gave up")
