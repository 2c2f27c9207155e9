"""Wake surrogate: a 1D Fourier neural operator (Li et al. 2021) that maps a
bunch's line-charge profile on 256 bins plus the bend parameters (gamma, R,
sigma_s, pipe width) to the longitudinal wake E_s on the same bins at 32
stations along the bend.

Training and inference run on the GPU through the library alone: every product
is the BF16 tensor-core GEMM (tcgen05, FP32 accumulation, csrst_gemm_bf16) and
every other step an element-wise or reduction kernel of nn.cu; torch holds
the device memory and supplies the stream.

Network (width w = 128, 32 Fourier modes, 4 layers, 32 outputs per bin):
  V0      = X P^T + p                          X: 64 features per bin (6 used)
  H_l     = V_l W_l^T + b_l + irfft(rfft(V_l)[:32] . (Wr_l + i Wi_l))
  V_{l+1} = gelu(H_l) (l < 3), V_4 = H_3
  out     = gelu(V_4 Q1^T + q1) Q2^T + q2
The spectral product is three GEMMs per layer: the forward DFT as a product
with a [64 x 256] matrix of cosines and sines (per member, its channels as
rows, reading V's rows of bins as an MN-major operand; output written
mode-major), the mode mixing as a batch of 32 real [2w x 2w] block matrices
(one per mode: [[Wr, -Wi], [Wi, Wr]] interleaved), and, per member, the
truncated inverse DFT with the layer's pointwise product as a second K
segment of the same accumulator, and bias, activation and the BF16 copy
fused into its epilogue.

Activations are BF16 between products (FP32 accumulation inside them); the
loss, gradients of biases and the Adam state are FP32.  Reductions are in a
fixed order, so a training run repeats bit for bit.
"""
import ctypes as C
import math

import numpy as np
import torch

from ._lib import CsrstError, lib
from .tensor import check_errors, gemm, gemm_dual, rowmap

NBINS, NFEAT = 256, 64
KSPLIT = 256          # K-columns per partial product of a weight gradient


def layout(width=128, modes=32, layers=4, nout=32):
    """(name, shape) of every parameter in the order of the flat FP32 buffer."""
    out = [("P", (width, NFEAT)), ("p", (width,))]
    for l in range(layers):
        out += [("W%d" % l, (width, width)), ("b%d" % l, (width,)), ("Wr%d" % l, (modes, width, width)),
                ("Wi%d" % l, (modes, width, width))]
    out += [("Q1", (width, width)), ("q1", (width,)), ("Q2", (nout, width)), ("q2", (nout,)), ("pad", (64 - nout,))]
    return out


def init_params(seed=0, width=128, modes=32, layers=4, nout=32):
    """Uniform initialisation: pointwise weights U(+-1/sqrt(fan_in)), spectral
    weights U(+-0.5/sqrt(width)), biases zero (numpy FP64, by name)."""
    g = np.random.Generator(np.random.Philox(seed))
    d = {}
    for name, shape in layout(width, modes, layers, nout):
        if name.startswith(("Wr", "Wi")):
            d[name] = g.uniform(-0.5, 0.5, shape) / np.sqrt(width)
        elif len(shape) == 2:
            d[name] = g.uniform(-1.0, 1.0, shape) / np.sqrt(shape[1])
        else:
            d[name] = np.zeros(shape)
    return d


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ck(rc, what):
    if rc:
        raise CsrstError(rc, what)


class _Buffers:
    """Activations and scratch of one batch size (training keeps every
    layer's input for the backward pass; inference ping-pongs two).

    Layouts (b member, n bin, c channel, k mode, ri real/imaginary):
      V16  [b][n][c]      rows of the pointwise products; per member, the forward
                          DFT's operand read MN-major (its 256 bins are the K rows)
      Vg16 [c][b][n]      every bin of a channel in one row: weight gradients
      U16  [k][b][2c+ri]  spectra, the mode mixing's operand
      Z16  [k][b][2o+p]   mixed spectra; Zp16 [b][o][2k+p] the inverse DFT's operand
    The pointwise product rides in the inverse DFT's accumulator as a second
    K segment, so the layer's FP32 pre-activation sum never goes to memory
    (it is kept only for training, for the activation's backward pass).
    Every product writes its large outputs in a layout its epilogue can store
    contiguously; the others come from transposes."""

    def __init__(self, net, B, train):
        w, m, L, dev = net.width, net.modes, net.layers, net.device
        R = B * NBINS
        bf, f32 = dict(dtype=torch.bfloat16, device=dev), dict(dtype=torch.float32, device=dev)
        nkeep = L + 1 if train else 2
        self.V16 = [torch.empty(R, w, **bf) for _ in range(nkeep)]
        self.U16 = torch.empty(m, B, 2 * w, **bf)
        self.Z16 = torch.empty(m, B, 2 * w, **bf)
        self.Zp16 = torch.empty(B * w, 2 * m, **bf)
        self.A1_16 = torch.empty(R, w, **bf)
        self.out = torch.empty(R, net.nout, **f32)
        self.train = train
        if not train:
            return
        self.Vg16 = [torch.empty(w, R, **bf) for _ in range(L + 1)]
        self.Ut16 = [torch.empty(m, 2 * w, B, **bf) for _ in range(L)]
        self.Hfull = [torch.empty(R, w, **f32) for _ in range(L - 1)]
        self.A1pre = torch.empty(R, w, **f32)
        self.A1t16 = torch.empty(w, R, **bf)
        self.Xt16 = torch.empty(NFEAT, R, **bf)
        self.dOut = torch.zeros(R, 64, **f32)
        self.dOut16 = torch.empty(R, 64, **bf)
        self.dOutT16 = torch.empty(64, R, **bf)
        self.dA1 = torch.empty(R, w, **f32)
        self.dH = torch.empty(R, w, **f32)
        self.dH16 = torch.empty(R, w, **bf)
        self.dHt16 = torch.empty(w, R, **bf)
        self.dV = torch.empty(R, w, **f32)
        self.dVn = torch.empty(R, w, **f32)
        self.dZ16 = torch.empty(m, B, 2 * w, **bf)
        self.dZt16 = torch.empty(m, 2 * w, B, **bf)
        self.dSk16 = torch.empty(m, B, 2 * w, **bf)
        self.dS16 = torch.empty(B * w, 2 * m, **bf)
        self.dMk = torch.empty(m, 2 * w, 2 * w, **f32)
        self.part = torch.empty(max(R // KSPLIT, 1) * max(w * w, w * NFEAT), **f32)
        # column-sum scratch: ceil(rows / 256) * cols floats for every column sum of the backward pass
        self.cpart = torch.empty(max(B * max(w, 64), ((R // KSPLIT + 255) // 256) * w * max(w, NFEAT)), **f32)
        self.lpart = torch.empty(256, dtype=torch.float64, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float64, device=dev)


class FNO:
    """The surrogate network on one GPU.  Parameters live in one flat FP32
    buffer (order: layout()) with its gradient and Adam moments beside it;
    BF16 copies of the weights (and transposed and block-packed copies) are
    refreshed after every update."""

    def __init__(self, width=128, modes=32, layers=4, nout=32, seed=0, params=None, device="cuda"):
        if width % 64 or modes % 32 or nout % 16 or not 16 <= nout <= 64 or layers < 1:
            raise ValueError("width must be a multiple of 64, modes of 32, nout of 16 (<= 64)")
        self.width, self.modes, self.layers, self.nout = width, modes, layers, nout
        self.device = torch.device(device)
        self.lay = layout(width, modes, layers, nout)
        sizes = [int(np.prod(s)) for _, s in self.lay]
        self.n = sum(sizes)
        f32 = dict(dtype=torch.float32, device=self.device)
        self.w = torch.zeros(self.n, **f32)
        self.g = torch.zeros(self.n, **f32)
        self.m1 = torch.zeros(self.n, **f32)
        self.m2 = torch.zeros(self.n, **f32)
        self.w16 = torch.zeros(self.n, dtype=torch.bfloat16, device=self.device)
        self.off = {}
        o = 0
        for (name, shape), sz in zip(self.lay, sizes):
            self.off[name] = (o, shape)
            o += sz
        self.set_params(params if params is not None else init_params(seed, width, modes, layers, nout))
        bf = dict(dtype=torch.bfloat16, device=self.device)
        self.WT16 = [torch.empty(width, width, **bf) for _ in range(layers)]
        self.Mk16 = [torch.empty(modes, 2 * width, 2 * width, **bf) for _ in range(layers)]
        self.MkT16 = [torch.empty(modes, 2 * width, 2 * width, **bf) for _ in range(layers)]
        self.Q1T16 = torch.empty(width, width, **bf)
        self.Q2T16 = torch.zeros(width, 64, **bf)
        F, G = _dft_matrices(modes)
        self.F16 = torch.from_numpy(F).to(**bf)
        self.FT16 = torch.from_numpy(np.ascontiguousarray(F.T)).to(**bf)
        self.G16 = torch.from_numpy(G).to(**bf)
        self.GT16 = torch.from_numpy(np.ascontiguousarray(G.T)).to(**bf)
        self.t = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.coef = torch.zeros(3, **f32)
        self._bufs = {}
        self.refresh()

    # ---- parameters ----
    def view(self, name, buf=None):
        o, shape = self.off[name]
        return (self.w if buf is None else buf)[o:o + int(np.prod(shape))].view(shape)

    def set_params(self, d):
        flat = np.concatenate([np.asarray(d.get(n, np.zeros(s)), dtype=np.float32).reshape(-1) for n, s in self.lay])
        self.w.copy_(torch.from_numpy(flat))
        if hasattr(self, "WT16"):
            self.refresh()

    def params(self):
        flat = self.w.cpu().numpy().astype(np.float64)
        return {n: flat[self.off[n][0]:self.off[n][0] + int(np.prod(s))].reshape(s) for n, s in self.lay}

    def grads(self):
        flat = self.g.cpu().numpy().astype(np.float64)
        return {n: flat[self.off[n][0]:self.off[n][0] + int(np.prod(s))].reshape(s) for n, s in self.lay}

    def refresh(self):
        """BF16 copies of the weights: one cast of the flat buffer, then the
        transposed pointwise weights and the block-packed spectral weights."""
        L, w, s = self.layers, self.width, _stream()
        _ck(lib().csrst_nn_cast_bf16(_p(self.w), _p(self.w16), self.n, s), "cast")
        for l in range(L):
            _ck(lib().csrst_nn_transpose_bf16(_p(self.view("W%d" % l, self.w16)), _p(self.WT16[l]), 1, w, w, w, s),
                "transpose")
            _ck(lib().csrst_nn_spectral_pack(_p(self.view("Wr%d" % l)), _p(self.view("Wi%d" % l)), self.modes, w,
                                             _p(self.Mk16[l]), _p(self.MkT16[l]), s), "spectral pack")
        _ck(lib().csrst_nn_transpose_bf16(_p(self.view("Q1", self.w16)), _p(self.Q1T16), 1, w, w, w, s), "transpose")
        _ck(lib().csrst_nn_transpose_bf16(_p(self.view("Q2", self.w16)), _p(self.Q2T16), 1, self.nout, w, 64, s),
            "transpose")

    def _buf(self, B, train):
        key = (B, train)
        if key not in self._bufs:
            self._bufs[key] = _Buffers(self, B, train)
        return self._bufs[key]

    # ---- forward ----
    def _tr16(self, src, dst, batch, rows, cols, ldd=None):
        _ck(lib().csrst_nn_transpose_bf16(_p(src), _p(dst), batch, rows, cols, ldd or rows, _stream()), "transpose")

    def _tr32(self, src, dst, rows, cols):
        _ck(lib().csrst_nn_transpose_b32(_p(src), _p(dst), 1, rows, cols, rows, _stream()), "transpose")

    def _forward(self, bf, B, X16, out=None):
        w, m, L, R = self.width, self.modes, self.layers, B * NBINS
        tr = bf.train
        w16 = lambda n: self.view(n, self.w16)
        # lift: V0 in rows and in per-member channel rows
        gemm(X16, w16("P"), R, w, NFEAT, bias=self.view("p"), out16=bf.V16[0])
        for l in range(L):
            i, o = (l, l + 1) if tr else (l & 1, (l + 1) & 1)
            if tr:
                self._tr16(bf.V16[i], bf.Vg16[i], 1, R, w)
            # forward DFT over the bins, per member b: rows c of V[b] read MN-major (the
            # bins are V's rows) -> U[k][b][2c + ri]
            gemm(bf.V16[i], self.F16, w, 2 * m, NBINS, a_mn=True, lda=w, batch=B, stride_a=NBINS * w,
                 out16=bf.U16, omap=dict(md=1, nd=2, sm0=2, sm1=0, sn0=2 * w * B, sn1=1), sb=2 * w)
            if tr:
                self._tr16(bf.U16, bf.Ut16[l], m, B, 2 * w)
            # mode mixing: per mode k, Z[b][2o + p] = sum U[b][2c + q] Mk[2o + p][2c + q]
            gemm(bf.U16, self.Mk16[l], B, 2 * w, 2 * w, batch=m, stride_a=2 * w * B, stride_b=4 * w * w,
                 out16=bf.Z16, omap=rowmap(2 * w), sb=2 * w * B)
            # (mode, (member, channel)) pairs -> ((member, channel), mode) pairs: Zp[(b, o)][2k + p]
            self._tr32(bf.Z16, bf.Zp16, m, B * w)
            # per member b, one accumulator: H_b[o][n] = sum_j Zp[(b, o)][j] G[n][j]   (truncated inverse DFT)
            #                                          + sum_c W[o][c] V[b][n][c]    (pointwise product)
            # + bias[o]; pre-activation, activation, V in rows and in per-member channel rows
            act = l < L - 1
            gemm_dual(bf.Zp16, self.G16, 2 * m, w16("W%d" % l), bf.V16[i], w, w, NBINS, stride_a1=2 * m * w,
                      stride_b2=NBINS * w, batch=B, bias_m=self.view("b%d" % l),
                      pre=bf.Hfull[l] if (tr and act) else None, act=1 if act else 0, out16=bf.V16[o],
                      omap=dict(md=1, nd=1, sm0=1, sm1=0, sn0=w, sn1=0), sb=NBINS * w)
        Vl = bf.V16[L if tr else L & 1]
        if tr:
            self._tr16(Vl, bf.Vg16[L], 1, R, w)
        gemm(Vl, w16("Q1"), R, w, w, bias=self.view("q1"), act=1, pre=bf.A1pre if tr else None, out16=bf.A1_16,
             out16t=bf.A1t16 if tr else None, tmap=dict(md=1, nd=1, sm0=1, sm1=0, sn0=R, sn1=0))
        gemm(bf.A1_16, w16("Q2"), R, self.nout, w, bias=self.view("q2"), out32=bf.out if out is None else out)

    def predict(self, X, chunk=4096):
        """X: [N][256][64] BF16 (device) -> wake [N][256][nout] FP32 (device), in chunks of members."""
        N = X.shape[0]
        out = torch.empty(N, NBINS, self.nout, dtype=torch.float32, device=self.device)
        for a in range(0, N, chunk):
            B = min(chunk, N - a)
            bf = self._buf(B, False)
            self._forward(bf, B, X[a:a + B].reshape(B * NBINS, NFEAT), out[a:a + B])
        return out

    # ---- backward ----
    def _wgrad(self, bf, At, Bt, M, N, K, name):
        """grad[name][M][N] = At[M][K] Bt[N][K]^T as KSPLIT-column partial
        products summed in order."""
        S = K // KSPLIT
        gemm(At, Bt, M, N, KSPLIT, lda=K, ldb=K, batch=S, stride_a=KSPLIT, stride_b=KSPLIT, out32=bf.part,
             omap=rowmap(N), sb=M * N)
        self._colsum(bf, bf.part, S, M * N, self.view(name, self.g))

    def _colsum(self, bf, x, rows, cols, out, accumulate=False):
        assert bf.cpart.numel() >= ((rows + 255) // 256) * cols
        _ck(lib().csrst_nn_colsum(_p(x), rows, cols, _p(bf.cpart), _p(out), 1 if accumulate else 0, _stream()),
            "colsum")

    def _backward(self, bf, B, X16, T, Wt=None):
        w, m, L, R, nout = self.width, self.modes, self.layers, B * NBINS, self.nout
        s = _stream()
        lb = lib()
        w16 = lambda n: self.view(n, self.w16)
        # loss and dLoss/dout into the first nout columns of a 64-column buffer
        _ck(lb.csrst_nn_mse(_p(bf.out), _p(T), _p(Wt), R * nout, _p(bf.dOut), nout, 64, 1, _p(bf.lpart),
                            _p(bf.loss), s), "mse")
        _ck(lb.csrst_nn_cast_bf16(_p(bf.dOut), _p(bf.dOut16), R * 64, s), "cast")
        _ck(lb.csrst_nn_transpose_bf16(_p(bf.dOut16), _p(bf.dOutT16), 1, R, 64, R, s), "transpose")
        self._wgrad(bf, bf.dOutT16, bf.A1t16, nout, w, R, "Q2")
        self._colsum(bf, bf.dOut, R, 64, self.view("q2", self.g))  # q2 and the padding after it
        gemm(bf.dOut16, self.Q2T16, R, w, 64, out32=bf.dA1)
        _ck(lb.csrst_nn_gelu_bwd(_p(bf.dA1), _p(bf.A1pre), _p(bf.dH), _p(bf.dH16), R * w, s), "gelu")
        _ck(lb.csrst_nn_transpose_bf16(_p(bf.dH16), _p(bf.dHt16), 1, R, w, R, s), "transpose")
        self._wgrad(bf, bf.dHt16, bf.Vg16[L], w, w, R, "Q1")
        self._colsum(bf, bf.dH, R, w, self.view("q1", self.g))
        gemm(bf.dH16, self.Q1T16, R, w, w, out32=bf.dV)
        dV, dVn = bf.dV, bf.dVn
        for l in reversed(range(L)):
            if l < L - 1:
                _ck(lb.csrst_nn_gelu_bwd(_p(dV), _p(bf.Hfull[l]), _p(bf.dH), _p(bf.dH16), R * w, s), "gelu")
                dH = bf.dH
            else:
                _ck(lb.csrst_nn_cast_bf16(_p(dV), _p(bf.dH16), R * w, s), "cast")
                dH = dV
            _ck(lb.csrst_nn_transpose_bf16(_p(bf.dH16), _p(bf.dHt16), 1, R, w, R, s), "transpose")
            self._wgrad(bf, bf.dHt16, bf.Vg16[l], w, w, R, "W%d" % l)
            self._colsum(bf, dH, R, w, self.view("b%d" % l, self.g))
            # adjoint of the inverse DFT: dZ[k][(o, ri)][b] = sum_n dH[b][n][o] G[n][2k + ri] (rows (o, b) of dH^T)
            gemm(bf.dHt16, self.GT16, w * B, 2 * m, NBINS, out16=bf.dZt16,
                 omap=dict(md=B, nd=2, sm0=2 * B, sm1=1, sn0=2 * w * B, sn1=B))
            self._tr16(bf.dZt16, bf.dZ16, m, 2 * w, B)
            # mode-mixing weights: dMk[k] = dZ_k^T U_k, then back to (dWr, dWi)
            gemm(bf.dZt16, bf.Ut16[l], 2 * w, 2 * w, B, batch=m, stride_a=2 * w * B, stride_b=2 * w * B,
                 out32=bf.dMk, omap=rowmap(2 * w), sb=4 * w * w)
            _ck(lb.csrst_nn_spectral_unpack(_p(bf.dMk), m, w, _p(self.view("Wr%d" % l, self.g)),
                                            _p(self.view("Wi%d" % l, self.g)), s), "spectral unpack")
            # dU_k = dZ_k Mk -> dSk[k][b][2c + q] -> dS[(b, c)][2k + q]
            gemm(bf.dZ16, self.MkT16[l], B, 2 * w, 2 * w, batch=m, stride_a=2 * w * B, stride_b=4 * w * w,
                 out16=bf.dSk16, omap=rowmap(2 * w), sb=2 * w * B)
            self._tr32(bf.dSk16, bf.dS16, m, B * w)
            # input gradient: pointwise part, then the adjoint of the forward DFT added on
            gemm(bf.dH16, self.WT16[l], R, w, w, out32=dVn)
            gemm(bf.dS16, self.FT16, B * w, NBINS, 2 * m, out32=dVn, accumulate=True,
                 omap=dict(md=w, nd=1, sm0=NBINS * w, sm1=1, sn0=w, sn1=0))
            dV, dVn = dVn, dV
        _ck(lb.csrst_nn_cast_bf16(_p(dV), _p(bf.dH16), R * w, s), "cast")
        _ck(lb.csrst_nn_transpose_bf16(_p(bf.dH16), _p(bf.dHt16), 1, R, w, R, s), "transpose")
        _ck(lb.csrst_nn_transpose_bf16(_p(X16), _p(bf.Xt16), 1, R, NFEAT, R, s), "transpose")
        self._wgrad(bf, bf.dHt16, bf.Xt16, w, NFEAT, R, "P")
        self._colsum(bf, dV, R, w, self.view("p", self.g))

    def loss_and_grad(self, X, T, weight=None):
        """X: [B][256][64] BF16, T: [B][256][nout] FP32 (device, B a multiple
        of 64), weight: optional FP32 per-output weights of the squared error
        (0 leaves an output out).  Fills the gradient buffer; returns the loss
        as a device scalar."""
        B = X.shape[0]
        if B % 64:
            raise ValueError("training batches must be a multiple of 64 members")
        bf = self._buf(B, True)
        X16 = X.reshape(B * NBINS, NFEAT)
        self._forward(bf, B, X16)
        self._backward(bf, B, X16, T.reshape(B * NBINS, self.nout),
                       None if weight is None else weight.reshape(B * NBINS, self.nout))
        return bf.loss

    def adam(self, lr0=1e-3, lr_min=1e-5, total=10000, b1=0.9, b2=0.999, eps=1e-8):
        s = _stream()
        _ck(lib().csrst_nn_adam_tick(_p(self.t), _p(self.coef), lr0, lr_min, total, b1, b2, s), "adam")
        _ck(lib().csrst_nn_adam(_p(self.w), _p(self.g), _p(self.m1), _p(self.m2), self.n, _p(self.coef), b1, b2, eps,
                                s), "adam")
        self.refresh()

    def check(self):
        check_errors(self.device)


def _dft_matrices(modes, n=NBINS):
    """F[2k + ri][t] (forward DFT, real and imaginary rows) and G[t][2k + ri]
    (the real inverse truncated to `modes` modes: weight 1/n for k = 0, 2/n
    for the others)."""
    k = np.arange(modes)[:, None]
    t = np.arange(n)[None, :]
    th = 2.0 * np.pi * k * t / n
    F = np.empty((2 * modes, n), dtype=np.float32)
    F[0::2], F[1::2] = np.cos(th), -np.sin(th)
    wk = np.where(np.arange(modes) == 0, 1.0 / n, 2.0 / n)[:, None]
    G = np.empty((2 * modes, n), dtype=np.float32)
    G[0::2], G[1::2] = wk * np.cos(th), -wk * np.sin(th)
    return F, np.ascontiguousarray(G.T)
