"""CPU oracle of the wake surrogate (a 1D Fourier neural operator): forward
pass, loss and hand-derived backward pass in numpy FP64.

Test infrastructure only: the GPU network (csrst_b200/surrogate.py over the
tensor-core GEMM) is checked against it; nothing in the product imports it.

The network has no counterpart in the reference code base, so there are no
reference vectors to pin it to.  It is pinned instead by (a) central finite
differences of the loss (tests/test_fno_oracle.py) and (b) two restatements of
the spectral layer: numpy's real FFT (`fft=True`) and explicit DFT matrices
(`fft=False`), which agree to rounding; `bf16=True` adds BF16 rounding at the
points where the GPU rounds, for a tight comparison with the GPU.

Architecture (Li et al., "Fourier Neural Operator for Parametric PDEs", 2021):
  V0      = X P^T + p                                   lift, 64 padded features -> width
  H_l     = V_l W_l^T + b_l + irfft_32(rfft_32(V_l) . (Wr_l + i Wi_l))
  V_{l+1} = gelu(H_l) for l < L - 1, H_l for the last layer
  out     = gelu(V_L Q1^T + q1) Q2^T + q2                 per bin, one value per station
  loss    = mean((out - target)^2)
The spectral product keeps the first `modes` Fourier modes of the 256 bins;
mode k multiplies the channel vector by the complex matrix Wr[k] + i Wi[k]
([cin][cout]).  gelu is the erf form.
"""
import numpy as np
from scipy.special import erf

NBINS, NFEAT = 256, 64


def layout(width=128, modes=32, layers=4, nout=32):
    """(name, shape) of every parameter in the order of the flat buffer."""
    out = [("P", (width, NFEAT)), ("p", (width,))]
    for l in range(layers):
        out += [("W%d" % l, (width, width)), ("b%d" % l, (width,)), ("Wr%d" % l, (modes, width, width)),
                ("Wi%d" % l, (modes, width, width))]
    out += [("Q1", (width, width)), ("q1", (width,)), ("Q2", (nout, width)), ("q2", (nout,)), ("pad", (64 - nout,))]
    return out


def unflatten(flat, width=128, modes=32, layers=4, nout=32):
    d, o = {}, 0
    for name, shape in layout(width, modes, layers, nout):
        n = int(np.prod(shape))
        d[name] = flat[o:o + n].reshape(shape)
        o += n
    assert o == flat.size
    return d


def flatten(d, width=128, modes=32, layers=4, nout=32):
    return np.concatenate([np.asarray(d.get(name, np.zeros(shape))).reshape(-1)
                           for name, shape in layout(width, modes, layers, nout)])


def rb(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def dft_matrices(modes, n=NBINS):
    """F[2k + ri][t]: real and imaginary part of mode k of the forward DFT;
    G[t][2k + ri]: the truncated real inverse (weight 1/n for k = 0, 2/n else)."""
    k = np.arange(modes)[:, None]
    t = np.arange(n)[None, :]
    th = 2.0 * np.pi * k * t / n
    F = np.empty((2 * modes, n))
    F[0::2], F[1::2] = np.cos(th), -np.sin(th)
    w = np.where(np.arange(modes) == 0, 1.0 / n, 2.0 / n)[:, None]
    G = np.empty((2 * modes, n))
    G[0::2], G[1::2] = w * np.cos(th), -w * np.sin(th)
    return F, G.T.copy()


class FNO:
    """Oracle network over a parameter dict (float64 arrays; the GPU's BF16
    copies of the weights are rb() of these when bf16=True)."""

    def __init__(self, params, width=128, modes=32, layers=4, nout=32, bf16=False, fft=None):
        self.width, self.modes, self.layers, self.nout, self.bf16 = width, modes, layers, nout, bf16
        self.fft = (not bf16) if fft is None else fft
        assert not (bf16 and self.fft), "the BF16 restatement uses the DFT matrices"
        self.p = {k: np.asarray(v, dtype=np.float64) for k, v in params.items()}
        self.r = rb if bf16 else (lambda x: np.asarray(x, dtype=np.float64))
        F, G = dft_matrices(modes)
        self.F, self.G = self.r(F), self.r(G)

    # spectral product on [B][n][c] activations -> [B][n][o]
    def _spec_fwd(self, V, l):
        B = V.shape[0]
        Wr, Wi = self.p["Wr%d" % l], self.p["Wi%d" % l]
        if not self.fft:
            S = self.r(np.einsum("jn,bnc->bjc", self.F, V))           # [B][2k+ri][c]
            Xr, Xi = S[:, 0::2, :], S[:, 1::2, :]
        else:
            X = np.fft.rfft(V, axis=1)[:, :self.modes, :]
            Xr, Xi = X.real, X.imag
        wr, wi = self.r(Wr), self.r(Wi)
        Zr = np.einsum("bkc,kco->bko", Xr, wr) - np.einsum("bkc,kco->bko", Xi, wi)
        Zi = np.einsum("bkc,kco->bko", Xr, wi) + np.einsum("bkc,kco->bko", Xi, wr)
        Zr, Zi = self.r(Zr), self.r(Zi)
        if not self.fft:
            Z = np.empty((B, 2 * self.modes, Zr.shape[2]))
            Z[:, 0::2], Z[:, 1::2] = Zr, Zi
            Y = np.einsum("nj,bjo->bno", self.G, Z)
        else:
            Zc = np.zeros((B, NBINS // 2 + 1, Zr.shape[2]), dtype=np.complex128)
            Zc[:, :self.modes] = Zr + 1j * Zi
            Y = np.fft.irfft(Zc, n=NBINS, axis=1)
        return Y, (Xr, Xi)

    def forward(self, X):
        """X: [B][256][64] features; returns out [B][256][nout] and the saved state."""
        p, r = self.p, self.r
        X = r(X)
        st = {"X": X, "V": [], "H": [], "spec": []}
        V = r(X @ r(p["P"]).T + p["p"])
        for l in range(self.layers):
            st["V"].append(V)
            Hp = V @ r(p["W%d" % l]).T + p["b%d" % l]
            Y, spec = self._spec_fwd(V, l)
            st["spec"].append(spec)
            H = Hp + Y
            st["H"].append(H)
            V = r(gelu(H)) if l < self.layers - 1 else r(H)
        st["V"].append(V)
        A1pre = V @ r(p["Q1"]).T + p["q1"]
        A1 = r(gelu(A1pre))
        st["A1pre"], st["A1"] = A1pre, A1
        out = A1 @ r(p["Q2"]).T + p["q2"]
        return out, st

    def loss(self, X, T):
        out, _ = self.forward(X)
        return float(np.mean((out - T) ** 2))

    def backward(self, X, T, weight=None):
        """Loss and gradient dict for the mean squared error against T
        [B][256][nout], each output's error multiplied by weight (default 1)."""
        p, r = self.p, self.r
        out, st = self.forward(X)
        n = out.size
        g = {}
        w = 1.0 if weight is None else np.asarray(weight, dtype=np.float64)
        dOut = 2.0 * w * w * (out - T) / n
        loss = float(np.mean((w * (out - T)) ** 2))
        dO16 = r(dOut)
        g["Q2"] = np.einsum("bns,bnc->sc", dO16, st["A1"])
        g["q2"] = dOut.sum(axis=(0, 1))
        dA1 = dO16 @ r(p["Q2"])
        dA1p = dA1 * gelu_grad(st["A1pre"])
        dA1p16 = r(dA1p)
        g["Q1"] = np.einsum("bno,bnc->oc", dA1p16, st["V"][self.layers])
        g["q1"] = dA1p.sum(axis=(0, 1))
        dV = dA1p16 @ r(p["Q1"])
        for l in reversed(range(self.layers)):
            dH = dV * gelu_grad(st["H"][l]) if l < self.layers - 1 else dV
            dH16 = r(dH)
            V = st["V"][l]
            g["W%d" % l] = np.einsum("bno,bnc->oc", dH16, V)
            g["b%d" % l] = dH.sum(axis=(0, 1))
            # spectral: Y = G Z  ->  dZ = G^T dY (the adjoint of the truncated inverse)
            if not self.fft:
                dZ = r(np.einsum("nj,bno->bjo", self.G, dH16))
                dZr, dZi = dZ[:, 0::2], dZ[:, 1::2]
            else:
                w = np.where(np.arange(self.modes) == 0, 1.0 / NBINS, 2.0 / NBINS)[None, :, None]
                D = np.fft.rfft(dH16, axis=1)[:, :self.modes, :] * w
                dZr, dZi = D.real, D.imag
            Xr, Xi = st["spec"][l]
            g["Wr%d" % l] = np.einsum("bko,bkc->kco", dZr, Xr) + np.einsum("bko,bkc->kco", dZi, Xi)
            g["Wi%d" % l] = np.einsum("bko,bkc->kco", dZi, Xr) - np.einsum("bko,bkc->kco", dZr, Xi)
            wr, wi = r(p["Wr%d" % l]), r(p["Wi%d" % l])
            dXr = r(np.einsum("bko,kco->bkc", dZr, wr) + np.einsum("bko,kco->bkc", dZi, wi))
            dXi = r(np.einsum("bko,kco->bkc", dZi, wr) - np.einsum("bko,kco->bkc", dZr, wi))
            dVn = dH16 @ r(p["W%d" % l])
            if not self.fft:
                dS = np.empty((dXr.shape[0], 2 * self.modes, dXr.shape[2]))
                dS[:, 0::2], dS[:, 1::2] = dXr, dXi
                dVn = dVn + np.einsum("jn,bjc->bnc", self.F, dS)
            else:  # adjoint of X_k = sum_t V_t e^{-i 2 pi k t / n}
                k = np.arange(self.modes)[:, None]
                th = 2.0 * np.pi * k * np.arange(NBINS)[None, :] / NBINS
                dVn = dVn + np.einsum("kn,bkc->bnc", np.cos(th), dXr) - np.einsum("kn,bkc->bnc", np.sin(th), dXi)
            dV = dVn
        dV0 = r(dV)
        g["P"] = np.einsum("bno,bnf->of", dV0, st["X"])
        g["p"] = dV.sum(axis=(0, 1))
        return loss, g


def init_params(seed=0, width=128, modes=32, layers=4, nout=32):
    """Uniform initialisation: pointwise weights U(+-1/sqrt(fan_in)), spectral
    weights U(+-0.5/sqrt(width)), biases zero."""
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
