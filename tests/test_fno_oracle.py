"""The surrogate's CPU oracle pinned on its own: its hand-derived gradients
against central finite differences of the loss, and its FFT and DFT-matrix
restatements of the spectral layer against each other."""
import numpy as np
import pytest

from oracle.fno_oracle import FNO, NBINS, NFEAT, flatten, init_params, layout, rb, unflatten

SMALL = dict(width=16, modes=8, layers=2, nout=4)


def problem(seed=3, B=2):
    g = np.random.default_rng(seed)
    X = np.zeros((B, NBINS, NFEAT))
    X[..., :6] = g.standard_normal((B, NBINS, 6))
    T = g.standard_normal((B, NBINS, SMALL["nout"]))
    p = init_params(seed, **SMALL)
    for k in p:  # non-zero biases so that their gradients are exercised too
        if p[k].ndim == 1 and k != "pad":
            p[k] = 0.1 * g.standard_normal(p[k].shape)
    return X, T, p


@pytest.mark.parametrize("fft", [True, False])
def test_gradients_match_finite_differences(fft):
    X, T, p = problem()
    loss, g = FNO(p, fft=fft, **SMALL).backward(X, T)
    flat, gflat = flatten(p, **SMALL), flatten(g, **SMALL)
    rng = np.random.default_rng(0)
    names = [n for n, _ in layout(**SMALL) if n != "pad"]
    offs = np.cumsum([0] + [int(np.prod(s)) for _, s in layout(**SMALL)])
    idx = []
    for k, (name, _) in enumerate(layout(**SMALL)):
        if name in names:  # three entries of every parameter tensor
            idx += list(rng.integers(offs[k], offs[k + 1], 3))
    eps = 1e-5
    for i in idx:
        a, b = flat.copy(), flat.copy()
        a[i] += eps
        b[i] -= eps
        fd = (FNO(unflatten(a, **SMALL), fft=fft, **SMALL).loss(X, T) -
              FNO(unflatten(b, **SMALL), fft=fft, **SMALL).loss(X, T)) / (2 * eps)
        assert abs(fd - gflat[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7 * np.abs(gflat).max(), (i, fd, gflat[i])


def test_fft_and_dft_restatements_agree():
    X, T, p = problem(5)
    la, ga = FNO(p, fft=True, **SMALL).backward(X, T)
    lb, gb = FNO(p, fft=False, **SMALL).backward(X, T)
    assert abs(la - lb) <= 1e-12 * la
    for k in ga:
        assert np.allclose(ga[k], gb[k], rtol=1e-9, atol=1e-12 * np.abs(ga[k]).max())


def test_bf16_restatement_close_to_fp64():
    """BF16 rounding of weights and activations moves the loss and the
    gradients by well under a percent."""
    X, T, p = problem(7)
    la, ga = FNO(p, **SMALL).backward(X, T)
    lb, gb = FNO(p, bf16=True, **SMALL).backward(X, T)
    assert abs(la - lb) <= 1e-2 * la
    for k in ga:
        if k == "pad" or not np.any(ga[k]):
            continue
        assert np.linalg.norm(ga[k] - gb[k]) <= 3e-2 * np.linalg.norm(ga[k]), k


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -3.14159, 1e-30, 65504.0], dtype=np.float32)
    r = rb(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6  # ties to even
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
