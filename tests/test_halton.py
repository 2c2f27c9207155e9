"""The reference's command-line bunch (Distribution.cpp:55-163): the Halton
points against scipy's construction of the same sequence, the Box-Muller
moments, the charges, and the reference's order (positions sorted by mesh row
then x, momenta left in generation order)."""
import math

import numpy as np
from scipy.stats import qmc

from csrst_b200.workloads import M_E_MEV, halton_bunch, radical_inverse


def test_radical_inverse_is_the_halton_sequence():
    ref = qmc.Halton(2, scramble=False).random(4097)[1:]     # the generator starts at index 1
    k = np.arange(1, 4097)
    assert np.abs(radical_inverse(k, 2) - ref[:, 0]).max() <= 1e-15
    assert np.abs(radical_inverse(k, 3) - ref[:, 1]).max() <= 1e-15
    assert radical_inverse([1, 2, 3], 2).tolist() == [0.5, 0.25, 0.75]


def test_bunch_moments_charges_and_order():
    n, h = 20000, (1e-4, 2e-4)
    x, y, px, py, q = halton_bunch(n, mean_rx=0.05, mean_ry=0.001, sigma_x=1e-3, ekin_mev=250.0, sigma_p=0.5,
                                   qtotal_nc=-1.0, origin=(0.0, -0.01), spacing=h)
    assert np.allclose(q, 1e-9 / n) and abs(q.sum() - 1e-9) < 1e-21
    assert abs(x.mean() - 0.05) < 2e-5 and abs(y.mean() - 0.001) < 2e-5
    assert abs(x.std() / 1e-3 - 1) < 0.01 and abs(y.std() / 1e-3 - 1) < 0.01
    g = 250.0 / M_E_MEV + 1
    assert abs(px.mean() - math.sqrt(g * g - 1)) < 0.01 and abs(py.std() / 0.5 - 1) < 0.01
    row = np.trunc((y + 0.01) / h[1])
    assert np.all(np.diff(row) >= 0)
    same = np.diff(row) == 0
    assert np.all(np.diff(x)[same] >= 0)
    # momenta stay in generation order: offset k is sigma_p / sigma_x times position offset k before the sort
    k = np.arange(1, n + 1)
    r = np.sqrt(-2 * np.log(radical_inverse(k, 2)))
    assert np.allclose(py, 0.5 * r * np.sin(2 * np.pi * radical_inverse(k, 3)), rtol=0, atol=1e-15)


def test_cpp_distribution_matches_python(tmp_path):
    """include/csrst/distribution.hpp builds the same bunch as the Python
    restatement: the same row-and-x order, values equal to a few ulps (the two
    sides' log, sqrt, cos and sin libraries may round differently)."""
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    exe, out = tmp_path / "halton_main", tmp_path / "bunch.bin"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(root / "include"), str(root / "tests/cpp/halton_main.cpp"),
                    "-o", str(exe)], check=True)
    subprocess.run([str(exe), str(out)], check=True)
    got = np.fromfile(out, dtype=np.float64).reshape(5, 3000)
    ref = halton_bunch(3000, mean_rx=1.7e-3, mean_ry=1.0e-3, sigma_x=40e-6, ekin_mev=510.489, sigma_p=1.0,
                       qtotal_nc=1.0, origin=(-20e-6, -20e-6), spacing=(20e-6, 20e-6))
    for a, b in zip(got, ref):
        assert np.allclose(a, b, rtol=4e-16 * 8, atol=0), np.abs(a - b).max()
