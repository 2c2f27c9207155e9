"""Regenerates tests/golden/reference_vectors.npz from the reference's own
code, compiled here by `make -C oracle ref REF=<checkout>` (oracle/_ref):
Utils::Q_rsqrt, Utils::calc(Dual)CellBorderCrossings (src/utils.hh:364-504),
the current deposits getCurrentDensityBaseImplX/Y of
src/{Zeroth,First,Second}OrderShapeFunction.cpp and FieldPatch::gather with
ScatterGatherImpl (src/FieldPatch.hh, src/ScatterGatherImpl.hh), on seeded
inputs.  The oracle is checked against these vectors where the reference
sources are absent.
Usage: python tests/golden/make_reference_vectors.py <path to the reference checkout>
"""
import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

SPACING = (1e-5, 1.2e-5)
ORIGIN = (-2.5e-5, 1.5e-5)
DT = 0.5 * SPACING[0] / 299792458.0
PATCH = (0, 0, 40, 40)  # i0, j0, ni, nj of the deposit patches


def moves(rng, n, reach):
    """Moves of up to `reach` cells along x and a third of it across."""
    ox = ORIGIN[0] + rng.uniform(10, 30, n) * SPACING[0]
    oy = ORIGIN[1] + rng.uniform(10, 30, n) * SPACING[1]
    ang = rng.uniform(0, 2 * np.pi, n)
    r = rng.uniform(0, reach, n)
    x = ox + r * np.cos(ang) * SPACING[0]
    y = oy + r * np.sin(ang) * SPACING[1] / 3
    q = rng.uniform(-2e-15, -1e-15, n)
    return ox, oy, x, y, q


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("reference", type=Path, help="root of the reference checkout (holds src/)")
    args = ap.parse_args()
    from oracle import reference as R
    R.REF = args.reference
    rng = np.random.default_rng(20261203)
    out = {"spacing": np.array(SPACING), "origin": np.array(ORIGIN), "dt": np.array(DT), "patch": np.array(PATCH)}
    xs = rng.uniform(1.0, 1e7, 256).astype(np.float32)
    out["q_rsqrt_in"] = xs
    out["q_rsqrt_out"] = np.array([R.q_rsqrt(float(v)) for v in xs], dtype=np.float32)
    # crossing splits: moves of up to 2.5 cells (at most 7 points)
    ox, oy, x, y, _ = moves(rng, 200, 2.5)
    cn, cf, cp = np.zeros((2, 200), np.int32), np.zeros((2, 200, 12)), np.zeros((2, 200, 12, 2))
    for d in (0, 1):
        for k in range(200):
            f, pts = R.crossings(d, (ox[k], oy[k]), (x[k], y[k]), SPACING, ORIGIN)
            cn[d, k] = len(f)
            cf[d, k, :len(f)] = f
            cp[d, k, :len(f)] = pts
    out.update(cross_moves=np.stack([ox, oy, x, y]), cross_n=cn, cross_frac=cf, cross_pts=cp)
    # deposits: 300 moves of up to 1.5 cells per order and component
    for order in (0, 1, 2):
        ox, oy, x, y, q = moves(rng, 300, 1.5)
        out[f"dep{order}_moves"] = np.stack([ox, oy, x, y, q])
        for comp in (0, 1):
            J, dom, bad = R.deposit(order, comp, ox, oy, x, y, q, ORIGIN, SPACING, DT, *PATCH)
            assert not bad
            out[f"dep{order}_{comp}"] = J
            out[f"dep{order}_{comp}_dom"] = np.array(dom)
    # gathers: random fields on a 30 x 24 patch, 200 positions, every order and component
    for order in (0, 1, 2):
        patch = rng.standard_normal((24, 30))
        px = ORIGIN[0] + rng.uniform(4, 25, 200) * SPACING[0]
        py = ORIGIN[1] + rng.uniform(4, 19, 200) * SPACING[1]
        out[f"gat{order}_patch"] = patch
        out[f"gat{order}_pos"] = np.stack([px, py])
        for comp in (0, 1, 2):
            out[f"gat{order}_{comp}"] = R.gather(order, comp, patch, ORIGIN, SPACING, px, py)
    dst = Path(__file__).with_name("reference_vectors.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, dst.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
