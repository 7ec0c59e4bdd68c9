"""Writes tests/golden/c1.npz: the oracle's C1 result (1,024-point grid, Helmholtz
k = 2 pi / 10, k-means tree minvalues 32, batched bottom-up ACA tol 1e-4, maxrank 50).

    python tests/golden/make_golden.py

The fixture pins the oracle (trees, phase-1 far pivots, ranks, pivots, products) so that a
change of the restatement shows up as a test failure.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from conftest import cgauss, grid_c1  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    test, trial = grid_c1()
    H = O.H2(test, trial, O.Kernel(O.KIND_HELMHOLTZ, k=2 * np.pi / 10), minvalues=32, tol=1e-4, maxrank=50)
    x = cgauss(1024, 1)
    out = dict(test_perm=H.trees[0].perm, trial_perm=H.trees[1].perm, x_gauss=x,
               y_ones=H.apply(np.ones(1024, complex)), y_gauss=H.apply(x))
    for side, name in ((0, "test"), (1, "trial")):
        out[f"{name}_ranks"] = H.ranks[side]
        out[f"{name}_pivots"] = np.concatenate(H.pivots[side]).astype(np.int32)
        out[f"{name}_farpivots"] = np.concatenate(H.farpivots[side]).astype(np.int32)
    np.savez_compressed(os.path.join(HERE, "c1.npz"), **out)


if __name__ == "__main__":
    main()
