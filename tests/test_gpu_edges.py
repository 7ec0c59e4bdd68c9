"""GPU: edge cases of the build and the product against the oracle — problems without a far field
(one leaf per side), rank-1 bases, products with no right-hand side, and the size limits that the
kernels refuse with an error instead of computing wrong results.

Bars as in the parity suite: pivots bit-exact, products within 1e-12 of the oracle, the dense
matrix within 5 tol."""
import ctypes as C

import numpy as np
import pytest

from conftest import cgauss, sphere

pytestmark = pytest.mark.gpu

REL = 1e-12


def _n():
    import nca_b200
    return nca_b200


def build_pair(test, trial, k, tol, minvalues, maxrank=50):
    from oracle import oracle as O
    N = _n()
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=minvalues))
    st = N.KMeansTree(trial, N.KMeansTreeBuilder(minvalues=minvalues))
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(tol))
    A = N.PetrovGalerkinNCA(N.HelmholtzKernel(k), test, trial, N.BlockTree(tt, st),
                            testcompressor=N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(test, trial, st),
                                                             compressor=aca),
                            trialcompressor=N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(trial, test, tt),
                                                              compressor=aca),
                            maxrank=maxrank)
    H = O.H2(test, trial, O.Kernel(O.KIND_HELMHOLTZ, k=k), minvalues=minvalues, tol=tol, maxrank=maxrank)
    return A, H


def relerr(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def dense(test, trial, k):
    from oracle import oracle as O
    ii, jj = np.meshgrid(np.arange(len(test)), np.arange(len(trial)), indexing="ij")
    return O.entries(O.Kernel(O.KIND_HELMHOLTZ, k=k), test, trial, ii.ravel(), jj.ravel()).reshape(len(test),
                                                                                                 len(trial))


def test_one_leaf_per_side_is_all_near_field():
    """Fewer points than minvalues: each tree is one leaf, the partition one near pair, the
    product one dense block (no far field, no coefficients)."""
    test, trial = sphere(40, 3), sphere(30, 4) * 1.5
    A, H = build_pair(test, trial, 2.0, 1e-6, 64)
    info = _n().core(A).info
    assert info.nnodes_test == 1 and info.nnodes_trial == 1
    assert info.coupling_entries == 0 and info.near_entries == 40 * 30
    D = dense(test, trial, 2.0)
    for b in (1, 3):
        x = cgauss((30, b), b)
        u = cgauss((40, b), 10 + b)
        assert relerr(A @ x, H.apply(x, 0)) < REL
        assert relerr(A @ x, D @ x) < 1e-13
        assert relerr(A.H @ u, D.conj().T @ u) < 1e-13
        assert relerr(A.T @ u, D.T @ u) < 1e-13


def test_rank_one_bases():
    """maxrank = 1: every basis, transfer and coupling has one column; pivots bit-exact and the
    product equal to the oracle's."""
    test, trial = sphere(1500, 5), sphere(1200, 6) * 1.4
    A, H = build_pair(test, trial, 1.0, 1e-8, 32, maxrank=1)
    c = _n().core(A)
    for side in (0, 1):
        piv, ranks, nrows = c.pivots(side)
        assert np.array_equal(ranks, H.ranks[side])
        assert ranks.max() <= 1
        for t in range(len(piv)):
            if piv[t] is not None:
                assert np.array_equal(piv[t], H.pivots[side][t])
    X = cgauss((1200, 5), 7)
    assert relerr(A @ X, H.apply(X, 0)) < REL
    assert relerr(A.H @ cgauss((1500, 2), 8), H.apply(cgauss((1500, 2), 8), 2)) < REL


def test_zero_right_hand_sides_leave_y_alone():
    import torch
    test, trial = sphere(800, 9), sphere(700, 10) * 1.3
    A, _ = build_pair(test, trial, 1.0, 1e-5, 32)
    N = _n()
    W = N.H2Workspace(N.core(A), max_nrhs=4)
    X = torch.zeros((1, 700), dtype=torch.complex128, device="cuda")
    Y = torch.full((1, 800), 3.0 + 1.0j, dtype=torch.complex128, device="cuda")
    st = N._lib.lib().nca_apply(W._h, 0, 0, C.c_void_p(X.data_ptr()), 700, C.c_void_p(Y.data_ptr()), 800, 0, 1.0,
                                0.0, 0.0, 0.0, 1)
    assert st == N._lib.NCA_OK
    torch.cuda.synchronize()
    assert torch.all(Y == 3.0 + 1.0j)


def test_oversized_blocks_are_refused():
    """Blocks that do not fit one CTA's shared memory are refused with NCA_ERR_ARG and a message
    naming the cause, before any kernel computes: a level block of ~600-point leaves times 50 far
    pivots in the build, and maxrank beyond 128 at the boundary."""
    N = _n()
    pts = sphere(1200, 11)
    far = pts + np.array([10.0, 0.0, 0.0])  # well separated: the leaves get far pivots
    with pytest.raises(N.ArgumentError, match="shared memory|more rows"):
        build_pair(pts, far, 1.0, 1e-12, 600)
    with pytest.raises(N.ArgumentError):
        build_pair(pts, far, 1.0, 1e-5, 32, maxrank=129)
