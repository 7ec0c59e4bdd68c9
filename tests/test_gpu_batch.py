"""GPU: many H^2 problems of uneven size applied as one block-diagonal batch.

Every member's block of a batched product must equal the member's own product (same kernels;
the tile shape of a launch can differ, so the bar is relative 1e-13) and the oracle's product
(relative 1e-12), for the three modes and blocks of right-hand sides, in both stored precisions.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cgauss, cube_surface, sphere

pytestmark = pytest.mark.gpu

REL = 1e-12


def _n():
    import nca_b200
    return nca_b200


def member(n, seed, k, minvalues, store_f32=False):
    N = _n()
    pts = sphere(n, seed) if seed % 2 == 0 else cube_surface(n, seed)
    tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=minvalues))
    bt = N.BlockTree(tree, tree)
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-4))
    comp = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(pts, pts, tree), compressor=aca)
    A = N.PetrovGalerkinNCA(N.HelmholtzKernel(k, rmin=1e-12), pts, pts, bt, testcompressor=comp,
                            trialcompressor=comp, store_f32=store_f32)
    return pts, k, A


@pytest.fixture(scope="module")
def members():
    rng = np.random.default_rng(5)
    sizes = [700, 2400, 300, 1500, 1100]
    return [member(n, 10 + i, float(rng.uniform(0.5, 4.0)), 32 if i % 2 else 48, store_f32=True)
            for i, n in enumerate(sizes)]


def relerr(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_batch_matches_members(members):
    N = _n()
    B = N.batch([A for _, _, A in members])
    assert B.members == len(members)
    assert B.dim == (sum(len(p) for p, _, _ in members),) * 2
    W = N.H2Workspace(B, max_nrhs=8)
    off = B.trialoffsets
    for b in (1, 8, 19):
        X = cgauss((B.dim[1], b), 100 + b)
        for mode, op in ((0, lambda M: M), (1, lambda M: M.T), (2, lambda M: M.H)):
            Y = op(W) @ X
            for i, (_, _, A) in enumerate(members):
                yi = op(A) @ X[off[i]:off[i + 1]]
                assert relerr(Y[off[i]:off[i + 1]], yi) < 1e-13, (b, mode, i)


def test_batch_against_oracle(members):
    from oracle import oracle as O
    N = _n()
    B = N.batch([A for _, _, A in members[:3]])
    W = N.H2Workspace(B)
    X = cgauss((B.dim[1], 4), 7)
    Y = W @ X
    Yh = W.H @ X
    off = B.trialoffsets
    for i, (pts, k, _) in enumerate(members[:3]):
        minvalues = 32 if i % 2 else 48
        H = O.H2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), minvalues=minvalues, tol=1e-4, maxrank=50)
        xi = X[off[i]:off[i + 1]]
        assert relerr(Y[off[i]:off[i + 1]], H.apply(xi, 0)) < REL
        assert relerr(Yh[off[i]:off[i + 1]], H.apply(xi, 2)) < REL


def test_batch_mixed_precision_and_info(members):
    N = _n()
    B = N.batch([A for _, _, A in members])
    W64 = N.H2Workspace(B)
    W32 = N.H2Workspace(B, np.complex64)
    X = cgauss((B.dim[1], 8), 9)
    assert relerr(W32 @ X, W64 @ X) < 1e-6
    s = sum(N.storage(A, verbose=False) for _, _, A in members)
    assert abs(N.storage(B, verbose=False) - s) < 1e-12 * s
    with pytest.raises(N.ArgumentError):
        B.pivots(0)


def test_batch_survives_members_and_static_path():
    import torch
    N = _n()
    ms = [member(n, 20 + i, 1.0 + i, 32) for i, n in enumerate((400, 900))]
    refs = []
    X = cgauss((1300, 3), 11)
    refs = [A @ X[:400] if i == 0 else A @ X[400:] for i, (_, _, A) in enumerate(ms)]
    B = N.batch([A for _, _, A in ms])
    del ms
    import gc
    gc.collect()
    W = N.H2Workspace(B)
    Y = W @ X
    assert relerr(Y[:400], refs[0]) < 1e-13 and relerr(Y[400:], refs[1]) < 1e-13
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda()
    Yd = torch.zeros_like(Xd)
    N._lib.check(N.lib().nca_apply_static(B._h, 0, 0, C.c_void_p(Xd.data_ptr()), 1300, C.c_void_p(Yd.data_ptr()),
                                          1300, 3, 1.0, 0.0, 0.0, 0.0, None))
    assert relerr(Yd.cpu().numpy().T, Y) < 1e-13


def test_batch_move_releases_members():
    N = _n()
    ms = [member(n, 30 + i, 2.0, 32) for i, n in enumerate((500, 800))]
    X = cgauss((1300, 2), 12)
    refs = [ms[0][2] @ X[:500], ms[1][2] @ X[500:]]
    B = N.batch([A for _, _, A in ms], move=True)
    # moved members refuse products and new workspaces
    with pytest.raises(N.ArgumentError):
        ms[0][2] @ X[:500]
    with pytest.raises(N.ArgumentError):
        N.H2Workspace(N.core(ms[1][2]))
    with pytest.raises(N.ArgumentError):
        N.batch([A for _, _, A in ms])
    Y = N.H2Workspace(B) @ X
    assert relerr(Y[:500], refs[0]) < 1e-13 and relerr(Y[500:], refs[1]) < 1e-13
