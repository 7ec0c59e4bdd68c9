"""IACA (the BottomUp compressor's factorization) on the CPU oracle, and the compressor surface.

The reference's IACA lives in AdaptiveCrossApproximation.jl, which is not in the reference tree;
its call sites fix what is kept here (src/pivoting/pivots.jl:66-68, :215-300, :329-364,
:450-513): the geometric side is picked by tree mimicry over the far nodes, the own side by the
maximum value, the rank limit is min(maxrank, candidates, far points), and the interpolation
operator is X = K[rows, sigma] K[tau, sigma]^-1 (src/nestedbasis.jl:43-57). The tests check
those properties and the project rule's stop on blocks with a known answer."""
import numpy as np
import pytest

from conftest import cgauss, sphere

from oracle import oracle as O


def _setup(n_own=64, n_far=900, seed=3, shift=(3.0, 0.0, 0.0)):
    rng = np.random.default_rng(seed)
    own = rng.uniform(0, 1, (n_own, 3))
    far = rng.uniform(0, 1, (n_far, 3)) + np.array(shift)
    F = O.OwnedTree(far, 16)
    roots = [1, 2]  # the far tree's two children: the whole far field
    return own, far, F, roots


def test_iaca_interpolates_and_bounds_the_rank():
    own, far, F, roots = _setup()
    K = O.Kernel(O.KIND_HELMHOLTZ, k=2.0)
    rows = np.arange(len(own))
    for tol, maxrank in ((1e-2, 50), (1e-6, 50), (1e-12, 7)):
        r, rp, cp, X = O.iaca(F, K, own, far, rows, rows, roots, maxrank, tol)
        assert 0 < r <= min(maxrank, len(rows))
        assert len(set(rp)) == r and len(set(cp)) == r
        # X[tau, :] is the identity, bit for bit
        assert np.array_equal(X[rp], np.eye(r))
        # X = K[rows, sigma] K[tau, sigma]^-1
        A = O.entries(K, own, far, np.repeat(rows, r), np.tile(cp, len(rows))).reshape(len(rows), r)
        ref = A @ np.linalg.inv(A[rp])
        assert np.linalg.norm(X - ref) / np.linalg.norm(ref) < 1e-9
    # rank limit: the far field offers fewer points than maxrank
    small = [int(F.firstchild[1])] if F.nchildren[1] else [1]
    nfar = int(sum(F.end[f] - F.begin[f] for f in small))
    r, *_ = O.iaca(F, K, own, far, rows, rows, small, 200, 0.0)
    assert r <= min(nfar, len(rows))


def test_iaca_tolerance_controls_the_block_error():
    """The interpolation error over the whole far field (900 points, of which IACA samples only
    its geometric columns) stays within 10 tol down to 1e-4 and keeps falling with tol below it,
    where the tree-mimicry sample of the far field limits it; ranks grow as tol falls."""
    for seed in (5, 6, 7):
        own, far, F, roots = _setup(seed=seed)
        K = O.Kernel(O.KIND_HELMHOLTZ, k=4.0)
        rows = np.arange(len(own))
        full = O.entries(K, own, far, np.repeat(rows, len(far)), np.tile(np.arange(len(far)), len(rows)))
        full = full.reshape(len(rows), len(far))
        prev = None
        for tol in (1e-2, 1e-3, 1e-4, 1e-6):
            r, rp, cp, X = O.iaca(F, K, own, far, rows, rows, roots, 64, tol)
            err = np.linalg.norm(X @ full[rp] - full) / np.linalg.norm(full)
            if tol >= 1e-4:
                assert err < 10 * tol, (seed, tol, err)
            else:
                assert err < prev[1], (seed, tol, err)
            if prev is not None:
                assert r >= prev[0]
            prev = (r, err)


def test_iaca_zero_block_and_trial_orientation():
    own, far, F, roots = _setup(n_own=20, n_far=200)
    rows = np.arange(len(own))
    Z = O.Kernel(O.KIND_MATRIX, matrix=np.zeros((len(far), len(own))))
    assert O.iaca(F, Z, own, far, rows, rows, roots, 20, 1e-4, side=1)[0] == 0
    # side 1: rows are trial points, columns test points: the block is K[far, own]^T
    K = O.Kernel(O.KIND_HELMHOLTZ, k=1.5)
    r, rp, cp, X = O.iaca(F, K, own, far, rows, rows, roots, 20, 1e-4, side=1)
    A = O.entries(K, far, own, np.tile(cp, len(rows)), np.repeat(rows, r)).reshape(len(rows), r)
    assert np.linalg.norm(X - A @ np.linalg.inv(A[rp])) / np.linalg.norm(X) < 1e-9


def test_iaca_picks_the_mimicry_sequence():
    """The geometric columns are the tree-mimicry pick sequence of _selectfarpivots, in order."""
    own, far, F, roots = _setup(seed=9)
    K = O.Kernel(O.KIND_HELMHOLTZ, k=3.0)
    rows = np.arange(len(own))
    r, rp, cp, X = O.iaca(F, K, own, far, rows, rows, roots, 40, 1e-10)
    seq = O.select_farpivots(F, own, far, rows, roots, 40)
    assert np.array_equal(cp, seq[:r])


def test_bottomup_iaca_end_to_end_error():
    """BottomUp(IACA) on the plain admissibility: relative error against the dense matrix below
    5 tol (test/nca/test_petrovgalerkinnca.jl:55-102)."""
    pts = sphere(3000, 4)
    K = O.Kernel(O.KIND_HELMHOLTZ, k=2.0, rmin=1e-12)
    x = cgauss(3000, 1)
    rows = np.arange(0, 3000, 7)
    ref = O.dense_rows(K, pts, pts, rows, x)
    for tol in (1e-3, 1e-5):
        H = O.H2(pts, pts, K, minvalues=32, tol=tol, iaca=True)
        err = np.linalg.norm(H.apply(x)[rows] - ref) / np.linalg.norm(ref)
        assert err < 5 * tol, (tol, err)


def test_directional_oracle_plan_matches_the_python_restatement():
    """The C directional oracle's plan equals oracle/directional.py's line-by-line restatement."""
    from oracle import directional as D
    for n, k, minv in ((2500, 12.0, 32), (1500, 3.0, 24)):
        pts = sphere(n, 8)
        H = D.DirectionalH2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), k, minvalues=minv, tol=1e-4)
        ot = O.OwnedTree(pts, minv)
        _, _, fptr, fnodes, tptr, tnodes = D.interactions_wideband(ot, ot, k)
        ref = (D.DirectionalData(ot, ot, fptr, fnodes, k), D.DirectionalData(ot, ot, tptr, tnodes, k))
        for side in (0, 1):
            for f in ("farnodes", "dirptr", "dirs", "dirfarptr", "item_basis", "item_chptr", "item_chidx"):
                assert np.array_equal(H.plan[side][f], getattr(ref[side], f)), (side, f)
            assert np.array_equal(H.plan[side]["dirvec"], ref[side].dirvec)


def test_directional_oracle_error_and_adjoint():
    """Directional BottomUp(IACA): dense-row error below 10 tol (test/nca/test_petrovgalerkinnca.jl:152);
    the adjoint product is the adjoint of the forward one; transpose = conj(adjoint(conj x))."""
    from oracle import directional as D
    n, k, tol = 3000, 16.0, 1e-4
    pts = sphere(n, 6)
    K = O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12)
    H = D.DirectionalH2(pts, pts, K, k, minvalues=32, tol=tol)
    assert any(d != 0 for d in H.plan[0]["dirs"])
    x, u = cgauss(n, 1), cgauss(n, 2)
    rows = np.arange(0, n, 5)
    ref = O.dense_rows(K, pts, pts, rows, x)
    y = H.apply(x)
    assert np.linalg.norm(y[rows] - ref) / np.linalg.norm(ref) < 10 * tol
    assert abs(np.vdot(u, y) - np.vdot(H.apply(u, 2), x)) < 1e-12 * abs(np.vdot(u, y))
    assert np.allclose(H.apply(u, 1), H.apply(u.conj(), 2).conj(), rtol=0, atol=1e-14 * np.abs(y).max())


def test_compressor_surface():
    """Wideband partitions take BottomUp(IACA) only (src/compressors/abstractcompressor.jl:39-47);
    IACA's pivotings are checked per side; the two sides take one compressor kind."""
    import nca_b200 as N
    pts = sphere(600, 3)
    t = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=32))
    bt = N.BlockTree(t, t)
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-4))
    batched = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(pts, pts, t), compressor=aca)
    conv = N.FNormExtrapolator(1e-4)
    tc = N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(pts, pts, t), conv))
    sc = N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(pts, pts, t), N.MaximumValue(), conv))
    K = N.HelmholtzKernel(20.0, rmin=1e-12)
    with pytest.raises(N.ArgumentError, match="only supported with BottomUp; got BatchedBottomUp as test"):
        N.PetrovGalerkinNCACore(K, pts, pts, bt, testcompressor=batched, trialcompressor=batched,
                                isnear=N.isnearwideband(20.0))
    with pytest.raises(N.ArgumentError, match="swapped"):
        N.PetrovGalerkinNCACore(K, pts, pts, bt, testcompressor=sc, trialcompressor=tc, isnear=N.isnearwideband(20.0))
    with pytest.raises(N.ArgumentError, match="one kind"):
        N.PetrovGalerkinNCACore(K, pts, pts, bt, testcompressor=tc, trialcompressor=batched)
    with pytest.raises(N.ArgumentError):
        N.BottomUp(factorization=aca)
    with pytest.raises(N.ArgumentError):
        N.IACA(N.MaximumValue(), N.MaximumValue(), conv)
    assert N.FNormExtrapolator(N.FNormEstimator(1e-3)).tol == 1e-3
