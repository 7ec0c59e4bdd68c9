"""GPU level seams against the reference's GPU tests (test/gpu/test_compresslevel.jl) and
the oracle: batched fully pivoted ACA, the interpolation solve, singular cross matrices."""
import numpy as np
import pytest

from conftest import cgauss

pytestmark = pytest.mark.gpu


def _n():
    import nca_b200
    return nca_b200


def _o():
    from oracle import oracle
    return oracle


def test_sampled_stopping_kat():
    """test/compressors/test_batchedbottomup.jl:43-52: rank 1 unsampled, 2 sampled."""
    N = _n()
    A = np.zeros((5, 3))
    A[0, 0], A[1, 1], A[2, 2] = 1, 0.009, 0.001
    cfg = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-2))
    assert cfg(A, 3, sampled=False)[0] == 1
    assert cfg(A, 3, sampled=True)[0] == 2


def test_aca_residual_and_oracle_agreement():
    """test/gpu/test_compresslevel.jl:127-189: decaying complex blocks and a zero block; ranks
    and pivots equal the CPU ACA, estimated error <= 1.01 tol."""
    N, O = _n(), _o()
    rng = np.random.default_rng(41)
    specs = [(40, 25), (90, 30), (65, 18)]
    blocks = []
    for i, (m, n) in enumerate(specs):
        U = np.linalg.qr(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))[0][:, :n]
        V = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))[0]
        blocks.append(np.zeros((m, n), complex) if i == 0 else U @ np.diag(10.0 ** np.linspace(0, -7, n)) @ V.conj().T)
    tol = 1e-3
    mr = 30
    ranks, rows, cols = N.seams.blocks_aca(blocks, mr, tol, sampled=True)
    Z = N.seams.blocks_factors(blocks, ranks, rows, cols, mr)
    for i, block in enumerate(blocks):
        r, rp, cp = O.aca(block, mr, tol, sampled=True)
        assert ranks[i] == r
        assert np.array_equal(rows[i], rp) and np.array_equal(cols[i], cp)
        if r == 0:
            assert np.linalg.norm(block) == 0
            continue
        recon = Z[i].T @ block[rp, :]
        m, n = block.shape
        assert r < min(m, n)
        assert np.linalg.norm(recon - block) / np.linalg.norm(block) * np.sqrt(n / (n - r)) <= 1.01 * tol


def test_solve_kat_above_rank_32():
    """test/gpu/test_compresslevel.jl:65-125: Z == transpose(L / L[rows, :]) to 1e-11."""
    N = _n()
    rng = np.random.default_rng(17)
    mr = 80
    lengths = [40, 90, 100, 160]
    ranks = [0, 8, 35, 80]
    blocks, rps, cps, expected = [], [], [], []
    for m, r in zip(lengths, ranks):
        buf = np.zeros((m, mr), complex)
        rows = rng.permutation(m)[:r]
        cols = rng.permutation(mr)[:r]
        L = rng.standard_normal((m, r)) + 1j * rng.standard_normal((m, r))
        L[rows, :] += r * np.eye(r)
        buf[:, cols] = L
        blocks.append(buf)
        rps.append(rows)
        cps.append(cols)
        expected.append((L @ np.linalg.inv(L[rows, :])).T if r else np.zeros((0, m)))
    Z = N.seams.blocks_factors(blocks, ranks, rps, cps, mr)
    for z, e in zip(Z, expected):
        assert z.shape == e.shape
        if e.size:
            assert np.allclose(z, e, rtol=1e-11, atol=1e-11)


def test_zero_rank_padding():
    """test/gpu/test_compresslevel.jl:191-211: zero blocks give rank 0."""
    N = _n()
    blocks = [np.zeros((0, 3)), np.zeros((4, 3)), np.zeros((9, 3))]
    ranks, rows, cols = N.seams.blocks_aca(blocks, 30, 1e-3)
    assert list(ranks) == [0, 0, 0]


def test_singular_cross_matrix():
    """Two identical rows make the cross matrix singular (test/utils/test_utils.jl:55-72)."""
    N = _n()
    L = cgauss((8, 2), 3)
    L[6, :] = L[2, :]
    with pytest.raises(N.SingularCrossMatrixError) as err:
        N.seams.blocks_factors([L], [2], [np.array([2, 6])], [np.array([0, 1])], 2)
    assert err.value.npivots == 2 and err.value.rank == 1


def test_nested_basis_identities():
    """test/test_nestedbasis.jl:10-30: basis * A[piv, :] = A[t, :], basis[piv, :] = I."""
    N = _n()
    rng = np.random.default_rng(1)
    buf = rng.random((12, 6)) + 1j * rng.random((12, 6))
    tvalues = [1, 2, 4, 6, 7, 8, 10]
    piv = [7, 2, 10]
    L = buf[tvalues, :3]
    local = [tvalues.index(p) for p in piv]
    Z = N.seams.blocks_factors([L], [3], [np.array(local)], [np.arange(3)], 3)[0]
    basis = Z.T
    assert np.allclose(basis @ buf[piv, :3], buf[tvalues, :3], atol=1e-12)
    assert np.allclose(basis[local, :], np.eye(3), atol=1e-12)


def test_large_batch_of_blocks_matches_oracle():
    """Many blocks in one launch, tolerance-driven stops, bit-exact pivots."""
    N, O = _n(), _o()
    rng = np.random.default_rng(5)
    blocks = []
    for _ in range(200):
        m, n, r = rng.integers(1, 100), rng.integers(1, 50), rng.integers(1, 12)
        B = (rng.standard_normal((m, r)) + 1j * rng.standard_normal((m, r))) @ \
            (rng.standard_normal((r, n)) + 1j * rng.standard_normal((r, n)))
        B += 1e-7 * (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))
        blocks.append(B)
    for sampled in (True, False):
        ranks, rows, cols = N.seams.blocks_aca(blocks, 50, 1e-5, sampled=sampled)
        for i, b in enumerate(blocks):
            r, rp, cp = O.aca(b, 50, 1e-5, sampled=sampled)
            assert ranks[i] == r and np.array_equal(rows[i], rp) and np.array_equal(cols[i], cp)
