"""The CPU oracle against the reference's known-answer tests (read from the reference test
files; Julia is not available, so the vectors are restated here) and against the golden
fixtures committed under tests/golden/."""
import os

import numpy as np
import pytest

from conftest import cgauss, grid_c1, sphere

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_sincos_accuracy():
    """The project sin/cos (Cody-Waite + Taylor) against libm: within 2 ulp of |result| <= 1."""
    xs = np.concatenate([np.linspace(0, 1, 1001), np.random.default_rng(0).uniform(0, 400, 5000),
                         np.arange(1, 200) * np.pi / 4])
    for x in xs:
        s, c = O.sincos(x)
        assert abs(s - np.sin(x)) <= 2.3e-16 and abs(c - np.cos(x)) <= 2.3e-16


def test_entries_match_formula():
    rng = np.random.default_rng(1)
    tp, sp = rng.uniform(0, 1, (200, 3)), rng.uniform(2, 3, (300, 3))
    ii, jj = rng.integers(0, 200, 5000), rng.integers(0, 300, 5000)
    for k, sign in ((0.7, 1), (30.0, -1)):
        v = O.entries(O.Kernel(O.KIND_HELMHOLTZ, k=k, sign=sign), tp, sp, ii, jj)
        r = np.linalg.norm(tp[ii] - sp[jj], axis=1)
        ref = np.exp(1j * sign * k * r) / (4 * np.pi * r)
        # a one-ulp difference in r moves the phase by k r ulp: scale the bound with k r
        assert np.all(np.abs(v - ref) / np.abs(ref) < 4e-16 * (4 + k * r))
    z = O.entries(O.Kernel(O.KIND_HELMHOLTZ, k=1.0), tp, tp, np.arange(5), np.arange(5))
    assert np.all(z == 0)


def test_sampled_stopping_kat():
    """test/compressors/test_batchedbottomup.jl:43-52."""
    A = np.zeros((5, 3))
    A[0, 0], A[1, 1], A[2, 2] = 1, 0.009, 0.001
    assert O.aca(A, 3, 1e-2, sampled=False)[0] == 1
    assert O.aca(A, 3, 1e-2, sampled=True)[0] == 2


def test_aca_residual_bound_and_zero_block():
    """test/gpu/test_compresslevel.jl:127-189 on the CPU ACA."""
    rng = np.random.default_rng(41)
    tol = 1e-3
    for m, n in ((90, 30), (65, 18)):
        U = np.linalg.qr(rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))[0][:, :n]
        V = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))[0]
        block = U @ np.diag(10.0 ** np.linspace(0, -7, n)) @ V.conj().T
        r, rp, cp = O.aca(block, 30, tol, sampled=True)
        assert 0 < r < min(m, n)
        assert len(set(rp)) == r and len(set(cp)) == r
        X = O.cross_solve(block[:, cp], rp)
        err = np.linalg.norm(X @ block[rp, :] - block) / np.linalg.norm(block) * np.sqrt(n / (n - r))
        assert err <= 1.01 * tol
    assert O.aca(np.zeros((40, 25)), 30, tol)[0] == 0


def test_crossfactorization_kats():
    """test/utils/test_utils.jl:55-72."""
    X = np.array([[2, 1], [1, 3]], dtype=complex)
    b = np.array([1, 2], dtype=complex)
    sol = O.cross_solve(np.vstack([X, b[None, :]]), [0, 1])
    assert np.allclose(sol[2] @ X, b)
    with pytest.raises(O.SingularCross) as err:
        O.cross_solve(np.array([[1, 2], [1, 2]], dtype=complex), [0, 1])
    assert err.value.npivots == 2 and err.value.rank == 1


def test_nested_basis_kats():
    """test/test_nestedbasis.jl:10-65 (0-based indices)."""
    rng = np.random.default_rng(1)
    buf = rng.random((12, 6)) + 1j * rng.random((12, 6))
    original = buf.copy()
    tvalues = [1, 2, 4, 6, 7, 8, 10]
    pivots = [7, 2, 10]
    local = [tvalues.index(p) for p in pivots]
    basis = O.cross_solve(buf[tvalues, :3], local)
    assert np.array_equal(buf, original)
    assert basis.shape == (7, 3)
    assert np.allclose(basis @ buf[pivots, :3], buf[tvalues, :3], atol=1e-13)
    assert np.allclose(basis[local, :], np.eye(3), atol=1e-13)
    empty = O.cross_solve(np.zeros((7, 0)), [])
    assert empty.shape == (7, 0)
    # trial side: basis = X^T satisfies buf[1:3, piv] * basis = buf[1:3, svalues]
    tb = basis.T
    assert np.allclose(buf[pivots, :3].T @ tb, buf[tvalues, :3].T, atol=1e-13)
    dup = rng.random((8, 2)) + 0j
    dup[6, :] = dup[2, :]
    with pytest.raises(O.SingularCross):
        O.cross_solve(dup, [2, 6])


def test_transfer_kats():
    """test/test_transfermatrices.jl:11-60: transfer * buf[rows] = buf[childrows]; nestedness."""
    rng = np.random.default_rng(1)
    buf = rng.random((12, 6)) + 1j * rng.random((12, 6))
    rows, childrows = [8, 1, 5], [3, 1, 10, 6]
    X = O.cross_solve(buf[:, :3], rows)
    transfer = X[childrows, :]
    assert transfer.shape == (4, 3)
    assert np.allclose(transfer @ buf[rows, :3], buf[childrows, :3], atol=1e-12)
    low = (rng.random((12, 3)) + 1j * rng.random((12, 3))) @ (rng.random((3, 6)) + 1j * rng.random((3, 6)))
    childvalues, childpivots = [0, 3, 4, 7, 9], [3, 9, 0]
    childbasis = O.cross_solve(low[childvalues, :3], [childvalues.index(p) for p in childpivots])
    parentbasis = O.cross_solve(low[:, :3], rows)
    transfer = parentbasis[childpivots, :]
    assert np.allclose(childbasis @ transfer, parentbasis[childvalues, :], rtol=100 * np.sqrt(2.2e-16))


def test_c1_against_dense():
    """test/nca/test_petrovgalerkinnca.jl:102: relative error < 5 tol."""
    test, trial = grid_c1()
    k = 2 * np.pi / 10
    kern = O.Kernel(O.KIND_HELMHOLTZ, k=k)
    H = O.H2(test, trial, kern, minvalues=32, tol=1e-4)
    ii, jj = np.meshgrid(np.arange(1024), np.arange(1024), indexing="ij")
    D = O.entries(kern, test, trial, ii.ravel(), jj.ravel()).reshape(1024, 1024)
    for x in (np.ones(1024, complex), cgauss(1024, 1)):
        for mode, M in ((0, D), (1, D.T), (2, D.conj().T)):
            y = H.apply(x, mode)
            assert np.linalg.norm(y - M @ x) / np.linalg.norm(M @ x) < 5e-4


def test_nonsymmetric_rectangular_tol_1e8():
    """test/compressors/test_trialassembly.jl:15-75: forward and adjoint < 1e-10 at ACA tol 1e-8,
    maxrank 10, with a separable nonsymmetric kernel given as a matrix."""
    for nt, ns in ((160, 160), (96, 160), (160, 96)):
        rng = np.random.default_rng(17)
        tp = rng.random((nt, 3))
        sp = rng.random((ns, 3)) + np.array([10, 0, 0])
        dense = np.outer(1 + 1j * tp[:, 0] + tp[:, 1] ** 2, np.exp(2 * sp[:, 1]) + 1j * sp[:, 2])
        H = O.H2(tp, sp, O.Kernel(O.KIND_MATRIX, matrix=dense), minvalues=80, tol=1e-8, maxrank=10)
        x, y = cgauss(ns, 2), cgauss(nt, 3)
        assert np.linalg.norm(H.apply(x, 0) - dense @ x) / np.linalg.norm(dense @ x) < 1e-10
        assert np.linalg.norm(H.apply(y, 2) - dense.conj().T @ y) / np.linalg.norm(dense.conj().T @ y) < 1e-10


def test_couplings_are_pivot_entries():
    """Coupling blocks equal A[test pivots, trial pivots] exactly (couplingmatrices.jl:11-53)."""
    test, trial = grid_c1()
    kern = O.Kernel(O.KIND_HELMHOLTZ, k=2 * np.pi / 10)
    H = O.H2(test, trial, kern, minvalues=32, tol=1e-4)
    i = 0
    for t in range(H.trees[0].nnodes):
        for s in H.farnodes[H.farptr[t]:H.farptr[t + 1]]:
            tp, sp = H.pivots[0][t], H.pivots[1][s]
            ii, jj = np.meshgrid(tp, sp, indexing="ij")
            ref = O.entries(kern, test, trial, ii.ravel(order="F"), jj.ravel(order="F"))
            assert np.array_equal(H.couplings[i].ravel(order="F"), ref)
            i += 1


def test_golden_c1():
    """The oracle reproduces the committed C1 fixture (tests/golden/make_golden.py)."""
    g = np.load(os.path.join(GOLDEN, "c1.npz"))
    test, trial = grid_c1()
    H = O.H2(test, trial, O.Kernel(O.KIND_HELMHOLTZ, k=2 * np.pi / 10), minvalues=32, tol=1e-4)
    assert np.array_equal(H.trees[0].perm, g["test_perm"])
    assert np.array_equal(H.trees[1].perm, g["trial_perm"])
    for side, name in ((0, "test"), (1, "trial")):
        assert np.array_equal(H.ranks[side], g[f"{name}_ranks"])
        assert np.array_equal(np.concatenate([p for p in H.pivots[side]]), g[f"{name}_pivots"])
        assert np.array_equal(np.concatenate([p for p in H.farpivots[side]]), g[f"{name}_farpivots"])
    y = H.apply(np.ones(1024, complex))
    assert np.linalg.norm(y - g["y_ones"]) / np.linalg.norm(g["y_ones"]) < 1e-13
    yx = H.apply(g["x_gauss"])
    assert np.linalg.norm(yx - g["y_gauss"]) / np.linalg.norm(g["y_gauss"]) < 1e-13


def test_oracle_galerkin_sphere():
    """Test = trial on a sphere (r = 0 on the diagonal): sampled dense rows within 5 tol."""
    pts = sphere(8192, 21)
    kern = O.Kernel(O.KIND_HELMHOLTZ, k=1.0)
    H = O.H2(pts, pts, kern, minvalues=64, tol=1e-5)
    x = cgauss(8192, 22)
    rows = np.random.default_rng(3).choice(8192, 256, replace=False)
    y = H.apply(x)
    yd = O.dense_rows(kern, pts, pts, rows, x)
    assert np.linalg.norm(y[rows] - yd) / np.linalg.norm(yd) < 5e-5
