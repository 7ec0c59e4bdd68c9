"""GPU: directional (wideband) H^2 matrices against the oracle.

The reference builds directional bases only with BottomUp(factorization=IACA(...)) and refuses
every other compressor (src/compressors/abstractcompressor.jl:39-47). Basis items (one per
(cluster, direction)), their ranks and pivots must agree exactly with the oracle's directional
compressor; products in the three modes and with blocks of right-hand sides within 1e-12
(relative) of the oracle's directional product; the error against the dense matrix below 10 tol
(the bar of the reference's IACA compressor tests, test/nca/test_petrovgalerkinnca.jl:152); the
mixed-precision product within 1e-5 of FP64.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cgauss, sphere

pytestmark = pytest.mark.gpu

REL = 1e-12


def _n():
    import nca_b200
    return nca_b200


def compressors(test, trial, tt, st, tol):
    """The reference's wideband compressors (test/nca/test_petrovgalerkinnca.jl:131-139)."""
    N = _n()
    conv = N.FNormExtrapolator(tol)
    tc = N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(test, trial, st), conv))
    sc = N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(trial, test, tt), N.MaximumValue(), conv))
    return tc, sc


def build(test, trial, k, tol, minvalues, store_f32=False):
    N = _n()
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=minvalues))
    st = N.KMeansTree(trial, N.KMeansTreeBuilder(minvalues=minvalues))
    tc, sc = compressors(test, trial, tt, st, tol)
    return N.PetrovGalerkinNCA(N.HelmholtzKernel(k, rmin=1e-12), test, trial, N.BlockTree(tt, st),
                               isnear=N.isnearwideband(k), testcompressor=tc, trialcompressor=sc,
                               store_f32=store_f32)


def items(A, side):
    N = _n()
    L = N.lib()
    n = C.c_int32()
    N._lib.check(L.nca_core_dir_items(A.core._h, side, C.byref(n), None, None, None, None))
    ni = n.value
    ranks = np.zeros(max(ni, 1), np.int32)
    nrows = np.zeros(max(ni, 1), np.int32)
    ptr = np.zeros(ni + 1, np.int32)
    idx = np.zeros(max(ni * A.core.maxrank, 1), np.int32)
    N._lib.check(L.nca_core_dir_items(A.core._h, side, C.byref(n), N._lib.ptr(ranks), N._lib.ptr(nrows),
                                      N._lib.ptr(ptr), N._lib.ptr(idx)))
    return ranks[:ni], [idx[ptr[i]:ptr[i + 1]] for i in range(ni)]


def relerr(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


CASES = [
    ("galerkin sphere k=12", lambda: (sphere(2000, 1), None), 12.0, 1e-4, 32),
    ("two point sets k=8", lambda: (sphere(1500, 2), sphere(1200, 3) * 0.8 + np.array([2.2, 0.4, 0.1])), 8.0, 1e-5, 24),
    ("low frequency k=0.5", lambda: (sphere(1200, 4), None), 0.5, 1e-4, 32),
]


@pytest.mark.parametrize("name,make,k,tol,minvalues", CASES, ids=[c[0] for c in CASES])
def test_directional_against_oracle(name, make, k, tol, minvalues):
    from oracle import directional as OD
    from oracle import oracle as O
    N = _n()
    test, trial = make()
    trial = test if trial is None else trial
    A = build(test, trial, k, tol, minvalues, store_f32=True)
    H = OD.DirectionalH2(test, trial, O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), k, minvalues=minvalues, tol=tol)
    for side in (0, 1):
        ranks, piv = items(A, side)
        assert len(ranks) == H.nitems[side]
        assert np.array_equal(ranks, H.ranks[side]), side
        for it in range(len(ranks)):
            assert np.array_equal(piv[it], H.piv[side][it]), (side, it)
    nt, ns = len(test), len(trial)
    for b in (1, 5, 17):
        x = cgauss((ns, b), 10 + b)
        u = cgauss((nt, b), 20 + b)
        assert relerr(A @ x, H.apply(x, 0)) < REL
        assert relerr(A.T @ u, H.apply(u, 1)) < REL
        assert relerr(A.H @ u, H.apply(u, 2)) < REL
    x = cgauss(ns, 7)
    rows = np.arange(0, nt, max(1, nt // 200))
    ref = O.dense_rows(O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), test, trial, rows, x)
    assert relerr((A @ x)[rows], ref) < 10 * tol
    # complex-FP32 stores and coefficient arena: one column, an odd block, an odd last pass, and
    # blocks whose columns leave lanes idle or take a second pass of the all-column kernel
    W = N.H2Workspace(N.core(A), np.complex64)
    for b in (1, 5, 8, 17, 67, 100, 130):
        X = cgauss((ns, b), 30 + b)
        assert relerr(W @ X, A @ X) < 1e-5, b
        U = cgauss((nt, b), 40 + b)
        assert relerr(W.H @ U, A.H @ U) < 1e-5, b
        assert relerr(W.T @ U, A.T @ U) < 1e-5, b


def test_directional_structure_and_limits():
    N = _n()
    pts = sphere(2000, 5)
    A = build(pts, pts, 20.0, 1e-4, 32)
    ranks, _ = items(A, 0)
    assert len(ranks) > N.core(A).info.nnodes_test  # several directions per cluster
    with pytest.raises(N.ArgumentError):
        N.batch([A])
    with pytest.raises(N.ArgumentError):
        N.core(A).pivots(0)


def test_directional_build_errors_reach_the_caller():
    """The two sides of a directional build run on their own host threads: a side that fails (here
    a basis item beyond the IACA kernel's 256 rows: ~600-point leaves with far fields) raises on
    the caller with its message, and the next build in the process is unaffected."""
    N = _n()
    pts = sphere(1200, 11)
    far = pts + np.array([10.0, 0.0, 0.0])
    with pytest.raises(N.ArgumentError, match="rows"):
        build(pts, far, 0.5, 1e-12, 600)
    test = sphere(900, 12)
    A = build(test, test, 12.0, 1e-4, 32)
    x = cgauss((900, 2), 13)
    y = A @ x
    assert y.shape == (900, 2) and np.all(np.isfinite(y))


def test_concurrent_directional_builds_match():
    """Two directional builds at once from two host threads (each with its own side threads and
    streams, and a plain build beside them raising the level kernel's shared-memory limit) give
    the pivots of a build made alone, bit for bit."""
    import threading
    N = _n()
    pts = sphere(2500, 21)
    alone = build(pts, pts, 16.0, 1e-4, 32)
    want = [items(alone, sd) for sd in (0, 1)]
    out, errors = {}, []

    def run(key, fn):
        try:
            out[key] = fn()
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)

    def plain():
        tt = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=128))
        aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-6))
        comp = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(pts, pts, tt), compressor=aca)
        return N.PetrovGalerkinNCA(N.HelmholtzKernel(1.0), pts, pts, N.BlockTree(tt, tt), testcompressor=comp,
                                   trialcompressor=comp)

    threads = [threading.Thread(target=run, args=(i, lambda: build(pts, pts, 16.0, 1e-4, 32))) for i in range(2)]
    threads.append(threading.Thread(target=run, args=("plain", plain)))
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for i in range(2):
        for sd in (0, 1):
            ranks, piv = items(out[i], sd)
            assert np.array_equal(ranks, want[sd][0])
            assert all(np.array_equal(a, b) for a, b in zip(piv, want[sd][1]))


def test_directional_parity_at_65536_points():
    """The 65,536-point unit sphere at the wideband workload's wavenumber k = 2 pi 8 (tol 1e-4,
    64-point leaves): every item's rank and pivots equal the oracle's, the products agree within
    1e-12 in the three modes, and the error against dense rows stays below 10 tol."""
    from oracle import directional as OD
    from oracle import oracle as O
    n, k, tol = 65536, 2 * np.pi * 8, 1e-4
    pts = sphere(n, 2024)
    A = build(pts, pts, k, tol, 64)
    H = OD.DirectionalH2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), k, minvalues=64, tol=tol)
    for side in (0, 1):
        ranks, piv = items(A, side)
        assert np.array_equal(ranks, H.ranks[side]), side
        bad = [it for it in range(len(ranks)) if not np.array_equal(piv[it], H.piv[side][it])]
        assert not bad, (side, len(bad), bad[:5])
    x = cgauss((n, 2), 5)
    assert relerr(A @ x, H.apply(x, 0)) < REL
    assert relerr(A.H @ x, H.apply(x, 2)) < REL
    rows = np.arange(0, n, n // 256)
    ref = O.dense_rows(O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), pts, pts, rows, x[:, 0])
    assert relerr((A @ x[:, 0])[rows], ref) < 10 * tol


def _mirror_env(on):
    import os
    if on:
        os.environ.pop("NCA_MIRROR_TRIAL", None)
    else:
        os.environ["NCA_MIRROR_TRIAL"] = "0"


@pytest.mark.parametrize("store_f32", [False, True])
def test_mirrored_galerkin_build_equals_two_compressions(store_f32):
    """A Galerkin core (one point set, one tree, a kernel of |x - y|) takes the trial side's
    skeleton from the test side and shares the transposed product's up, down and leaf stages; it
    must equal the core whose trial side is compressed on its own: ranks and pivots of both sides
    bit for bit, products in the three modes to rounding."""
    import os
    pts = sphere(6000, 41)
    old = os.environ.get("NCA_MIRROR_TRIAL")
    try:
        _mirror_env(False)
        B = build(pts, pts, 2 * np.pi * 3, 1e-4, 32, store_f32)
        _mirror_env(True)
        A = build(pts, pts, 2 * np.pi * 3, 1e-4, 32, store_f32)
    finally:
        if old is None:
            os.environ.pop("NCA_MIRROR_TRIAL", None)
        else:
            os.environ["NCA_MIRROR_TRIAL"] = old
    for side in (0, 1):
        ra, pa = items(A, side)
        rb, pb = items(B, side)
        assert np.array_equal(ra, rb), side
        assert all(np.array_equal(p, q) for p, q in zip(pa, pb)), side
    ra0, pa0 = items(A, 0)
    ra1, pa1 = items(A, 1)
    assert np.array_equal(ra0, ra1) and all(np.array_equal(p, q) for p, q in zip(pa0, pa1))
    x = cgauss((len(pts), 4), 5)
    rel = 1e-5 if store_f32 else 1e-13
    for op in (lambda M: M @ x, lambda M: M.T @ x, lambda M: M.H @ x):
        ya, yb = op(A), op(B)
        assert np.linalg.norm(ya - yb) <= rel * np.linalg.norm(yb)
