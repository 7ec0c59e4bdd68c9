"""GPU: differentiation on frozen skeletons.

  - d/dk kernel entries against central differences of the entries;
  - refilling the stores at the build's own wavenumber is bit-identical to the build;
  - dH/dk x (tangent product) against central differences (H(k+h) x - H(k-h) x) / 2h of
    frozen-skeleton refills, h = 1e-6 k: relative 1e-6;
  - gradients of J = ||H(k) x - b||^2 from the rrule (x_bar = H^H y_bar, k_bar = Re y_bar^H dH/dk x)
    against central differences (relative 1e-6) and x_bar against the oracle's adjoint product
    (relative 1e-12).
"""
import numpy as np
import pytest

from conftest import cgauss, grid_c1, sphere

pytestmark = pytest.mark.gpu


def _n():
    import nca_b200
    return nca_b200


def relerr(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def build(test, trial, k, tol, minvalues, sign=1, rmin=0.0):
    N = _n()
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=minvalues))
    st = N.KMeansTree(trial, N.KMeansTreeBuilder(minvalues=minvalues))
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(tol))
    tc = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(test, trial, st), compressor=aca)
    sc = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(trial, test, tt), compressor=aca)
    return N.PetrovGalerkinNCA(N.HelmholtzKernel(k, sign=sign, rmin=rmin), test, trial, N.BlockTree(tt, st),
                               testcompressor=tc, trialcompressor=sc)


def test_entries_dk_against_differences():
    N = _n()
    rng = np.random.default_rng(1)
    test = rng.uniform(-2, 2, (300, 3))
    trial = rng.uniform(-2, 2, (200, 3))
    ii = rng.integers(0, 300, 5000)
    jj = rng.integers(0, 200, 5000)
    for k, sign in ((0.7, 1), (12.0, -1)):
        h = 1e-5 * k
        d = N.seams.entries(N.HelmholtzKernel(k, sign=sign), test, trial, ii, jj, dk=True)
        fp = N.seams.entries(N.HelmholtzKernel(k + h, sign=sign), test, trial, ii, jj)
        fm = N.seams.entries(N.HelmholtzKernel(k - h, sign=sign), test, trial, ii, jj)
        assert relerr(d, (fp - fm) / (2 * h)) < 1e-7
    assert np.all(N.seams.entries(N.LaplaceKernel(), test, trial, ii, jj, dk=True) == 0)


def test_refill_at_build_wavenumber_is_bit_identical():
    test, trial = grid_c1()
    k = 2 * np.pi / 10
    A = build(test, trial, k, 1e-4, 32)
    x = cgauss((1024, 3), 2)
    y0 = A @ x
    yt0 = A.T @ x
    X0 = [A.core.interpolation(s) for s in (0, 1)]
    A.core.set_wavenumber(1.3 * k)
    y1 = A @ x
    assert not np.array_equal(y1, y0)
    A.core.set_wavenumber(k)
    assert np.array_equal(A @ x, y0)
    assert np.array_equal(A.T @ x, yt0)
    for s in (0, 1):
        X1 = A.core.interpolation(s)
        for a, b in zip(X0[s], X1):
            assert (a is None and b is None) or np.array_equal(a, b)


def test_refill_at_new_wavenumber_stays_accurate():
    from oracle import oracle as O
    test, trial = grid_c1()
    k = 2 * np.pi / 10
    A = build(test, trial, k, 1e-4, 32)
    A.core.set_wavenumber(1.05 * k)
    x = cgauss(1024, 3)
    rows = np.arange(0, 1024, 8)
    ref = O.dense_rows(O.Kernel(O.KIND_HELMHOLTZ, k=1.05 * k), test, trial, rows, x)
    assert relerr((A @ x)[rows], ref) < 1e-3


@pytest.mark.parametrize("nrhs", [1, 3, 19])
def test_dHdk_against_central_differences(nrhs):
    N = _n()
    test, trial = grid_c1()
    k = 2 * np.pi / 10
    A = build(test, trial, k, 1e-4, 32)
    x = cgauss((1024, nrhs), 4 + nrhs)
    d = N.dHdk(A) @ x
    h = 1e-6 * k
    A.core.set_wavenumber(k + h)
    yp = A @ x
    A.core.set_wavenumber(k - h)
    ym = A @ x
    A.core.set_wavenumber(k)
    assert relerr(d, (yp - ym) / (2 * h)) < 1e-6


def test_rrule_gradients_sphere():
    from oracle import oracle as O
    N = _n()
    pts = sphere(3000, 9) * (1.0 + 0.1 * np.sin(np.arange(3000) % 7)[:, None])
    k = 6.0
    A = build(pts, pts, k, 1e-5, 40, rmin=1e-12)
    x = cgauss((3000, 2), 10)
    b = cgauss((3000, 2), 11)

    def J(xx):
        r = A @ xx - b
        return float(np.vdot(r, r).real)

    y, pb = N.rrule_mul(A, x)
    kbar, xbar = pb(2 * (y - b))
    # k: central differences on the frozen skeleton
    h = 1e-6 * k
    A.core.set_wavenumber(k + h)
    jp = J(x)
    A.core.set_wavenumber(k - h)
    jm = J(x)
    A.core.set_wavenumber(k)
    assert abs(kbar - (jp - jm) / (2 * h)) < 1e-6 * abs(kbar)
    # x: a random complex direction
    v = cgauss((3000, 2), 12)
    eps = 1e-6
    fd = (J(x + eps * v) - J(x - eps * v)) / (2 * eps)
    assert abs(np.vdot(xbar, v).real - fd) < 1e-6 * abs(fd)
    # x_bar is the adjoint product: the oracle's adjoint on the same input
    H = O.H2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), minvalues=40, tol=1e-5, maxrank=50)
    assert relerr(xbar, H.apply(2 * (y - b), 2)) < 1e-12


def test_gradient_errors():
    N = _n()
    test, trial = grid_c1()
    A = build(test, trial, 1.0, 1e-4, 32)
    B = N.batch([A])
    with pytest.raises(N.ArgumentError):
        N.dHdk(N.H2Workspace(B)) @ cgauss(1024, 1)
    with pytest.raises(N.ArgumentError):
        N.dHdk(A).T @ cgauss(1024, 1)
    with pytest.raises(N.ArgumentError):
        N.dHdk(A.H) @ cgauss(1024, 1)


def build_wideband(pts, k, tol, minvalues):
    """A directional core: BottomUp(IACA) on isnearwideband(k) (test/nca/test_petrovgalerkinnca.jl:131-149)."""
    N = _n()
    t = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=minvalues))
    conv = N.FNormExtrapolator(tol)
    tc = N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(pts, pts, t), conv))
    sc = N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(pts, pts, t), N.MaximumValue(), conv))
    return N.PetrovGalerkinNCA(N.HelmholtzKernel(k, rmin=1e-12), pts, pts, N.BlockTree(t, t),
                               isnear=N.isnearwideband(k), testcompressor=tc, trialcompressor=sc, store_f32=True)


def test_directional_frozen_skeleton_gradients():
    """Directional (wideband) cores on their frozen skeleton: the refill at the build's own
    wavenumber reproduces the product (X recomputed as K[rows, sigma] K[tau, sigma]^-1, equal to
    IACA's U L^-1 up to rounding); dH/dk x matches central differences of refills; the rrule's
    k_bar matches central differences of J = ||H(k) x - b||^2 and its x_bar is the adjoint
    product, which agrees with the oracle's."""
    from oracle import directional as OD
    from oracle import oracle as O
    N = _n()
    n, k, tol = 3000, 16.0, 1e-5
    pts = sphere(n, 51)
    A = build_wideband(pts, k, tol, 32)
    x = cgauss((n, 2), 52)
    b = cgauss((n, 2), 53)
    ybar = cgauss((n, 2), 54)
    H = OD.DirectionalH2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), k, minvalues=32, tol=tol)
    assert relerr(A.H @ ybar, H.apply(ybar, 2)) < 1e-12
    y0 = A @ x
    A.core.set_wavenumber(k)
    assert relerr(A @ x, y0) < 1e-9
    h = 1e-6 * k
    dy = N.dHdk(A) @ x
    A.core.set_wavenumber(k + h)
    yp = A @ x
    A.core.set_wavenumber(k - h)
    ym = A @ x
    A.core.set_wavenumber(k)
    assert relerr(dy, (yp - ym) / (2 * h)) < 1e-6

    def J():
        return float(np.sum(np.abs(A @ x - b) ** 2))
    y, pullback = N.rrule_mul(A, x)
    kbar, xbar = pullback(2 * (y - b))
    A.core.set_wavenumber(k + h)
    jp = J()
    A.core.set_wavenumber(k - h)
    jm = J()
    A.core.set_wavenumber(k)
    assert abs(kbar - (jp - jm) / (2 * h)) < 1e-6 * abs(kbar)
    assert relerr(xbar, A.H @ (2 * (y - b))) < 1e-13
    # the mixed-precision stores follow the refill
    W = N.H2Workspace(N.core(A), np.complex64)
    assert relerr(W @ x, A @ x) < 1e-5
