"""GPU parity: the sm_100a build and product against the CPU oracle on the same inputs.

Bar (pivot/skeleton index sets are argmax decisions on FP64 data, so they must agree exactly):
  - kernel entries, tree, partition, phase-1 far pivots, ranks and pivots: bit-exact;
  - interpolation operators, couplings and near blocks: relative 1e-12;
  - FP64 products (forward, transpose, adjoint, blocks of right-hand sides): relative 1e-12;
  - error against the dense FP64 kernel matrix: < 5 tol (test/nca/test_petrovgalerkinnca.jl:102).
"""
import numpy as np
import pytest

from conftest import cgauss, grid_c1, sphere

pytestmark = pytest.mark.gpu

REL = 1e-12


def _n():
    import nca_b200
    return nca_b200


def _o():
    from oracle import oracle
    return oracle


def build_pair(test, trial, k, tol, minvalues, maxrank=50, sign=1, rmin=0.0, store_f32=False, iaca=False):
    """The GPU core and the oracle on the same inputs: BatchedBottomUp(ACA), or with iaca=True
    BottomUp(IACA) on both sides (test/nca/test_petrovgalerkinnca.jl:73-80)."""
    N, O = _n(), _o()
    kern = N.HelmholtzKernel(k, sign=sign, rmin=rmin)
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=minvalues))
    st = N.KMeansTree(trial, N.KMeansTreeBuilder(minvalues=minvalues))
    tree = N.BlockTree(tt, st)
    if iaca:
        conv = N.FNormExtrapolator(tol)
        tc = N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(test, trial, st), conv))
        sc = N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(trial, test, tt), N.MaximumValue(), conv))
    else:
        aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(tol))
        tc = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(test, trial, st), compressor=aca)
        sc = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(trial, test, tt), compressor=aca)
    A = N.PetrovGalerkinNCA(kern, test, trial, tree, testcompressor=tc, trialcompressor=sc, maxrank=maxrank,
                            store_f32=store_f32)
    H = O.H2(test, trial, O.Kernel(O.KIND_HELMHOLTZ, k=k, sign=sign, rmin=rmin), minvalues=minvalues, tol=tol,
             maxrank=maxrank, iaca=iaca)
    return A, H


def relerr(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def c1():
    test, trial = grid_c1()
    return (test, trial) + build_pair(test, trial, 2 * np.pi / 10, 1e-4, 32)


def test_entries_bit_exact():
    N, O = _n(), _o()
    rng = np.random.default_rng(0)
    test = rng.uniform(-3, 3, (500, 3))
    trial = rng.uniform(-3, 3, (400, 3))
    ii = rng.integers(0, 500, 20000)
    jj = rng.integers(0, 400, 20000)
    for k, sign in ((2 * np.pi / 10, 1), (50.26548245743669, 1), (20.0, -1), (1.0, 1)):
        dev = N.seams.entries(N.HelmholtzKernel(k, sign=sign), test, trial, ii, jj)
        ref = O.entries(O.Kernel(O.KIND_HELMHOLTZ, k=k, sign=sign), test, trial, ii, jj)
        assert np.array_equal(dev.view(np.float64), ref.view(np.float64))
    dev = N.seams.entries(N.LaplaceKernel(), test, trial, ii, jj)
    ref = O.entries(O.Kernel(O.KIND_LAPLACE), test, trial, ii, jj)
    assert np.array_equal(dev, ref)
    # coincident points give zero
    z = N.seams.entries(N.HelmholtzKernel(1.0), test, test, np.arange(10), np.arange(10))
    assert np.all(z == 0)


def compare_build(A, H, rel=REL):
    c = A.core
    for side in (0, 1):
        fp = c.farpivots(side)
        for t in range(len(fp)):
            assert np.array_equal(fp[t], H.farpivots[side][t]), (side, t)
        piv, ranks, nrows = c.pivots(side)
        assert np.array_equal(ranks, H.ranks[side])
        assert np.array_equal(nrows, H.nrows[side])
        for t in range(len(piv)):
            if piv[t] is not None:
                assert np.array_equal(piv[t], H.pivots[side][t]), (side, t)
        Xs = c.interpolation(side)
        for t in range(len(Xs)):
            if Xs[t].size:
                assert relerr(Xs[t], H.X[side][t]) < rel, (side, t)
    Cs = c.couplingmatrices.blocks
    assert len(Cs) == len(H.couplings)
    for a, b in zip(Cs, H.couplings):
        assert a.shape == b.shape
        if a.size:
            assert np.array_equal(a, b)
    near = c.nearblocks
    nb = [b for b in H.near if b.size]
    assert len(near) == len(nb)
    for (_, _, a), b in zip(near, nb):
        assert np.array_equal(a, b)


def test_c1_build_bit_exact(c1):
    test, trial, A, H = c1
    compare_build(A, H)


def test_c1_products(c1):
    test, trial, A, H = c1
    N = _n()
    for x in (np.ones(1024, complex), cgauss(1024, 3)):
        for mode, op in ((0, lambda v: A @ v), (1, lambda v: N.transpose(A) @ v), (2, lambda v: N.adjoint(A) @ v)):
            y = op(x)
            assert relerr(y, H.apply(x, mode)) < REL


def test_c1_against_dense(c1):
    test, trial, A, H = c1
    O = _o()
    kern = O.Kernel(O.KIND_HELMHOLTZ, k=2 * np.pi / 10)
    ii, jj = np.meshgrid(np.arange(1024), np.arange(1024), indexing="ij")
    D = O.entries(kern, test, trial, ii.ravel(), jj.ravel()).reshape(1024, 1024)
    for x in (np.ones(1024, complex), cgauss(1024, 4)):
        assert relerr(A @ x, D @ x) < 5e-4
        assert relerr(A.T @ x, D.T @ x) < 5e-4
        assert relerr(A.H @ x, D.conj().T @ x) < 5e-4


def test_multi_rhs_and_mul(c1):
    test, trial, A, H = c1
    N = _n()
    X = cgauss((1024, 16), 7)
    Y = A @ X
    for q in range(16):
        assert relerr(Y[:, q], H.apply(X[:, q], 0)) < REL
    Yt = N.adjoint(A) @ X
    assert relerr(Yt, H.apply(X, 2)) < REL
    y0 = cgauss(1024, 8)
    y = y0.copy()
    al, be = 0.3 + 0.2j, -1.1
    N.mul(y, A, X[:, 0], al, be)
    assert relerr(y, al * H.apply(X[:, 0], 0) + be * y0) < REL
    # more right-hand sides than one tile of 16
    X3 = cgauss((1024, 37), 9)
    assert relerr(A @ X3, H.apply(X3, 0)) < REL


def test_linear_maps(c1):
    test, trial, A, H = c1
    N = _n()
    x = cgauss(1024, 11)
    ref = H.apply(x, 0)
    assert relerr((A + 2 * A) @ x, 3 * ref) < REL
    assert relerr((A.H @ A) @ x, H.apply(ref, 2)) < REL
    assert relerr((A.T - A.H) @ x, H.apply(x, 1) - H.apply(x, 2)) < REL
    xr = np.random.default_rng(1).standard_normal(1024)
    assert relerr(A @ xr, A @ xr.astype(complex)) < 1e-15
    with pytest.raises(N.DimensionMismatch):
        A @ x[:-1]


def test_workspaces_share_core(c1):
    test, trial, A, H = c1
    N = _n()
    x = cgauss(1024, 12)
    other = N.H2Workspace(N.core(A))
    assert N.core(other) is N.core(A)
    for mode in (0, 1, 2):
        op = (lambda W: W) if mode == 0 else (lambda W: W.T) if mode == 1 else (lambda W: W.H)
        assert np.array_equal(op(other) @ x, op(A) @ x)
    # repeated products are bitwise stable
    assert np.array_equal(A @ x, A @ x)


def test_concurrency_guard(c1):
    test, trial, A, H = c1
    N = _n()
    x = cgauss(1024, 13)
    expected = A @ x

    def inside():
        assert A.busy
        with pytest.raises(N.ConcurrentWorkspaceError):
            N.mul(np.zeros(1024, complex), A, x)
        with pytest.raises(N.ConcurrentWorkspaceError):
            A.T @ x

    N.withworkspace(inside, A)
    assert not A.busy
    with pytest.raises(RuntimeError):
        N.withworkspace(lambda: (_ for _ in ()).throw(RuntimeError("boom")), A)
    assert not A.busy
    assert np.array_equal(A @ x, expected)


def test_small_workspaces_padded_strides(c1):
    """Right-hand-side counts whose padded vector stride is b + 3 (b = 3 mod 4), from workspaces
    sized exactly for them and from one that grows."""
    test, trial, A, H = c1
    N = _n()
    for b in (3, 7, 1, 2):
        W = N.H2Workspace(N.core(A), max_nrhs=b)
        X = cgauss((1024, b), 50 + b)
        assert relerr(W @ X, H.apply(X, 0)) < REL
        assert relerr(W.H @ X, H.apply(X, 2)) < REL
    W = N.H2Workspace(N.core(A), max_nrhs=1)
    X = cgauss((1024, 19), 60)
    assert relerr(W @ X, H.apply(X, 0)) < REL
    assert relerr(W.T @ X[:, :11], H.apply(X[:, :11], 1)) < REL


def test_device_arrays(c1):
    import torch
    test, trial, A, H = c1
    X = cgauss((1024, 5), 14)
    Yd = A @ torch.from_numpy(X).cuda()
    assert Yd.is_cuda
    assert relerr(Yd.cpu().numpy(), H.apply(X, 0)) < REL


def test_galerkin_sphere_against_oracle():
    """Test = trial (r = 0 on the diagonal), low frequency: the Galerkin configuration at 8,192
    points, compared with the oracle and with sampled dense rows."""
    pts = sphere(8192, 21)
    A, H = build_pair(pts, pts, 1.0, 1e-5, 64)
    compare_build(A, H)
    O = _o()
    X = cgauss((8192, 16), 22)
    Y = A @ X
    assert relerr(Y, H.apply(X, 0)) < REL
    assert relerr(A.H @ X, H.apply(X, 2)) < REL
    rows = np.random.default_rng(3).choice(8192, 256, replace=False)
    yd = O.dense_rows(O.Kernel(O.KIND_HELMHOLTZ, k=1.0), pts, pts, rows, X[:, 0])
    assert relerr(Y[rows, 0], yd) < 5e-5


def test_galerkin_sphere_full_size():
    """The 65,536-point low-frequency Galerkin sphere (k = 1, tol 1e-5, 64-point leaves) at full
    size: tree, far pivots, ranks and pivots bit-exact, operators within 1e-12, and a 16-column
    block within 1e-12 of the oracle in the forward and adjoint modes."""
    pts = sphere(65536, 2024)
    A, H = build_pair(pts, pts, 1.0, 1e-5, 64, rmin=1e-12)
    compare_build(A, H)
    X = cgauss((65536, 16), 5)
    assert relerr(A @ X, H.apply(X, 0)) < REL
    assert relerr(A.H @ X, H.apply(X, 2)) < REL


@pytest.mark.parametrize("case", ["c1", "sphere"])
def test_bottomup_iaca_against_oracle(case):
    """BottomUp(IACA) on the plain admissibility: pivots bit-exact, operators and products within
    1e-12 of the oracle's IACA build, dense error below 5 tol (test/nca/test_petrovgalerkinnca.jl:102)."""
    O = _o()
    if case == "c1":
        test, trial = grid_c1()
        k, tol, mv = 2 * np.pi / 10, 1e-4, 32
    else:
        test = trial = sphere(8192, 41)
        k, tol, mv = 2.0, 1e-5, 64
    A, H = build_pair(test, trial, k, tol, mv, rmin=1e-12, iaca=True)
    compare_build(A, H)
    X = cgauss((len(trial), 3), 42)
    for mode, op in ((0, lambda v: A @ v), (1, lambda v: A.T @ v), (2, lambda v: A.H @ v)):
        V = X if mode == 0 else cgauss((len(test), 3), 43)
        assert relerr(op(V), H.apply(V, mode)) < REL
    rows = np.arange(0, len(test), max(1, len(test) // 512))
    yd = O.dense_rows(O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12), test, trial, rows, X[:, 0])
    assert relerr((A @ X[:, 0])[rows], yd) < 5 * tol


def test_exp_minus_ikr_and_rmin():
    test = sphere(2048, 31)
    trial = sphere(1500, 32) * 1.3
    A, H = build_pair(test, trial, 3.0, 1e-6, 40, sign=-1, rmin=1e-12, maxrank=40)
    compare_build(A, H)
    x = cgauss(1500, 33)
    assert relerr(A @ x, H.apply(x, 0)) < REL


def test_f32_product(c1):
    test, trial, _, H = c1
    N = _n()
    A, _ = build_pair(test, trial, 2 * np.pi / 10, 1e-4, 32, store_f32=True)
    W = N.H2Workspace(N.core(A), np.complex64)
    X = cgauss((1024, 8), 41)
    ref = H.apply(X, 0)
    assert relerr(W @ X, ref) < 1e-5
    assert relerr(W.H @ X, H.apply(X, 2)) < 1e-5


def test_parts_and_overlapped_stages(c1):
    """The workspace runs the far-field sweeps on its second stream beside the near field and adds
    the leaf bases after the join; far-only and near-only workspaces run the serial leaf launch.
    far + near = whole product, and each part against the oracle's own split."""
    test, trial, A, H = c1
    N = _n()
    X = cgauss((1024, 37), 70)  # three 16-column passes
    whole = A @ X
    far, near = N.farmatrix(A), N.nearmatrix(A)
    assert relerr(far @ X + near @ X, whole) < REL
    assert relerr(whole, H.apply(X, 0)) < REL
    y0 = cgauss((1024, 37), 71)
    y = y0.copy()
    N.mul(y, N.adjoint(A), X, 0.5 - 0.25j, 2.0)
    assert relerr(y, (0.5 - 0.25j) * H.apply(X, 2) + 2.0 * y0) < REL
    A.set_profiling(True)
    try:
        A @ X[:, :16]
        st = A.stage_times()
        assert st["near"][1] == 1 and st["leaves"][1] == 1 and st["coupling"][1] == 1
        assert all(t >= 0 for t, _ in st.values())
        far.set_profiling(True)
        far @ X[:, :16]
        sf = far.stage_times()
        assert sf["near"][1] == 0 and sf["leaves"][1] == 1
    finally:
        A.set_profiling(False)


def test_graph_replay_matches_enqueued_products(c1):
    """Repeated products on device arrays replay a CUDA graph from the third identical call on;
    every replay is bitwise the enqueued product, for both orientations alternating, with stage
    timers on, after alpha / beta change and after the workspace's buffers grow."""
    import ctypes as C
    import torch
    test, trial, A, H = c1
    N = _n()
    L = N._lib.lib()
    W = N.H2Workspace(N.core(A), max_nrhs=4)
    W.set_graphs(True)
    E = N.H2Workspace(N.core(A), max_nrhs=4)  # graphs off by default

    def run(ws, mode, X, Y, b, al, be):
        N._lib.check(L.nca_apply(ws._h, mode, 0, C.c_void_p(X.data_ptr()), 1024, C.c_void_p(Y.data_ptr()), 1024, b,
                                 al.real, al.imag, be.real, be.imag, 1))
        torch.cuda.synchronize()

    X = torch.from_numpy(np.ascontiguousarray(cgauss((1024, 20), 80).T)).cuda()
    Y0 = torch.from_numpy(np.ascontiguousarray(cgauss((1024, 20), 81).T)).cuda()
    for b, al, be in ((4, 1 + 0j, 0j), (4, 0.5 - 1j, 2 + 0.5j), (20, 1 + 0j, 0j)):
        for rep in range(4):
            for mode in (0, 2):
                Yg, Ye = Y0.clone(), Y0.clone()
                run(W, mode, X, Yg, b, al, be)
                run(E, mode, X, Ye, b, al, be)
                assert torch.equal(Yg, Ye), (b, rep, mode)
        ref = H.apply(X[:b].cpu().numpy().T, 0)
        Yg = Y0.clone()
        run(W, 0, X, Yg, b, al, be)
        assert relerr(Yg[:b].cpu().numpy().T, al * ref + be * Y0[:b].cpu().numpy().T) < REL
    W.set_profiling(True)
    for rep in range(3):
        Yg = Y0.clone()
        run(W, 0, X, Yg, 4, 1 + 0j, 0j)
        st = W.stage_times()
        assert st["near"][1] == 1 and st["near"][0] > 0 and st["leaves"][0] > 0
    W.set_profiling(False)


def test_autotune_keeps_results(c1):
    """The schedule autotuner picks one of four schedules; products afterwards still match the
    oracle (and each other bitwise across repeated calls)."""
    test, trial, A, H = c1
    N = _n()
    W = N.H2Workspace(N.core(A), max_nrhs=8)
    choice = W.autotune(0, 8)
    assert set(choice) == {"overlap", "graphs"}
    X = cgauss((1024, 8), 90)
    assert relerr(W @ X, H.apply(X, 0)) < REL
    assert np.array_equal(W @ X, W @ X)
    assert relerr(W.H @ X, H.apply(X, 2)) < REL


def test_two_workspaces_on_two_threads(c1):
    """Workspaces of one core run products at the same time from two host threads (each its own
    streams and buffers, the core read-only): every result equals the one computed alone."""
    import threading
    test, trial, A, H = c1
    N = _n()
    X = [cgauss((1024, 5), 100 + i) for i in range(2)]
    ref = [H.apply(x, 0) for x in X]
    W = [N.H2Workspace(N.core(A), max_nrhs=5) for _ in range(2)]
    out = [None, None]
    err = []

    def work(i):
        try:
            for _ in range(20):
                out[i] = W[i] @ X[i]
        except Exception as e:  # reported below
            err.append(e)

    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not err
    for i in range(2):
        assert relerr(out[i], ref[i]) < REL
        assert np.array_equal(out[i], W[i] @ X[i])
