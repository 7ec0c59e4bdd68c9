"""Serialised cores: nca_core_save / nca_core_load (the reference dumps a built matrix's stores
and plans for reuse across runs, scripts/create_test_matrix.jl:50-68). A loaded core rebuilds its
couplings, near field and product plans from the saved skeleton, so its products must equal the
saved core's bit for bit, in every mode and stored precision."""
import os

import numpy as np
import pytest

from conftest import cgauss, grid_c1, sphere

pytestmark = pytest.mark.gpu


def _n():
    import nca_b200
    return nca_b200


def _products(A, ntest, ntrial, f32=False):
    N = _n()
    W = N.H2Workspace(N.core(A) if isinstance(A, N.H2Workspace) else A, np.complex64 if f32 else np.complex128)
    X = cgauss((ntrial, 3), 5)
    U = cgauss((ntest, 3), 6)
    return [W @ X, W.T @ U, W.H @ U]


def _roundtrip(tmp_path, A, ntest, ntrial, f32=False):
    N = _n()
    core = N.core(A)
    path = os.path.join(str(tmp_path), "core.nca")
    core.save(path)
    L = N.load_core(path)
    assert L.dim == core.dim
    for name in ("near_entries", "coupling_entries", "ncoeff_test", "ncoeff_trial", "basis_entries_test",
                 "transfer_entries_trial"):
        assert getattr(L.info, name) == getattr(core.info, name), name
    for a, b in zip(_products(core, ntest, ntrial), _products(L, ntest, ntrial)):
        assert np.array_equal(a, b)
    if f32:
        for a, b in zip(_products(core, ntest, ntrial, True), _products(L, ntest, ntrial, True)):
            assert np.array_equal(a, b)
    return core, L


def test_batched_core_roundtrip(tmp_path):
    N = _n()
    test, trial = grid_c1()
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=32))
    st = N.KMeansTree(trial, N.KMeansTreeBuilder(minvalues=32))
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-4))
    A = N.PetrovGalerkinNCA(N.HelmholtzKernel(2 * np.pi / 10), test, trial, N.BlockTree(tt, st),
                            testcompressor=N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(test, trial, st),
                                                             compressor=aca),
                            trialcompressor=N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(trial, test, tt),
                                                              compressor=aca), store_f32=True)
    core, L = _roundtrip(tmp_path, A, 1024, 1024, f32=True)
    for side in (0, 1):
        p0, r0, n0 = core.pivots(side)
        p1, r1, n1 = L.pivots(side)
        assert np.array_equal(r0, r1) and np.array_equal(n0, n1)
        assert all((a is None and b is None) or np.array_equal(a, b) for a, b in zip(p0, p1))


def test_bottomup_iaca_and_directional_roundtrip(tmp_path):
    N = _n()
    pts = sphere(4096, 9)
    t = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=32))
    conv = N.FNormExtrapolator(1e-5)
    tc = N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(pts, pts, t), conv))
    sc = N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(pts, pts, t), N.MaximumValue(), conv))
    A = N.PetrovGalerkinNCA(N.HelmholtzKernel(2.0, rmin=1e-12), pts, pts, N.BlockTree(t, t), testcompressor=tc,
                            trialcompressor=sc)
    _roundtrip(tmp_path, A, 4096, 4096)
    B = N.PetrovGalerkinNCA(N.HelmholtzKernel(14.0, rmin=1e-12), pts, pts, N.BlockTree(t, t),
                            isnear=N.isnearwideband(14.0), testcompressor=tc, trialcompressor=sc, store_f32=True)
    core, L = _roundtrip(tmp_path, B, 4096, 4096, f32=True)
    import ctypes as C
    for side in (0, 1):
        n0, n1 = C.c_int32(), C.c_int32()
        N._lib.check(N.lib().nca_core_dir_items(core._h, side, C.byref(n0), None, None, None, None))
        N._lib.check(N.lib().nca_core_dir_items(L._h, side, C.byref(n1), None, None, None, None))
        assert n0.value == n1.value > 0


def test_batches_are_not_saved(tmp_path):
    N = _n()
    test, trial = grid_c1()
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=32))
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-4))
    comp = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(test, test, tt), compressor=aca)
    A = N.PetrovGalerkinNCA(N.HelmholtzKernel(1.0, rmin=1e-12), test, test, N.BlockTree(tt, tt), testcompressor=comp,
                            trialcompressor=comp)
    b = N.batch([A])
    with pytest.raises(N.ArgumentError, match="batch"):
        b.save(os.path.join(str(tmp_path), "b.nca"))
