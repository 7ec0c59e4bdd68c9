"""GPU: the allocation-free product nca_apply_static against the workspace product nca_apply.

Both run the same kernels in the same order, so the bar is the product bar of the parity suite
(relative 1e-12); the scratch array is reused across calls and cores, so results must not
depend on what an earlier call left in it. This file is collected last so that it also runs
after every other GPU test in one process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cgauss, grid_c1, sphere

pytestmark = pytest.mark.gpu

REL = 1e-12
SCRATCH = 32 << 20  # NCA_STATIC_SCRATCH_BYTES
PREC_F64 = 0


def _n():
    import nca_b200
    return nca_b200


def build(test, trial, k, tol, minvalues, maxrank=50):
    N = _n()
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=minvalues))
    st = N.KMeansTree(trial, N.KMeansTreeBuilder(minvalues=minvalues))
    tree = N.BlockTree(tt, st)
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(tol))
    tc = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(test, trial, st), compressor=aca)
    sc = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(trial, test, tt), compressor=aca)
    A = N.PetrovGalerkinNCA(N.HelmholtzKernel(k), test, trial, tree, testcompressor=tc, trialcompressor=sc,
                            maxrank=maxrank)
    return N.core(A)


@pytest.fixture(scope="module")
def cores():
    test, trial = grid_c1()
    a = build(test, trial, 2 * np.pi / 10, 1e-4, 32)
    b = build(sphere(2048, 31), sphere(1500, 32) * 1.3, 3.0, 1e-6, 40, maxrank=40)
    return a, b


def dims(core, mode):
    ntest, ntrial = core.dim
    return (ntrial, ntest) if mode == 0 else (ntest, ntrial)


def device_cols(M):
    """Column-major complex128 device array of M (n x b) as a (b, n) row-major tensor."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(M.T)).cuda()


def call_static(core, mode, X, Y, alpha, beta, stream=None):
    N = _n()
    nin, nout = dims(core, mode)
    b = X.shape[0]
    return N._lib.lib().nca_apply_static(core._h, mode, PREC_F64, C.c_void_p(X.data_ptr()), nin,
                                         C.c_void_p(Y.data_ptr()), nout, b, alpha.real, alpha.imag, beta.real,
                                         beta.imag, C.c_void_p(stream) if stream else None)


def call_workspace(ws, mode, X, Y, alpha, beta):
    N = _n()
    nin, nout = dims(ws.core, mode)
    N._lib.check(N._lib.lib().nca_apply(ws._h, mode, PREC_F64, C.c_void_p(X.data_ptr()), nin,
                                        C.c_void_p(Y.data_ptr()), nout, X.shape[0], alpha.real, alpha.imag,
                                        beta.real, beta.imag, 1))


def relerr(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("b", [1, 3, 16, 19])
def test_static_matches_workspace(cores, b):
    import torch
    N = _n()
    for ci, core in enumerate(cores):
        ws = N.H2Workspace(core, max_nrhs=b)
        for mode in (0, 1, 2):
            nin, nout = dims(core, mode)
            X = device_cols(cgauss((nin, b), 100 + 10 * ci + mode))
            Y0 = device_cols(cgauss((nout, b), 200 + 10 * ci + mode))
            alpha, beta = complex(0.7, -0.3), (complex(-1.1, 0.4) if mode == 1 else 0j)
            ref = Y0.clone()
            call_workspace(ws, mode, X, ref, alpha, beta)
            torch.cuda.synchronize()
            # two calls in a row on fresh output copies
            for _ in range(2):
                Y = Y0.clone()
                torch.cuda.synchronize()
                N._lib.check(call_static(core, mode, X, Y, alpha, beta))
                assert relerr(Y, ref) < REL, (ci, mode, b)


def test_static_alternating_cores_and_streams(cores):
    """The scratch holds another core's data between calls; results stay those of nca_apply.
    A non-default stream is used for half the calls."""
    import torch
    N = _n()
    s = torch.cuda.Stream()
    refs = []
    for ci, core in enumerate(cores):
        nin, nout = dims(core, 0)
        X = device_cols(cgauss((nin, 5), 300 + ci))
        ref = torch.zeros((5, nout), dtype=torch.complex128, device="cuda")
        call_workspace(N.H2Workspace(core, max_nrhs=5), 0, X, ref, 1 + 0j, 0j)
        refs.append((core, X, ref))
    torch.cuda.synchronize()
    for it in range(4):
        for core, X, ref in (refs if it % 2 == 0 else refs[::-1]):
            Y = torch.full_like(ref, float("nan"))
            torch.cuda.synchronize()
            N._lib.check(call_static(core, 0, X, Y, 1 + 0j, 0j, s.cuda_stream if it >= 2 else None))
            assert relerr(Y, ref) < REL


def test_static_allocates_no_device_memory(cores):
    import torch
    N = _n()
    core = cores[1]
    nin, nout = dims(core, 2)
    X = device_cols(cgauss((nin, 16), 400))
    Y = torch.zeros((16, nout), dtype=torch.complex128, device="cuda")
    N._lib.check(call_static(core, 2, X, Y, 1 + 0j, 0j))  # setup and kernel loading happen here
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        N._lib.check(call_static(core, 2, X, Y, 1 + 0j, 0j))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_rejections(cores):
    import torch
    N = _n()
    core = cores[0]
    nin, nout = dims(core, 0)
    info = core.info
    per_rhs = 16 * (nin + info.ncoeff_test + info.ncoeff_trial)
    b = SCRATCH // per_rhs + 8
    X = torch.zeros((b, nin), dtype=torch.complex128, device="cuda")
    Y = torch.zeros((b, nout), dtype=torch.complex128, device="cuda")
    st = call_static(core, 0, X, Y, 1 + 0j, 0j)
    assert st == N._lib.NCA_ERR_ARG
    msg = N._lib.last_error()
    assert "NCA_STATIC_SCRATCH_BYTES" in msg and str(SCRATCH) in msg
    # the largest accepted count still works
    ok = SCRATCH // per_rhs - 8
    ref = torch.zeros((ok, nout), dtype=torch.complex128, device="cuda")
    call_workspace(N.H2Workspace(core, max_nrhs=ok), 0, X[:ok], ref, 1 + 0j, 0j)
    Yok = torch.zeros_like(ref)
    N._lib.check(call_static(core, 0, X[:ok], Yok, 1 + 0j, 0j))
    assert torch.equal(Yok, ref) or relerr(Yok, ref) < REL
    # misaligned device pointer, short leading dimension, bad mode: refused before any launch
    lib = N._lib.lib()
    st = lib.nca_apply_static(core._h, 0, 0, C.c_void_p(X.data_ptr() + 8), nin, C.c_void_p(Y.data_ptr()), nout, 1,
                              1.0, 0.0, 0.0, 0.0, None)
    assert st == N._lib.NCA_ERR_ARG
    st = lib.nca_apply_static(core._h, 0, 0, C.c_void_p(X.data_ptr()), nin - 1, C.c_void_p(Y.data_ptr()), nout, 1,
                              1.0, 0.0, 0.0, 0.0, None)
    assert st == N._lib.NCA_ERR_DIM
    st = lib.nca_apply_static(core._h, 5, 0, C.c_void_p(X.data_ptr()), nin, C.c_void_p(Y.data_ptr()), nout, 1,
                              1.0, 0.0, 0.0, 0.0, None)
    assert st == N._lib.NCA_ERR_ARG


def _cudart():
    """The CUDA runtime that torch has loaded (by soname), for stream creation and host functions."""
    return C.CDLL("libcudart.so.12")


def test_static_refuses_directional_cores():
    """Directional (wideband) cores go through nca_apply only."""
    import torch
    N = _n()
    pts = sphere(1500, 61)
    t = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=32))
    conv = N.FNormExtrapolator(1e-4)
    A = N.PetrovGalerkinNCA(
        N.HelmholtzKernel(12.0, rmin=1e-12), pts, pts, N.BlockTree(t, t), isnear=N.isnearwideband(12.0),
        testcompressor=N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(pts, pts, t), conv)),
        trialcompressor=N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(pts, pts, t), N.MaximumValue(), conv)))
    X = device_cols(cgauss((1500, 1), 62))
    Y = torch.zeros_like(X)
    assert call_static(N.core(A), 0, X, Y, 1 + 0j, 0j) == N._lib.NCA_ERR_ARG
    assert "directional" in N._lib.last_error()


def test_static_refuses_stream_capture(cores):
    """The call waits for its stream, so on a capturing stream it is refused before any work and
    the capture stays valid."""
    import torch
    N = _n()
    core = cores[0]
    nin, nout = dims(core, 0)
    X = device_cols(cgauss((nin, 2), 71))
    Y = torch.zeros((2, nout), dtype=torch.complex128, device="cuda")
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        st = call_static(core, 0, X, Y, 1 + 0j, 0j, torch.cuda.current_stream().cuda_stream)
        Y.add_(1.0)
    assert st == N._lib.NCA_ERR_ARG
    assert "captured" in N._lib.last_error()
    g.replay()
    torch.cuda.synchronize()
    assert torch.all(Y == 1.0)


def test_static_overlapping_calls_are_refused(cores):
    """A call that holds the scratch (its stream held up by a host function that waits, with a
    timeout, on a host event) makes a second call from another thread return NCA_ERR_BUSY; once
    the event is set, the first call completes with the product of nca_apply. Only the host
    waits: no kernel spins."""
    import threading
    import time
    import torch
    N = _n()
    rt = _cudart()
    core = cores[0]
    nin, nout = dims(core, 0)
    X = device_cols(cgauss((nin, 3), 81))
    ref = torch.zeros((3, nout), dtype=torch.complex128, device="cuda")
    call_workspace(N.H2Workspace(core, max_nrhs=3), 0, X, ref, 1 + 0j, 0j)
    torch.cuda.synchronize()
    streams = []
    for _ in range(2):
        h = C.c_void_p()
        assert rt.cudaStreamCreateWithFlags(C.byref(h), 1) == 0  # cudaStreamNonBlocking
        streams.append(h)
    release = threading.Event()
    HOSTFN = C.CFUNCTYPE(None, C.c_void_p)
    hold = HOSTFN(lambda _: release.wait(10.0))
    Ya = torch.zeros_like(ref)
    Yb = torch.zeros_like(ref)
    out = {}
    try:
        assert rt.cudaLaunchHostFunc(streams[0], hold, None) == 0
        thread_a = threading.Thread(target=lambda: out.setdefault("a", call_static(core, 0, X, Ya, 1 + 0j, 0j,
                                                                                   streams[0].value)))
        thread_a.start()
        busy = False
        t_end = time.time() + 5.0
        while time.time() < t_end and not busy:
            st = call_static(core, 0, X, Yb, 1 + 0j, 0j, streams[1].value)
            busy = st == N._lib.NCA_ERR_BUSY
            if not busy:
                assert st == N._lib.NCA_OK
                time.sleep(0.001)
        assert busy, "the second call was never refused"
        assert "another call" in N._lib.last_error()
    finally:
        release.set()
        thread_a.join(30.0)
        for h in streams:
            rt.cudaStreamSynchronize(h)
            rt.cudaStreamDestroy(h)
    assert out.get("a") == N._lib.NCA_OK
    assert relerr(Ya, ref) < REL
