"""Level seams on caller-given data: batched fully pivoted ACA, the interpolation solve and
entry evaluation, each one device launch (ext/NestedCrossApproximationCUDAExt/compresslevel.jl
`_compress` / `_solve_transposed_factors`; AbstractKernelMatrix entry evaluation)."""
from __future__ import annotations

import numpy as np

from ._lib import check, lib, ptr


def _pack(blocks, width=None):
    rows = [b.shape[0] for b in blocks]
    width = width or max([b.shape[1] for b in blocks] + [1])
    off = np.zeros(len(blocks) + 1, dtype=np.int64)
    np.cumsum(rows, out=off[1:])
    buf = np.zeros((max(int(off[-1]), 1), width), dtype=np.complex128, order="F")
    for i, b in enumerate(blocks):
        buf[off[i]:off[i + 1], :b.shape[1]] = b
    return buf, off


def blocks_aca(blocks, maxrank, tol, sampled=True, device=0):
    """ACA(FullPivoting(), FullPivoting(), FNormEstimator(tol)) on every block in one launch:
    (ranks, rowpivots, colpivots) with 0-based local pivots."""
    blocks = [np.asfortranarray(b, dtype=np.complex128) for b in blocks]
    buf, off = _pack(blocks)
    ncols = np.array([b.shape[1] for b in blocks], dtype=np.int32)
    nb = len(blocks)
    ranks = np.zeros(max(nb, 1), np.int32)
    rp = np.zeros((max(nb, 1), maxrank), np.int32)
    cp = np.zeros((max(nb, 1), maxrank), np.int32)
    check(lib().nca_blocks_aca(ptr(buf), buf.shape[0], buf.shape[1], ptr(off), ptr(ncols), nb, int(maxrank),
                               float(tol), int(sampled), int(device), ptr(ranks), ptr(rp), ptr(cp)))
    return ranks[:nb], [rp[i, :ranks[i]].copy() for i in range(nb)], [cp[i, :ranks[i]].copy() for i in range(nb)]


def blocks_factors(blocks, ranks, rowpivots, colpivots, maxrank, device=0, width=None):
    """Z_i = (L_i P_i^{-1})^T, L_i = A_i[:, colpivots], P_i = L_i[rowpivots, :] (rank_i x m_i)."""
    blocks = [np.asfortranarray(b, dtype=np.complex128) for b in blocks]
    buf, off = _pack(blocks, width)
    nb = len(blocks)
    rk = np.asarray(ranks, dtype=np.int32)
    rp = np.full((max(nb, 1), maxrank), -1, np.int32)
    cp = np.full((max(nb, 1), maxrank), -1, np.int32)
    for i in range(nb):
        rp[i, :rk[i]] = rowpivots[i][:rk[i]]
        cp[i, :rk[i]] = colpivots[i][:rk[i]]
    sizes = [int(rk[i]) * b.shape[0] for i, b in enumerate(blocks)]
    zoff = np.zeros(nb + 1, dtype=np.int64)
    np.cumsum(sizes, out=zoff[1:])
    Z = np.zeros(max(int(zoff[-1]), 1), dtype=np.complex128)
    check(lib().nca_blocks_factors(ptr(buf), buf.shape[0], buf.shape[1], ptr(off), nb, ptr(rk), ptr(rp), ptr(cp),
                                   int(maxrank), int(device), ptr(zoff), ptr(Z)), kind="nested_test_basis")
    return [Z[zoff[i]:zoff[i + 1]].reshape((int(rk[i]), blocks[i].shape[0]), order="F") for i in range(nb)]


def entries(kernel, testpoints, trialpoints, ii, jj, device=0, dk=False):
    """Kernel entries A(ii[e], jj[e]) evaluated on the device (dk=True: their d/dk)."""
    tp = np.ascontiguousarray(testpoints, dtype=np.float64).reshape(-1, 3)
    sp = np.ascontiguousarray(trialpoints, dtype=np.float64).reshape(-1, 3)
    ii = np.ascontiguousarray(ii, dtype=np.int64)
    jj = np.ascontiguousarray(jj, dtype=np.int64)
    out = np.zeros(max(len(ii), 1), dtype=np.complex128)
    d = kernel.desc()
    import ctypes as C
    f = lib().nca_entries_dk if dk else lib().nca_entries
    check(f(C.byref(d), ptr(tp), len(tp), ptr(sp), len(sp), ptr(ii), ptr(jj), len(ii), int(device), ptr(out)))
    return out[:len(ii)]
