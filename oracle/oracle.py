"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates NestedCrossApproximation.jl's batched bottom-up build and H^2 product
in plain C (``nca_oracle.c``, see its header for the reference files it follows). Only the
tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py`` import this
module; the library under ``nestedcrossapproximation.jl_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_build", "libnca_oracle.so")

KIND_HELMHOLTZ, KIND_LAPLACE, KIND_MATRIX = 0, 1, 2

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(LIBPATH) or os.path.getmtime(LIBPATH) < os.path.getmtime(
        os.path.join(HERE, "nca_oracle.c")
    ):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIBPATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            build()
        L = C.CDLL(LIBPATH)
        P, I, D, LG = C.c_void_p, C.c_int, C.c_double, C.c_long
        L.oracle_build.restype = P
        L.oracle_build.argtypes = [P, LG, P, LG, I, D, I, I, D, D, P, LG, D, D, I, I, I, I]
        L.oracle_free.argtypes = [P]
        L.oracle_status.argtypes = [P, P, P, P, P]
        L.oracle_tree.restype = P
        L.oracle_tree.argtypes = [P, I]
        L.oracle_tree_build.restype = P
        L.oracle_tree_build.argtypes = [P, LG, I]
        L.oracle_tree_free.argtypes = [P]
        L.oracle_tree_nnodes.argtypes = [P]
        L.oracle_tree_nlevels.argtypes = [P]
        L.oracle_tree_export.argtypes = [P] * 10
        L.oracle_partition_sizes.argtypes = [P, P, P]
        L.oracle_partition.argtypes = [P] * 7
        L.oracle_farpivots_total.argtypes = [P, I]
        L.oracle_farpivots.argtypes = [P, I, P, P]
        L.oracle_pivots_total.argtypes = [P, I]
        L.oracle_pivots.argtypes = [P, I, P, P, P, P]
        L.oracle_x_total.restype = LG
        L.oracle_x_total.argtypes = [P, I]
        L.oracle_x.argtypes = [P, I, P, P]
        L.oracle_coupling_total.restype = LG
        L.oracle_coupling_total.argtypes = [P]
        L.oracle_couplings.argtypes = [P, P, P]
        L.oracle_near_total.restype = LG
        L.oracle_near_total.argtypes = [P]
        L.oracle_near.argtypes = [P, P, P, P]
        L.oracle_apply.argtypes = [P, I, P, LG, P, LG, LG]
        L.oracle_dense_rows.argtypes = [I, I, D, D, P, LG, P, P, LG, P, LG, I, P, P, I]
        L.oracle_sincos.argtypes = [D, P, P]
        L.oracle_entries.argtypes = [I, I, D, D, P, LG, P, P, P, P, LG, P]
        L.oracle_aca.argtypes = [P, I, I, I, D, I, P, P]
        L.oracle_cross_solve.argtypes = [P, I, I, P, P, P]
        L.oracle_select_farpivots.argtypes = [P, P, P, P, I, P, I, I, P]
        L.oracle_iaca.argtypes = [P, P, P, I, I, D, D, P, LG, I, P, I, P, I, P, I, I, D, P, P, P, P]
        L.oracle_dir_build.restype = P
        L.oracle_dir_build.argtypes = [P, LG, P, LG, I, D, D, D, D, I, I, D, D, P, LG, D, D, I, I]
        L.oracle_dir_free.argtypes = [P]
        L.oracle_dir_status.argtypes = [P, P, P, P, P]
        L.oracle_dir_tree.restype = P
        L.oracle_dir_tree.argtypes = [P, I]
        L.oracle_dir_nitems.argtypes = [P, I]
        L.oracle_dir_nfar.restype = LG
        L.oracle_dir_nfar.argtypes = [P, I]
        L.oracle_dir_nchildren.argtypes = [P, I]
        L.oracle_dir_plan.argtypes = [P, I] + [P] * 8
        L.oracle_dir_pivots.argtypes = [P, I, P, P, P, P]
        L.oracle_dir_x_total.restype = LG
        L.oracle_dir_x_total.argtypes = [P, I]
        L.oracle_dir_x.argtypes = [P, I, P, P]
        L.oracle_dir_sizes.argtypes = [P, P, P, P, P]
        L.oracle_dir_apply.argtypes = [P, I, P, LG, P, LG, LG]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def sincos(x: float):
    s, c = C.c_double(), C.c_double()
    lib().oracle_sincos(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


class Kernel:
    """Kernel spec: Helmholtz cis(sign k r)/(4 pi r), Laplace 1/(4 pi r), or a dense matrix."""

    def __init__(self, kind=KIND_HELMHOLTZ, k=0.0, sign=1, rmin=0.0, matrix=None):
        self.kind, self.k, self.sign, self.rmin = kind, float(k), int(sign), float(rmin)
        self.matrix = None if matrix is None else np.asfortranarray(matrix, dtype=np.complex128)

    def args(self):
        if self.matrix is None:
            return (self.kind, self.sign, self.k, self.rmin, None, 0)
        return (self.kind, self.sign, self.k, self.rmin, _p(self.matrix), self.matrix.shape[0])


def entries(kernel: Kernel, xs, ys, ii, jj):
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    ys = np.ascontiguousarray(ys, dtype=np.float64)
    ii = np.ascontiguousarray(ii, dtype=np.int64)
    jj = np.ascontiguousarray(jj, dtype=np.int64)
    out = np.empty(len(ii), dtype=np.complex128)
    lib().oracle_entries(*kernel.args(), _p(xs), _p(ys), _p(ii), _p(jj), len(ii), _p(out))
    return out


def aca(block, maxrank, tol, sampled=True):
    """Fully pivoted ACA on a dense block: (rank, rowpivots, colpivots), 0-based."""
    A = np.asfortranarray(block, dtype=np.complex128)
    m, n = A.shape
    rp = np.zeros(max(maxrank, 1), dtype=np.int32)
    cp = np.zeros(max(maxrank, 1), dtype=np.int32)
    r = lib().oracle_aca(_p(A), m, n, maxrank, float(tol), int(sampled), _p(rp), _p(cp))
    return r, rp[:r].copy(), cp[:r].copy()


class SingularCross(Exception):
    def __init__(self, npivots, rank):
        super().__init__(f"singular cross matrix: {npivots} pivots, rank {rank}")
        self.npivots, self.rank = npivots, rank


def cross_solve(L, rows):
    """X = L P^{-1} with P = L[rows, :] (the interpolation operator of a cluster)."""
    L = np.asfortranarray(L, dtype=np.complex128)
    m, r = L.shape
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    X = np.zeros((m, r), dtype=np.complex128, order="F")
    rank = C.c_int()
    st = lib().oracle_cross_solve(_p(L), m, r, _p(rows), _p(X), C.byref(rank))
    if st:
        raise SingularCross(r, rank.value)
    return X


class Tree:
    """Export of an oracle k-means tree (0-based node ids, BFS order)."""

    def __init__(self, ptr, npts, owner=None):
        L = lib()
        self._ptr, self._owner = ptr, owner
        nn = L.oracle_tree_nnodes(ptr)
        self.nnodes, self.nlevels = nn, L.oracle_tree_nlevels(ptr)
        self.perm = np.zeros(npts, dtype=np.int32)
        ints = [np.zeros(nn, dtype=np.int32) for _ in range(6)]
        self.center = np.zeros((nn, 3))
        self.radius = np.zeros(nn)
        L.oracle_tree_export(ptr, _p(self.perm), *[_p(a) for a in ints], _p(self.center), _p(self.radius))
        self.begin, self.end, self.parent, self.firstchild, self.nchildren, self.level = ints

    def values(self, node):
        return self.perm[self.begin[node]:self.end[node]]

    def children(self, node):
        return list(range(self.firstchild[node], self.firstchild[node] + self.nchildren[node]))

    def isleaf(self, node):
        return self.nchildren[node] == 0


class OwnedTree(Tree):
    def __init__(self, pts, minvalues):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        ptr = lib().oracle_tree_build(_p(pts), len(pts), int(minvalues))
        super().__init__(ptr, len(pts))
        self._pts = pts

    def __del__(self):
        if getattr(self, "_ptr", None):
            lib().oracle_tree_free(self._ptr)
            self._ptr = None


def select_farpivots(fartree: OwnedTree, ownpts, farpts, refidcs, farnodes, maxrank):
    ownpts = np.ascontiguousarray(ownpts, dtype=np.float64)
    farpts = np.ascontiguousarray(farpts, dtype=np.float64)
    ref = np.ascontiguousarray(refidcs, dtype=np.int32)
    fn = np.ascontiguousarray(farnodes, dtype=np.int32)
    out = np.zeros(max(maxrank, 1), dtype=np.int32)
    n = lib().oracle_select_farpivots(
        fartree._ptr, _p(ownpts), _p(farpts), _p(ref), len(ref), _p(fn), len(fn), int(maxrank), _p(out)
    )
    return out[:n].copy()


def iaca(fartree: OwnedTree, kernel: Kernel, ownpts, farpts, refidcs, rows, farnodes, maxrank, tol, side=0):
    """IACA of K[rows, far field] with tree-mimicry columns over `farnodes` (centroid of the
    points `refidcs`): (rank, local row pivots, far column pivots, X = K[rows, sigma] K[tau, sigma]^-1)."""
    ownpts = np.ascontiguousarray(ownpts, dtype=np.float64)
    farpts = np.ascontiguousarray(farpts, dtype=np.float64)
    ref = np.ascontiguousarray(refidcs, dtype=np.int32)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    fn = np.ascontiguousarray(farnodes, dtype=np.int32)
    m = len(rows)
    lim = max(min(maxrank, m), 1)
    rp = np.zeros(lim, np.int32)
    cp = np.zeros(lim, np.int32)
    X = np.zeros(m * lim + 1, np.complex128)
    nr = C.c_int()
    r = lib().oracle_iaca(fartree._ptr, _p(ownpts), _p(farpts), *kernel.args(), int(side), _p(ref), len(ref),
                          _p(rows), m, _p(fn), len(fn), int(maxrank), float(tol), _p(rp), _p(cp), _p(X),
                          C.byref(nr))
    if r < 0:
        raise SingularCross(lim, nr.value)
    return r, rp[:r].copy(), cp[:r].copy(), X[:m * r].reshape((m, r), order="F").copy()


class SingularBuild(Exception):
    pass


class H2:
    """Oracle H^2 build and its product: the batched bottom-up NCA, or with iaca=True the plain
    BottomUp compressor with IACA per cluster (src/compressors/bottomup.jl:96-208)."""

    def __init__(self, testpts, trialpts, kernel: Kernel, minvalues=32, eta=1.0, tol=1e-4,
                 tol_trial=None, maxrank=50, sampled=True, nthreads=None, iaca=False):
        self.testpts = np.ascontiguousarray(testpts, dtype=np.float64)
        self.trialpts = np.ascontiguousarray(trialpts, dtype=np.float64)
        self.kernel = kernel
        nthreads = nthreads or os.cpu_count() or 1
        if maxrank > 256:
            raise ValueError("the oracle supports maxrank <= 256")
        L = lib()
        self._h = L.oracle_build(
            _p(self.testpts), len(self.testpts), _p(self.trialpts), len(self.trialpts),
            int(minvalues), float(eta), *kernel.args(), float(tol),
            float(tol if tol_trial is None else tol_trial), int(maxrank), int(sampled), int(nthreads),
            int(bool(iaca)),
        )
        side, node, npiv, rank = (C.c_int() for _ in range(4))
        st = L.oracle_status(self._h, C.byref(side), C.byref(node), C.byref(npiv), C.byref(rank))
        self.status = (st, side.value, node.value, npiv.value, rank.value)
        self.trees = [Tree(L.oracle_tree(self._h, s), len(p), self) for s, p in
                      ((0, self.testpts), (1, self.trialpts))]
        if st:
            raise SingularBuild(f"singular cross matrix (side {side.value}, node {node.value}, "
                                f"{npiv.value} pivots, rank {rank.value})")
        nn, nf = C.c_long(), C.c_long()
        L.oracle_partition_sizes(self._h, C.byref(nn), C.byref(nf))
        nt, ns = self.trees[0].nnodes, self.trees[1].nnodes
        self.nearptr = np.zeros(nt + 1, np.int32)
        self.nearnodes = np.zeros(nn.value, np.int32)
        self.farptr = np.zeros(nt + 1, np.int32)
        self.farnodes = np.zeros(nf.value, np.int32)
        self.tfarptr = np.zeros(ns + 1, np.int32)
        self.tfarnodes = np.zeros(nf.value, np.int32)
        L.oracle_partition(self._h, *[_p(a) for a in (self.nearptr, self.nearnodes, self.farptr,
                                                    self.farnodes, self.tfarptr, self.tfarnodes)])
        self.farpivots, self.ranks, self.nrows, self.pivots, self.X = [], [], [], [], []
        for s, tr in enumerate(self.trees):
            tot = L.oracle_farpivots_total(self._h, s)
            ptr = np.zeros(tr.nnodes + 1, np.int32)
            idx = np.zeros(tot, np.int32)
            L.oracle_farpivots(self._h, s, _p(ptr), _p(idx))
            self.farpivots.append([idx[ptr[i]:ptr[i + 1]] for i in range(tr.nnodes)])
            tot = L.oracle_pivots_total(self._h, s)
            rank = np.zeros(tr.nnodes, np.int32)
            nrows = np.zeros(tr.nnodes, np.int32)
            ptr = np.zeros(tr.nnodes + 1, np.int32)
            idx = np.zeros(tot, np.int32)
            L.oracle_pivots(self._h, s, _p(rank), _p(nrows), _p(ptr), _p(idx))
            self.ranks.append(rank)
            self.nrows.append(nrows)
            self.pivots.append([idx[ptr[i]:ptr[i + 1]] for i in range(tr.nnodes)])
            tot = L.oracle_x_total(self._h, s)
            off = np.zeros(tr.nnodes + 1, np.int64)
            X = np.zeros(tot, np.complex128)
            L.oracle_x(self._h, s, _p(off), _p(X))
            self.X.append([X[off[i]:off[i + 1]].reshape((nrows[i], rank[i]), order="F")
                           for i in range(tr.nnodes)])
        tot = L.oracle_coupling_total(self._h)
        off = np.zeros(nf.value + 1, np.int64)
        Cc = np.zeros(tot, np.complex128)
        L.oracle_couplings(self._h, _p(off), _p(Cc))
        self.couplings = []
        for t in range(nt):
            for i in range(self.farptr[t], self.farptr[t + 1]):
                s = self.farnodes[i]
                self.couplings.append(Cc[off[i]:off[i + 1]].reshape(
                    (self.ranks[0][t], self.ranks[1][s]), order="F"))
        tot = L.oracle_near_total(self._h)
        off = np.zeros(nt + 1, np.int64)
        ncols = np.zeros(nt, np.int32)
        Nn = np.zeros(tot, np.complex128)
        L.oracle_near(self._h, _p(off), _p(ncols), _p(Nn))
        tt = self.trees[0]
        self.near = [Nn[off[t]:off[t + 1]].reshape((tt.end[t] - tt.begin[t], ncols[t]), order="F")
                     for t in range(nt)]

    @property
    def shape(self):
        return (len(self.testpts), len(self.trialpts))

    def apply(self, x, mode=0):
        """op(H) x for mode 0 (forward), 1 (transpose), 2 (adjoint); x is a vector or a matrix."""
        x = np.asarray(x, dtype=np.complex128)
        vec = x.ndim == 1
        X = np.asfortranarray(x.reshape(x.shape[0], -1))
        nin, nout = (self.shape[1], self.shape[0]) if mode == 0 else self.shape
        if X.shape[0] != nin:
            raise ValueError("dimension mismatch")
        Y = np.zeros((nout, X.shape[1]), dtype=np.complex128, order="F")
        lib().oracle_apply(self._h, int(mode), _p(X), nin, _p(Y), nout, X.shape[1])
        return Y[:, 0] if vec else Y

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_free(self._h)
            self._h = None


def dense_rows(kernel: Kernel, testpts, trialpts, rows, x, transposed=False, nthreads=None):
    """Rows of the dense FP64 kernel matrix times x (long double accumulation)."""
    tp = np.ascontiguousarray(testpts, dtype=np.float64)
    sp = np.ascontiguousarray(trialpts, dtype=np.float64)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    x = _c128(x)
    y = np.zeros(len(rows), dtype=np.complex128)
    ns = len(tp) if transposed else len(sp)
    lib().oracle_dense_rows(*kernel.args(), _p(tp), _p(sp), ns, _p(rows), len(rows), int(transposed),
                            _p(x), _p(y), int(nthreads or os.cpu_count() or 1))
    return y
