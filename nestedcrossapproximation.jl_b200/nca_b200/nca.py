"""PetrovGalerkinNCA: the H^2 matrix as a linear map (src/nca/petrovgalerkinnca.jl).

`PetrovGalerkinNCACore` runs the whole batched bottom-up build on the GPU
(`nca_core_build`); `H2Workspace` owns the device coefficient buffers and a CUDA stream and
is the linear map: `A @ x`, `mul(y, A, x, alpha, beta)`, `transpose(A)`, `adjoint(A)`,
vectors or blocks of right-hand sides, host (numpy) or device (torch.cuda) arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from ._lib import (ArgumentError, BuildOpts, ConcurrentWorkspaceError, CoreInfo, DimensionMismatch, check, lib,
                   ptr)
from .admissibility import IsNear, IsNearWideband, Partition, isnear as _isnear
from .compressors import ACA, BatchedBottomUp, BottomUp
from .trees import BlockTree
from .utils import CoefficientPlan

PREC_F64, PREC_F32 = 0, 1
MODE_N, MODE_T, MODE_C = 0, 1, 2


class BasisStore:
    """Leaf bases of one side: blocks[i] belongs to plan_nodes[i] ((points, rank) on the test
    side, (rank, points) on the trial side)."""

    def __init__(self, nodes, blocks):
        self.nodes, self.blocks = nodes, blocks


class TransferStore:
    """Transfer matrices level by level: (parent, child, block) with blocks (child rank, parent
    rank) on the test side and (parent rank, child rank) on the trial side."""

    def __init__(self, levelidcs, leveltoidcsptr, idxtochdsptr, chdsidcs, blocks):
        self.levelidcs, self.leveltoidcsptr = levelidcs, leveltoidcsptr
        self.idxtochdsptr, self.chdsidcs, self.blocks = idxtochdsptr, chdsidcs, blocks


class CouplingStore:
    def __init__(self, nodetofarnodesptr, farnodes, blocks):
        self.nodetofarnodesptr, self.farnodes, self.blocks = nodetofarnodesptr, farnodes, blocks


class PetrovGalerkinNCACore:
    """Read-only H^2 matrix built by the batched bottom-up NCA on one GPU."""

    def __init__(self, operator, testspace, trialspace, tree: BlockTree, *, testcompressor, trialcompressor,
                 isnear: IsNear | None = None, maxrank: int = 50, ntasks: int | None = None, store_f32: bool = False,
                 device: int = 0, sampled: bool = True, partition: Partition | None = None, verbose: bool = False):
        if ntasks is not None and ntasks < 1:
            raise ArgumentError(f"ntasks must be positive, got {ntasks}")
        self.isnear = isnear or _isnear()
        wideband = isinstance(self.isnear, IsNearWideband) or (partition is not None and partition.wideband)
        for side, comp in (("test", testcompressor), ("trial", trialcompressor)):
            if wideband and not isinstance(comp, BottomUp):
                # src/compressors/abstractcompressor.jl:39-47
                raise ArgumentError("Wideband (directional) NCA is only supported with BottomUp; got "
                                    f"{type(comp).__name__} as {side} compressor.")
            if isinstance(comp, BatchedBottomUp):
                if not isinstance(comp.compressor, ACA):
                    raise ArgumentError("BatchedBottomUp needs compressor=ACA(FullPivoting(), FullPivoting(), "
                                        "FNormEstimator(tol))")
            elif isinstance(comp, BottomUp):
                if comp.factorization.geometric_side() != (0 if side == "test" else 1):
                    raise ArgumentError(f"the {side} side's IACA has its pivotings swapped: test side "
                                        "IACA(MaximumValue(), TreeMimicryPivoting, conv), trial side "
                                        "IACA(TreeMimicryPivoting, MaximumValue(), conv)")
            else:
                raise ArgumentError("compressors must be BatchedBottomUp(pivotselector=TreeMimicryPivoting, "
                                    "compressor=ACA(...)) or BottomUp(factorization=IACA(...))")
        if type(testcompressor) is not type(trialcompressor):
            raise ArgumentError("the test and trial compressors must be of one kind (both BatchedBottomUp or both "
                                "BottomUp)")
        iaca = isinstance(testcompressor, BottomUp)
        self.operator = operator
        self.testpoints = np.ascontiguousarray(testspace, dtype=np.float64).reshape(-1, 3)
        self.trialpoints = np.ascontiguousarray(trialspace, dtype=np.float64).reshape(-1, 3)
        self.tree = tree
        self.partition = partition or Partition(tree, self.isnear)
        self.maxrank = int(maxrank)
        self.device = int(device)
        self.f32 = bool(store_f32)
        opts = BuildOpts()
        if iaca:
            opts.tol_test = testcompressor.factorization.tol
            opts.tol_trial = trialcompressor.factorization.tol
        else:
            opts.tol_test, opts.tol_trial = testcompressor.compressor.tol, trialcompressor.compressor.tol
        opts.compressor = 1 if iaca else 0
        opts.maxrank, opts.sampled, opts.device, opts.store_f32 = self.maxrank, int(sampled), self.device, int(self.f32)
        desc = operator.desc()
        h = C.c_void_p()
        check(lib().nca_core_build(ptr(self.testpoints), len(self.testpoints), ptr(self.trialpoints),
                                   len(self.trialpoints), tree.test._h, tree.trial._h, self.partition._h,
                                   C.byref(desc), C.byref(opts), C.byref(h)))
        self._h = h
        info = CoreInfo()
        check(lib().nca_core_get_info(h, C.byref(info)))
        self.info = info
        self.dim = (len(self.testpoints), len(self.trialpoints))
        self._cache = {}

    def __del__(self):
        h = self.__dict__.get("_h")
        if h is not None and h.value:
            lib().nca_core_destroy(h)
            self._h = None

    @property
    def shape(self):
        return self.dim

    # ---- serialised cores ----
    def save(self, path):
        """Write the core's inputs and skeleton (points, trees, partition, kernel, pivots and
        interpolation operators) to `path`; `load_core(path)` rebuilds the rest (the reference dumps
        a built matrix's stores and plans, scripts/create_test_matrix.jl:50-68)."""
        check(lib().nca_core_save(self._h, os.fsencode(path)))

    # ---- frozen-skeleton refills and derivatives ----
    @property
    def wavenumber(self):
        return getattr(self.operator, "k", None)

    def set_wavenumber(self, k: float):
        """Refill every store at wavenumber k with the frozen skeleton (tree, ranks and pivots of
        the build); bit-identical to the build at the build's own k."""
        check(lib().nca_core_set_wavenumber(self._h, float(k)))
        op = self.operator
        self.operator = type(op)(float(k), sign=op.sign, rmin=op.rmin)
        self._cache = {}

    def prepare_dk(self):
        """Device stores of dX/dk, dS/dk and dN/dk on the frozen skeleton (for dHdk products)."""
        check(lib().nca_core_prepare_dk(self._h))

    # ---- exports (host copies of the device stores) ----
    def pivots(self, side: int):
        """Pivots per node (None for nodes without far field), ranks and block rows."""
        key = ("piv", side)
        if key not in self._cache:
            tr = self.tree.test if side == 0 else self.tree.trial
            n = tr.nnodes
            ranks, nrows, p = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n + 1, np.int32)
            idx = np.zeros(max(self.maxrank * n, 1), np.int32)
            check(lib().nca_core_export_pivots(self._h, side, ptr(ranks), ptr(nrows), ptr(p), ptr(idx)))
            fp = self.farpivots(side)
            piv = [idx[p[i]:p[i + 1]].copy() if len(fp[i]) else None for i in range(n)]
            self._cache[key] = (piv, ranks, nrows)
        return self._cache[key]

    def farpivots(self, side: int):
        key = ("fp", side)
        if key not in self._cache:
            tr = self.tree.test if side == 0 else self.tree.trial
            tot = C.c_int64()
            check(lib().nca_core_farpivots_total(self._h, side, C.byref(tot)))
            p = np.zeros(tr.nnodes + 1, np.int32)
            idx = np.zeros(max(tot.value, 1), np.int32)
            check(lib().nca_core_export_farpivots(self._h, side, ptr(p), ptr(idx)))
            self._cache[key] = [idx[p[i]:p[i + 1]].copy() for i in range(tr.nnodes)]
        return self._cache[key]

    def interpolation(self, side: int):
        """X_t = A[rows, sigma] A[tau, sigma]^{-1} per node (nrows x rank)."""
        key = ("X", side)
        if key not in self._cache:
            piv, ranks, nrows = self.pivots(side)
            n = len(ranks)
            off = np.zeros(n + 1, np.int64)
            X = np.zeros(max(int(np.dot(ranks.astype(np.int64), nrows)), 1), np.complex128)
            check(lib().nca_core_export_x(self._h, side, ptr(off), ptr(X)))
            self._cache[key] = [X[off[i]:off[i + 1]].reshape((nrows[i], ranks[i]), order="F") for i in range(n)]
        return self._cache[key]

    def _bases(self, side):
        tr = self.tree.test if side == 0 else self.tree.trial
        piv, _, _ = self.pivots(side)
        Xs = self.interpolation(side)
        nodes = [t for t in range(tr.nnodes) if tr.isleaf(t) and piv[t] is not None]
        blocks = [Xs[t] if side == 0 else Xs[t].T for t in nodes]
        return BasisStore(nodes, blocks)

    def _transfers(self, side):
        tr = self.tree.test if side == 0 else self.tree.trial
        piv, ranks, _ = self.pivots(side)
        Xs = self.interpolation(side)
        levelidcs, lptr, cptr, chds, blocks = [], [0], [0], [], []
        for lev in tr.levels():
            for t in tr.levelnodes(lev):
                if tr.isleaf(t) or piv[t] is None:
                    continue
                levelidcs.append(t)
                row = 0
                for ch in tr.children(t):
                    k = int(ranks[ch])
                    E = Xs[t][row:row + k, :]
                    blocks.append(E if side == 0 else E.T)
                    chds.append(ch)
                    row += k
                cptr.append(len(chds))
            lptr.append(len(levelidcs))
        return TransferStore(levelidcs, lptr, cptr, chds, blocks)

    @property
    def nestedtestbases(self):
        return self._bases(0)

    @property
    def nestedtrialbases(self):
        return self._bases(1)

    @property
    def testtransfermatrices(self):
        return self._transfers(0)

    @property
    def trialtransfermatrices(self):
        return self._transfers(1)

    @property
    def couplingmatrices(self):
        if "C" not in self._cache:
            part = self.partition
            off = np.zeros(len(part.farnodes) + 1, np.int64)
            Cf = np.zeros(max(self.info.coupling_entries, 1), np.complex128)
            check(lib().nca_core_export_couplings(self._h, ptr(off), ptr(Cf)))
            _, rt, _ = self.pivots(0)
            _, rs, _ = self.pivots(1)
            blocks = []
            for t in range(self.tree.test.nnodes):
                for i in range(part.farptr[t], part.farptr[t + 1]):
                    s = part.farnodes[i]
                    blocks.append(Cf[off[i]:off[i + 1]].reshape((rt[t], rs[s]), order="F"))
            self._cache["C"] = CouplingStore(part.farptr, part.farnodes, blocks)
        return self._cache["C"]

    @property
    def nearblocks(self):
        """Near-field block rows: list of (rows, cols, block) per test node with near blocks."""
        if "N" not in self._cache:
            part, tt, st = self.partition, self.tree.test, self.tree.trial
            n = tt.nnodes
            off = np.zeros(n + 1, np.int64)
            ncols = np.zeros(n, np.int32)
            Nf = np.zeros(max(self.info.near_entries, 1), np.complex128)
            check(lib().nca_core_export_near(self._h, ptr(off), ptr(ncols), ptr(Nf)))
            out = []
            for t in range(n):
                if part.nearptr[t + 1] == part.nearptr[t]:
                    continue
                rows = tt.values(t)
                cols = np.concatenate([st.values(s) for s in part.nearnodes[part.nearptr[t]:part.nearptr[t + 1]]])
                out.append((rows, cols, Nf[off[t]:off[t + 1]].reshape((len(rows), ncols[t]), order="F")))
            self._cache["N"] = out
        return self._cache["N"]

    @property
    def aggregationplan(self):
        return CoefficientPlan(np.concatenate([[0], np.cumsum(self.pivots(1)[1])]))

    @property
    def disaggregationplan(self):
        return CoefficientPlan(np.concatenate([[0], np.cumsum(self.pivots(0)[1])]))


class LinearMap:
    """Minimal LinearMaps algebra: sums, scalar multiples and products of maps."""

    shape = (0, 0)

    def _apply(self, x, mode):
        raise NotImplementedError

    def __matmul__(self, x):
        if isinstance(x, LinearMap):
            return _Composed(self, x)
        return self._apply(x, MODE_N)

    __mul__ = __matmul__

    def __rmul__(self, a):
        return _Scaled(self, a)

    def __add__(self, other):
        return _Sum(self, other)

    def __sub__(self, other):
        return _Sum(self, _Scaled(other, -1.0))

    @property
    def T(self):
        return _Transposed(self, MODE_T)

    @property
    def H(self):
        return _Transposed(self, MODE_C)


class _Scaled(LinearMap):
    def __init__(self, A, a):
        self.A, self.a, self.shape = A, a, A.shape

    def _apply(self, x, mode):
        a = np.conj(self.a) if mode == MODE_C else self.a
        return a * self.A._apply(x, mode)


class _Sum(LinearMap):
    def __init__(self, A, B):
        self.A, self.B, self.shape = A, B, A.shape

    def _apply(self, x, mode):
        return self.A._apply(x, mode) + self.B._apply(x, mode)


class _Composed(LinearMap):
    def __init__(self, A, B):
        self.A, self.B, self.shape = A, B, (A.shape[0], B.shape[1])

    def _apply(self, x, mode):
        if mode == MODE_N:
            return self.A._apply(self.B._apply(x, MODE_N), MODE_N)
        return self.B._apply(self.A._apply(x, mode), mode)


class _Transposed(LinearMap):
    def __init__(self, A, mode):
        self.A, self.mode = A, mode
        self.shape = (A.shape[1], A.shape[0])

    def _apply(self, x, mode):
        if mode != MODE_N:
            raise ArgumentError("nested transposes are not supported")
        return self.A._apply(x, self.mode)

    @property
    def lmap(self):
        return self.A


class H2Workspace(LinearMap):
    """H^2 matrix as a linear map: a shared read-only core plus this workspace's device
    buffers and stream. One product at a time per workspace (ConcurrentWorkspaceError)."""

    def __init__(self, core: PetrovGalerkinNCACore, dtype=np.complex128, *, max_nrhs: int = 16,
                 parts: str = "all"):
        self.core = core
        self.dtype = np.dtype(dtype)
        if self.dtype not in (np.dtype(np.complex128), np.dtype(np.complex64)):
            raise ArgumentError("H2Workspace element type must be complex128 or complex64")
        self.precision = PREC_F32 if self.dtype == np.complex64 else PREC_F64
        if self.precision == PREC_F32 and not core.f32:
            raise ArgumentError("a complex64 workspace needs a core built with store_f32=True")
        if parts not in ("all", "far", "near"):
            raise ArgumentError("parts must be 'all', 'far' or 'near'")
        self.parts = parts
        h = C.c_void_p()
        check(lib().nca_workspace_create(core._h, int(max_nrhs), C.byref(h)))
        self._h = h
        check(lib().nca_workspace_set_parts(h, int(parts != "near"), int(parts != "far")))
        self._lock = threading.Lock()
        self.shape = core.dim
        self.last_seconds = 0.0

    def __del__(self):
        # the instance's own handle only (a failed __init__ leaves none; never the core's)
        h = self.__dict__.get("_h")
        if h is not None and h.value:
            lib().nca_workspace_destroy(h)
            self._h = None

    @property
    def busy(self):
        return self._lock.locked()

    def __getattr__(self, name):
        core = self.__dict__.get("core")
        if core is None or name.startswith("_"):
            raise AttributeError(name)
        return getattr(core, name)

    def _apply(self, x, mode):
        return mul(None, self if mode == MODE_N else _Transposed(self, mode), x)


    def set_graphs(self, on: bool = True):
        """Replay repeated products on device arrays from CUDA graphs (off by default; pays off for
        launch-bound small problems)."""
        check(lib().nca_workspace_set_graphs(self._h, int(on)))

    def autotune(self, mode: int = MODE_N, nrhs: int = 1):
        """Time the product under each schedule (near field beside or after the sweeps, with or
        without CUDA graphs) and keep the fastest; returns {"overlap": bool, "graphs": bool}."""
        ch = C.c_int32()
        check(lib().nca_workspace_autotune(self._h, int(mode), self.precision, int(nrhs), C.byref(ch)))
        return {"overlap": bool(ch.value & 1), "graphs": bool(ch.value & 2)}

    def set_profiling(self, on: bool = True):
        """Record CUDA events around each stage of every product (see stage_times)."""
        check(lib().nca_workspace_set_profiling(self._h, int(on)))

    def stage_times(self):
        """Device seconds and launches of the last product per stage: gather, upward sweep,
        coupling, downward sweep, near field, leaves. The workspace runs the sweeps on a second
        stream beside the near field (both parts present), then adds the leaf bases ("leaves");
        otherwise the near field is part of the leaf launches and "near" is empty."""
        t = (C.c_double * 6)()
        n = (C.c_int32 * 6)()
        check(lib().nca_workspace_stage_times(self._h, t, n, 6))
        names = ("gather", "upward", "coupling", "downward", "near", "leaves")
        return {k: (t[i], n[i]) for i, k in enumerate(names)}

    def launches(self):
        n = C.c_int32()
        check(lib().nca_workspace_last_launches(self._h, C.byref(n)))
        return n.value


def farmatrix(h2mat: H2Workspace) -> H2Workspace:
    """The far field of h2mat as a workspace with an empty near field; the stores are shared,
    the buffers are not (petrovgalerkinnca.jl:344-362)."""
    return H2Workspace(h2mat.core, h2mat.dtype, parts="far")


def nearmatrix(h2mat: H2Workspace) -> H2Workspace:
    """The near field of h2mat as a linear map (its dense blocks: core.nearblocks)."""
    return H2Workspace(h2mat.core, h2mat.dtype, parts="near")


def withworkspace(f, ws: H2Workspace):
    """Run f as the only product on ws; fails instead of waiting (petrovgalerkinnca.jl:293-300)."""
    if not ws._lock.acquire(blocking=False):
        raise ConcurrentWorkspaceError()
    try:
        return f()
    finally:
        ws._lock.release()


def _unwrap(A):
    if isinstance(A, H2Workspace):
        return A, MODE_N
    if isinstance(A, _Transposed) and isinstance(A.A, H2Workspace):
        return A.A, A.mode
    raise ArgumentError("mul needs an H2Workspace, its transpose or its adjoint")


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _product(ws, mode, xp, nin, yp, nout, nrhs, al, be, memspace, tangent):
    if tangent:
        return lib().nca_apply_dk(ws._h, xp, nin, yp, nout, nrhs, al.real, al.imag, be.real, be.imag, memspace)
    return lib().nca_apply(ws._h, mode, ws.precision, xp, nin, yp, nout, nrhs, al.real, al.imag, be.real, be.imag,
                           memspace)


def mul(y, A, x, alpha=1.0, beta=0.0, _tangent=False):
    """y = alpha op(A) x + beta y (LinearMaps' 5-argument mul!). y None allocates it."""
    ws, mode = _unwrap(A)
    if _tangent and (mode != MODE_N or ws.precision != PREC_F64):
        raise ArgumentError("the d/dk product is forward mode on a complex FP64 workspace")
    core = ws.core
    nin = core.dim[1] if mode == MODE_N else core.dim[0]
    nout = core.dim[0] if mode == MODE_N else core.dim[1]
    if _is_torch(x) and x.is_cuda:
        import torch
        vec = x.dim() == 1
        Xr = x.reshape(x.shape[0], -1).to(torch.complex128).t().contiguous()  # (nrhs, nin): column-major block
        if Xr.shape[1] != nin:
            raise DimensionMismatch(f"x has {Xr.shape[1]} rows, the operator {nin} columns")
        nrhs = Xr.shape[0]
        if y is None:
            Yr = torch.zeros((nrhs, nout), dtype=torch.complex128, device=x.device)
            beta = 0.0
        else:
            Yr = y.reshape(nout, -1).t().contiguous()
        if not ws._lock.acquire(blocking=False):
            raise ConcurrentWorkspaceError()
        try:
            al, be = complex(alpha), complex(beta)
            check(_product(ws, mode, C.c_void_p(Xr.data_ptr()), nin, C.c_void_p(Yr.data_ptr()), nout, nrhs, al, be,
                           1, _tangent))
        finally:
            ws._lock.release()
        out = Yr.t()
        if y is not None:
            y.copy_(out.reshape(y.shape))
            return y
        return out.reshape(-1) if vec else out
    if _is_torch(x):
        x = x.numpy()
    x = np.asarray(x)
    vec = x.ndim == 1
    X = np.asfortranarray(x.reshape(x.shape[0], -1), dtype=np.complex128)
    if X.shape[0] != nin:
        raise DimensionMismatch(f"x has {X.shape[0]} rows, the operator {nin} columns")
    nrhs = X.shape[1]
    if y is None:
        Y = np.zeros((nout, nrhs), dtype=np.complex128, order="F")
        beta = 0.0
        target = None
    else:
        if y.shape[0] != nout:
            raise DimensionMismatch(f"y has {y.shape[0]} rows, the operator {nout} rows")
        Y = np.asfortranarray(y.reshape(nout, -1), dtype=np.complex128)
        target = y
    if not ws._lock.acquire(blocking=False):
        raise ConcurrentWorkspaceError()
    try:
        al, be = complex(alpha), complex(beta)
        check(_product(ws, mode, ptr(X), nin, ptr(Y), nout, nrhs, al, be, 0, _tangent))
        t = C.c_double()
        lib().nca_workspace_last_time(ws._h, C.byref(t))
        ws.last_seconds = t.value
    finally:
        ws._lock.release()
    out = Y[:, 0] if vec else Y
    if target is not None:
        target[...] = out.reshape(target.shape).astype(target.dtype, copy=False)
        return target
    return out.astype(ws.dtype, copy=False) if ws.dtype != np.complex128 else out


class _DHDK(LinearMap):
    """dH/dk of an FP64 workspace on its frozen skeleton, forward mode (y = dH/dk x)."""

    def __init__(self, ws):
        self.ws = ws
        self.shape = ws.shape

    def _apply(self, x, mode):
        if mode != MODE_N:
            raise ArgumentError("dH/dk is applied in forward mode only (use the real part of y_bar^H dH/dk x)")
        self.ws.core.prepare_dk()
        return mul(None, self.ws, x, _tangent=True)


def dHdk(A) -> LinearMap:
    """dH/dk as a forward-mode linear map on the frozen skeleton of A's core."""
    ws, mode = _unwrap(A)
    if mode != MODE_N:
        raise ArgumentError("dH/dk is taken of H itself (forward mode); use Re(y_bar^H dH/dk x) for transposes")
    return _DHDK(ws)


def rrule_mul(A, x):
    """ChainRulesCore-style rrule of y = H(k) x: returns (y, pullback) with
    pullback(y_bar) = (k_bar, x_bar), x_bar = H^H y_bar (the adjoint product) and
    k_bar = Re(y_bar^H dH/dk x) (the tangent product on the frozen skeleton). Cotangents follow
    ChainRules' convention dJ = Re<y_bar, dy>, so J = ||y - b||^2 gives y_bar = 2 (y - b)."""
    ws, mode = _unwrap(A)
    if mode != MODE_N:
        raise ArgumentError("rrule_mul differentiates y = H x")
    y = A @ x
    x_saved = x.copy() if hasattr(x, "copy") else x

    def pullback(ybar):
        xbar = ws.H @ ybar
        dy = dHdk(ws) @ x_saved
        kbar = float(np.real(np.vdot(np.asarray(ybar), np.asarray(dy))))
        return kbar, xbar
    return y, pullback


class BatchCore(PetrovGalerkinNCACore):
    """Block-diagonal H^2 operator over several built cores (many problems of uneven size in one
    product). Vectors are the members' vectors stacked in member order: test offsets
    `testoffsets`, trial offsets `trialoffsets`. The batch owns copies of the members' stores
    (with move=True the members' device stores are released as they are copied). Exports of the
    members' blocks are taken from the members."""

    def __init__(self, cores, move: bool = False):
        cores = list(cores)
        if not cores:
            raise ArgumentError("a batch needs at least one core")
        arr = (C.c_void_p * len(cores))(*[c._h.value for c in cores])
        h = C.c_void_p()
        check(lib().nca_core_batch(arr, len(cores), 1 if move else 0, C.byref(h)))
        self._h = h
        info = CoreInfo()
        check(lib().nca_core_get_info(h, C.byref(info)))
        self.info = info
        self.members = len(cores)
        self.testoffsets = np.concatenate([[0], np.cumsum([c.dim[0] for c in cores])]).astype(np.int64)
        self.trialoffsets = np.concatenate([[0], np.cumsum([c.dim[1] for c in cores])]).astype(np.int64)
        self.dim = (int(self.testoffsets[-1]), int(self.trialoffsets[-1]))
        self.f32 = all(c.f32 for c in cores)
        self.device = cores[0].device
        self.maxrank = max(c.maxrank for c in cores)
        self._cache = {}

    def _member_export(self, *args, **kwargs):
        raise ArgumentError("export the member cores of a batch")

    pivots = farpivots = interpolation = _member_export


class _TreeSizes:
    def __init__(self, nnodes):
        self.nnodes = nnodes


class _LoadedTree:
    def __init__(self, info):
        self.test, self.trial = _TreeSizes(info.nnodes_test), _TreeSizes(info.nnodes_trial)


class LoadedCore(PetrovGalerkinNCACore):
    """A core read back by load_core: products, workspaces and exports as the saved core's (its
    products equal the saved core's bit for bit); the Python-side trees and points stay with the
    file."""

    def __init__(self, path, device: int = 0):
        h = C.c_void_p()
        check(lib().nca_core_load(os.fsencode(path), int(device), C.byref(h)))
        self._h = h
        info = CoreInfo()
        check(lib().nca_core_get_info(h, C.byref(info)))
        self.info = info
        self.dim = (int(info.ntest), int(info.ntrial))
        self.device = int(device)
        self.tree = _LoadedTree(info)
        self.operator = None
        self._cache = {}
        # a complex-FP32 product needs the FP32 copies, which the saved core either had or not
        self.f32 = True
        self.maxrank = 128

    def set_wavenumber(self, k: float):
        raise ArgumentError("a loaded core keeps no operator object: refill the core it was saved from")


def load_core(path, device: int = 0) -> LoadedCore:
    """Read a core written by PetrovGalerkinNCACore.save onto `device`."""
    return LoadedCore(path, device)


def batch(cores, move: bool = False) -> BatchCore:
    """One block-diagonal core over several built cores (see BatchCore). move=True releases each
    member's device stores as soon as they are copied; the members are then unusable."""
    return BatchCore([c.core if isinstance(c, H2Workspace) else c for c in cores], move)


def PetrovGalerkinNCA(operator, testspace, trialspace, tree, **kwargs) -> H2Workspace:
    """Build the core and one workspace over it (petrovgalerkinnca.jl:327-331)."""
    dtype = kwargs.pop("dtype", np.complex128)
    return H2Workspace(PetrovGalerkinNCACore(operator, testspace, trialspace, tree, **kwargs), dtype)


def core(A):
    ws, _ = _unwrap(A)
    return ws.core


def transpose(A):
    return A.T


def adjoint(A):
    return A.H


def storage(h2mat, verbose: bool = True) -> float:
    """Stored entries of near field, couplings, transfers and bases in GB (petrovgalerkinnca.jl:386-411)."""
    c = h2mat.core if isinstance(h2mat, H2Workspace) else h2mat
    i = c.info
    n = (i.near_entries + i.coupling_entries + i.transfer_entries_test + i.transfer_entries_trial +
         i.basis_entries_test + i.basis_entries_trial)
    gb = n * 16 * 1e-9
    if verbose:
        print("storage:", gb, "GB")
        print("compression ratio:", n / (c.dim[0] * c.dim[1]))
    return gb
