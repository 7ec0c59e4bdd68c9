"""The compressors and their configuration objects.

Mirrors src/compressors/batchedbottomup.jl: `BatchedBottomUp(pivotselector, compressor)` with a
geometric pivot selector (tree mimicry) and a dense fully pivoted ACA with the sampled
Frobenius-norm stop; and src/compressors/bottomup.jl: `BottomUp(factorization=IACA(...))`, the
only compressor of directional (wideband) H^2 matrices, with IACA(MaximumValue(),
TreeMimicryPivoting(...), FNormExtrapolator(tol)) on the test side and the mirrored
IACA(TreeMimicryPivoting(...), MaximumValue(), ...) on the trial side
(test/nca/test_petrovgalerkinnca.jl:131-139). The work itself runs in libnca_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import ArgumentError, check, lib, ptr


class FullPivoting:
    """Full pivoting: the argmax of |R_ij| over the whole residual (ties: lowest index)."""


class FNormEstimator:
    """Stop after r crosses once ||R_r||_F^2 (s/(s-r) when sampled) <= tol^2 ||A||_F^2."""

    def __init__(self, tol: float = 1e-4):
        self.tol = float(tol)


class ACA:
    """ACA(rowpivoting, columnpivoting, convergence); only full pivoting is batched."""

    def __init__(self, rowpivoting=None, columnpivoting=None, convergence=None, *, tol=None):
        self.rowpivoting = rowpivoting or FullPivoting()
        self.columnpivoting = columnpivoting or FullPivoting()
        if convergence is None:
            convergence = FNormEstimator(1e-4 if tol is None else tol)
        self.convergence = convergence
        if not (isinstance(self.rowpivoting, FullPivoting) and isinstance(self.columnpivoting, FullPivoting)):
            raise ArgumentError("the batched compressor needs ACA(FullPivoting(), FullPivoting(), ...)")

    @property
    def tol(self):
        return self.convergence.tol

    def __call__(self, block, maxrank, sampled=False):
        """Fully pivoted ACA of one dense block on the GPU: (rank, rowpivots, colpivots)."""
        from .seams import blocks_aca
        A = np.asfortranarray(block, dtype=np.complex128)
        ranks, rows, cols = blocks_aca([A], maxrank, self.tol, sampled=sampled)
        r = int(ranks[0])
        return r, rows[0][:r], cols[0][:r]


class TreeMimicryPivoting:
    """Geometric far-pivot selection by descending the far tree (tree mimicry).

    Each pivot maximises dmin(y)^2 / |y - c_t|^2 over the untaken far points y, where dmin is
    the distance to the pivots already chosen and c_t the centroid of the cluster: the first
    pivot is the far point closest to the cluster, later ones spread over the far field as seen
    from the cluster. The far tree is descended by the same score at its node centres.
    """

    def __init__(self, ownpoints, farpoints, fartree):
        self.ownpoints = np.ascontiguousarray(ownpoints, dtype=np.float64).reshape(-1, 3)
        self.farpoints = np.ascontiguousarray(farpoints, dtype=np.float64).reshape(-1, 3)
        self.fartree = fartree


class MaximumValue:
    """Value pivoting of IACA: the row of the largest residual entry (ties: lowest row)."""


class FNormExtrapolator:
    """IACA stop: the candidate column's residual r passes when ||r||^2 k <= tol^2 S (S: squared
    Frobenius norm of the k sampled columns). This is FNormEstimator's test ||u_k|| ||v_k|| <= tol
    ||A_k||_F with the norms over the whole far field extrapolated uniformly from the sampled
    columns. The factorization stops, rejecting the candidate, once two consecutive candidates
    pass (or a residual is exactly zero). Accepts a tolerance or an FNormEstimator
    (FNormExtrapolator(FNormEstimator(tol)), test/pivoting/test_pivots.jl:34-38)."""

    def __init__(self, tol=1e-4):
        self.tol = float(tol.tol if isinstance(tol, FNormEstimator) else tol)


class IACA:
    """IACA(rowpivoting, columnpivoting, convergence): one side geometric (TreeMimicryPivoting),
    the other by value (MaximumValue); test side IACA(MaximumValue(), TreeMimicryPivoting, conv),
    trial side IACA(TreeMimicryPivoting, MaximumValue(), conv)."""

    def __init__(self, rowpivoting=None, columnpivoting=None, convergence=None):
        self.rowpivoting, self.columnpivoting = rowpivoting, columnpivoting
        self.convergence = convergence if convergence is not None else FNormExtrapolator(1e-4)
        kinds = (type(rowpivoting), type(columnpivoting))
        if kinds not in ((MaximumValue, TreeMimicryPivoting), (TreeMimicryPivoting, MaximumValue)):
            raise ArgumentError("IACA needs one TreeMimicryPivoting side and one MaximumValue side")
        if not isinstance(self.convergence, FNormExtrapolator):
            raise ArgumentError("IACA needs an FNormExtrapolator convergence criterion")

    @property
    def tol(self):
        return self.convergence.tol

    def geometric_side(self):
        """0 when the columns are geometric (a test-side IACA), 1 when the rows are."""
        return 0 if isinstance(self.columnpivoting, TreeMimicryPivoting) else 1


class BottomUp:
    """BottomUp(factorization=IACA(...), representor=None) (src/compressors/bottomup.jl:1-96).
    The factorization must be an IACA with tree-mimicry pivoting; representors are not offered."""

    def __init__(self, factorization=None, representor=None):
        if not isinstance(factorization, IACA):
            raise ArgumentError("BottomUp needs factorization=IACA(MaximumValue(), TreeMimicryPivoting(...), "
                                "FNormExtrapolator(tol)) (trial side: the pivotings swapped)")
        if representor is not None:
            raise ArgumentError("BottomUp representors are not offered")
        self.factorization, self.representor = factorization, representor


class BatchedBottomUp:
    """BatchedBottomUp(pivotselector, compressor) (batchedbottomup.jl:30-51)."""

    def __init__(self, pivotselector=None, compressor=None):
        if pivotselector is None or compressor is None:
            raise TypeError("BatchedBottomUp needs both pivotselector and compressor")
        self.pivotselector = pivotselector
        self.compressor = compressor


def _clustersize(tree, node: int, limit: int | None = None) -> int:
    """Points of `node`, capped at `limit` (pivots.jl:4-25)."""
    n = tree.numberofvalues(node)
    if limit is None:
        return n
    return 0 if limit <= 0 else min(limit, n)


def _selectfarpivots(pivotselector: TreeMimicryPivoting, refidcs, idcs, fartree, maxrank: int):
    """Phase 1 for one cluster (batchedbottomup.jl:54-72): up to min(maxrank, |refidcs|) far
    points, without matrix entries."""
    ref = np.ascontiguousarray(refidcs, dtype=np.int32)
    nodes = np.ascontiguousarray(idcs, dtype=np.int32)
    out = np.zeros(max(int(maxrank), 1), dtype=np.int32)
    n = C.c_int32()
    check(lib().nca_select_farpivots(fartree._h, ptr(pivotselector.ownpoints), ptr(pivotselector.farpoints),
                                     ptr(ref), len(ref), ptr(nodes), len(nodes), int(maxrank), ptr(out),
                                     C.byref(n)))
    return out[:n.value].copy()
