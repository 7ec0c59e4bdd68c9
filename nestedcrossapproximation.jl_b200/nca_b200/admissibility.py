"""Admissibility, interaction lists and far data (src/admissibility/farinteractions.jl).

`isnear(eta)` is the ball condition: a pair is near when
2 max(r_t, r_s) > eta * max(|c_t - c_s| - r_t - r_s, 0) (the low-frequency branch of
src/admissibility/nearinteractions.jl:84-95). `interactions` walks both trees from the roots:
a far pair is stored, a near pair of leaves is stored, otherwise the non-leaf side(s) split.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, ptr
from .trees import BlockTree


class IsNear:
    def __init__(self, eta: float = 1.0):
        self.eta = float(eta)

    def __call__(self, ttree, stree, t, s):
        rt, rs = ttree.radius(t), stree.radius(s)
        gap = np.linalg.norm(ttree.center(t) - stree.center(s)) - (rt + rs)
        return 2 * max(rt, rs) > self.eta * max(gap, 0.0)


def isnear(eta: float = 1.0) -> IsNear:
    return IsNear(eta)


class Partition:
    """Near and far interaction lists over the test nodes (CSR, each list ascending)."""

    def __init__(self, tree: BlockTree, condition: IsNear):
        if not isinstance(condition, IsNear):
            raise TypeError("isnear must be nca_b200.isnear(eta)")
        self.tree, self.isnear = tree, condition
        h = C.c_void_p()
        check(lib().nca_interactions(tree.test._h, tree.trial._h, condition.eta, C.byref(h)))
        self._h = h
        nn, nf = C.c_int64(), C.c_int64()
        check(lib().nca_partition_sizes(h, C.byref(nn), C.byref(nf)))
        nt, ns = tree.test.nnodes, tree.trial.nnodes
        self.nearptr = np.zeros(nt + 1, np.int32)
        self.nearnodes = np.zeros(nn.value, np.int32)
        self.farptr = np.zeros(nt + 1, np.int32)
        self.farnodes = np.zeros(nf.value, np.int32)
        self.trialfarptr = np.zeros(ns + 1, np.int32)
        self.trialfarnodes = np.zeros(nf.value, np.int32)
        check(lib().nca_partition_export(h, *[ptr(a) for a in (self.nearptr, self.nearnodes, self.farptr,
                                                               self.farnodes, self.trialfarptr, self.trialfarnodes)]))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().nca_partition_destroy(h)
            self._h = None


def interactions(tree: BlockTree, condition: IsNear) -> Partition:
    return Partition(tree, condition)


class FarData:
    """Far interactions of the clusters of one tree in CSR layout (farinteractions.jl:16-19)."""

    def __init__(self, nodetofarnodesptr, farnodes):
        self.nodetofarnodesptr = np.asarray(nodetofarnodesptr)
        self.farnodes = np.asarray(farnodes)


def farptr(data: FarData):
    return data.nodetofarnodesptr


def farnodes(data: FarData, node: int | None = None):
    if node is None:
        return data.farnodes
    p = data.nodetofarnodesptr
    return data.farnodes[p[node]:p[node + 1]]


def farfield(tree, data: FarData, node: int):
    """Own far nodes, then those of each ancestor (farinteractions.jl:38-60)."""
    out = list(farnodes(data, node))
    for p in tree.parents_upwards(node):
        out.extend(farnodes(data, p))
    return np.asarray(out, dtype=np.int32)


def farinteractions(tree: BlockTree, partition: Partition):
    return (FarData(partition.farptr, partition.farnodes),
            FarData(partition.trialfarptr, partition.trialfarnodes))


def fardata(tree: BlockTree, condition: IsNear, partition: Partition | None = None):
    return farinteractions(tree, partition or interactions(tree, condition))
