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


class IsNearWideband:
    """Wideband admissibility (nearinteractions.jl:62-95): low frequency when k min(d) <= gamma,
    then near iff max(d) > eta_lf sep; otherwise near iff 4 k max(r)^2 > eta_hf sep. A core built
    on it is a directional H^2 matrix."""

    def __init__(self, k: float, etalf: float = 1.0, etahf: float = 5.0, gamma: float = 1.0):
        self.k, self.etalf, self.etahf, self.gamma = float(k), float(etalf), float(etahf), float(gamma)

    def islf(self, diam: float) -> bool:
        return self.k * diam <= self.gamma

    def __call__(self, ttree, stree, t, s):
        rt, rs = ttree.radius(t), stree.radius(s)
        gap = np.linalg.norm(ttree.center(t) - stree.center(s)) - (rt + rs)
        sep = max(gap, 0.0)
        if self.islf(min(2 * rt, 2 * rs)):
            return 2 * max(rt, rs) > self.etalf * sep
        return 4 * self.k * max(rt * rt, rs * rs) > self.etahf * sep


def isnearwideband(k: float, etalf: float = 1.0, etahf: float = 5.0, gamma: float = 1.0) -> IsNearWideband:
    return IsNearWideband(k, etalf, etahf, gamma)


class Partition:
    """Near and far interaction lists over the test nodes (CSR, each list ascending)."""

    def __init__(self, tree: BlockTree, condition):
        if not isinstance(condition, (IsNear, IsNearWideband)):
            raise TypeError("isnear must be nca_b200.isnear(eta) or nca_b200.isnearwideband(k)")
        self.tree, self.isnear = tree, condition
        self.wideband = isinstance(condition, IsNearWideband)
        h = C.c_void_p()
        if self.wideband:
            check(lib().nca_interactions_wideband(tree.test._h, tree.trial._h, condition.k, condition.etalf,
                                                  condition.etahf, condition.gamma, C.byref(h)))
        else:
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


class DirectionalData:
    """Far interactions of one tree subdivided into directions, with the basis items of the
    directional compressor (abstractdirections.jl:3-55): items are (cluster, direction) pairs in
    node order; `dirs[item]` is 0 for the low-frequency direction, else the 1-based candidate
    direction; far nodes are grouped by direction (`dirfarptr`); nested items list their
    children's items (`item_chptr`, `item_chidx`)."""

    def __init__(self, tree: BlockTree, partition: Partition, side: int):
        if not partition.wideband:
            raise TypeError("directional data need a wideband partition (isnearwideband)")
        own, far = (tree.test, tree.trial) if side == 0 else (tree.trial, tree.test)
        h = C.c_void_p()
        check(lib().nca_directional_plan(own._h, far._h, partition._h, int(side), C.byref(h)))
        self._h, self.side, self.tree = h, side, own
        ni, nf, nc = C.c_int32(), C.c_int64(), C.c_int64()
        check(lib().nca_dirplan_sizes(h, C.byref(ni), C.byref(nf), C.byref(nc)))
        n = ni.value
        self.farnodes = np.zeros(nf.value, np.int32)
        self.dirptr = np.zeros(own.nnodes + 1, np.int32)
        self.dirs = np.zeros(n, np.int32)
        self.dirvec = np.zeros((n, 3))
        self.dirfarptr = np.zeros(n + 1, np.int32)
        self.item_basis = np.zeros(n, np.int32)
        self.item_chptr = np.zeros(n + 1, np.int32)
        self.item_chidx = np.zeros(nc.value, np.int32)
        check(lib().nca_dirplan_export(h, *[ptr(a) for a in (self.farnodes, self.dirptr, self.dirs, self.dirvec,
                                                             self.dirfarptr, self.item_basis, self.item_chptr,
                                                             self.item_chidx)]))
        self.nitems = n

    def farfield(self, item: int):
        n = C.c_int32()
        check(lib().nca_dirplan_farfield(self._h, int(item), None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.int32)
        check(lib().nca_dirplan_farfield(self._h, int(item), ptr(out), n.value, C.byref(n)))
        return out[:n.value]

    def __del__(self):
        h = self.__dict__.get("_h")
        if h is not None and h.value:
            lib().nca_dirplan_destroy(h)
            self._h = None


def directionalfardata(tree: BlockTree, partition: Partition):
    """(test, trial) directional far data of a wideband partition (boundingballdirections.jl:44-152)."""
    return DirectionalData(tree, partition, 0), DirectionalData(tree, partition, 1)
