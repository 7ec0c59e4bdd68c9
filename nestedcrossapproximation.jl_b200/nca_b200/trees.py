"""Cluster trees and the block tree (the H2Trees.jl interface the reference consumes).

The reference receives the tree as an argument of PetrovGalerkinNCA
(src/nca/petrovgalerkinnca.jl:138-142) and reads it through H2Trees' values, children,
parent, isleaf, center, radius and level iterators. Node ids here are 0-based and in
breadth-first order (root 0, siblings consecutive); point indices are 0-based.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, ptr


class KMeansTreeBuilder:
    """H2Trees.KMeansTreeBuilder(; numberofclusters=2, minvalues)."""

    def __init__(self, numberofclusters: int = 2, minvalues: int = 32):
        self.numberofclusters = int(numberofclusters)
        self.minvalues = int(minvalues)


class KMeansTree:
    """k-means cluster tree of a point set: a node with more than `minvalues` points is split
    into two clusters (2-means, farthest-point seeds, Lloyd iterations, stable partition)."""

    def __init__(self, points, builder: KMeansTreeBuilder | None = None, minvalues: int | None = None):
        builder = builder or KMeansTreeBuilder(minvalues=minvalues or 32)
        self.points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        self.builder = builder
        h = C.c_void_p()
        check(lib().nca_tree_kmeans(ptr(self.points), len(self.points), builder.minvalues,
                                    builder.numberofclusters, C.byref(h)))
        self._h = h
        nn, nl, npts = C.c_int32(), C.c_int32(), C.c_int64()
        check(lib().nca_tree_sizes(h, C.byref(nn), C.byref(nl), C.byref(npts)))
        n = nn.value
        self.nnodes, self.nlevels = n, nl.value
        self.perm = np.zeros(npts.value, np.int32)
        arrs = [np.zeros(n, np.int32) for _ in range(6)]
        self._center = np.zeros((n, 3))
        self._radius = np.zeros(n)
        check(lib().nca_tree_export(h, ptr(self.perm), *[ptr(a) for a in arrs], ptr(self._center),
                                    ptr(self._radius)))
        self.begin, self.end, self._parent, self.firstchild, self.nchildren, self.level = arrs

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().nca_tree_destroy(h)
            self._h = None

    # H2Trees-style accessors
    def numberofnodes(self):
        return self.nnodes

    def numberofvalues(self, node=None):
        return len(self.perm) if node is None else int(self.end[node] - self.begin[node])

    def root(self):
        return 0

    def values(self, node):
        return self.perm[self.begin[node]:self.end[node]]

    def children(self, node):
        f = self.firstchild[node]
        return list(range(f, f + self.nchildren[node])) if f >= 0 else []

    def isleaf(self, node):
        return self.nchildren[node] == 0

    def parent(self, node):
        return int(self._parent[node])

    def center(self, node):
        return self._center[node]

    def radius(self, node):
        return float(self._radius[node])

    def levels(self):
        return list(range(self.nlevels))

    def levelnodes(self, level):
        return [int(n) for n in np.nonzero(self.level == level)[0]]

    def leaves(self):
        return [n for n in range(self.nnodes) if self.isleaf(n)]

    def parents_upwards(self, node):
        out = []
        p = self.parent(node)
        while p >= 0:
            out.append(p)
            p = self.parent(p)
        return out


class BlockTree:
    """Pair of a test and a trial cluster tree (H2Trees.BlockTree)."""

    def __init__(self, testtree: KMeansTree, trialtree: KMeansTree):
        self.test, self.trial = testtree, trialtree


def testtree(tree: BlockTree) -> KMeansTree:
    return tree.test


def trialtree(tree: BlockTree) -> KMeansTree:
    return tree.trial
