"""Oracle restatement of the directional (wideband) host plan (test infrastructure only).

Follows NestedCrossApproximation.jl line by line, in Python on 0-based ids:
  - isnearwideband for bounding balls: src/admissibility/nearinteractions.jl:62-95, with the
    dual tree traversal of the ACA interactions (a far pair is stored, a near pair of leaves is
    stored, otherwise the non-leaf side(s) split);
  - the generalised radius and the low-frequency class: nearinteractions.jl:138-158;
  - candidate directions (spherical Fibonacci points): boundingballdirections.jl:12-29;
  - directionalfardata (direction sets, far nodes grouped by direction, parent-to-child
    direction maps): boundingballdirections.jl:44-152, _finalize_directionaldata:
    abstractdirections.jl:57-116;
  - dirfarfield: abstractdirections.jl:192-231; isbasisnode: abstractdirections.jl:238-243;
  - the basis items of the bottom-up compressor and their children's items:
    src/compressors/bottomup.jl:214-320.
Dot products and sums are written out element by element in the same order as the library's
host code, so ties resolve identically. DirectionalH2 wraps the C restatement of the same plan,
the directional build (IACA per item) and the directional product (nca_oracle.c). Only the tests
and the CPU legs of the benchmark import this module.
"""
from __future__ import annotations

import math

import numpy as np


def _dist(a, b):
    x, y, z = a[0] - b[0], a[1] - b[1], a[2] - b[2]
    return math.sqrt(x * x + y * y + z * z)


def isnearwideband(T, S, t, s, k, etalf, etahf, gamma):
    ths, shs = T.radius[t], S.radius[s]
    dist = _dist(T.center[t], S.center[s]) - (ths + shs)
    sep = max(dist, 0.0)
    if k * min(2.0 * ths, 2.0 * shs) <= gamma:
        return 2.0 * max(ths, shs) > etalf * sep
    return 4.0 * k * max(ths * ths, shs * shs) > etahf * sep


def interactions_wideband(T, S, k, etalf=1.0, etahf=5.0, gamma=1.0):
    """(nearptr, nearnodes, farptr, farnodes, tfarptr, tfarnodes), lists ascending."""
    near, far = [], []

    def visit(t, s):
        if not isnearwideband(T, S, t, s, k, etalf, etahf, gamma):
            far.append((t, s))
            return
        lt, ls = T.isleaf(t), S.isleaf(s)
        if lt and ls:
            near.append((t, s))
        elif lt:
            for c in S.children(s):
                visit(t, c)
        elif ls:
            for c in T.children(t):
                visit(c, s)
        else:
            for c in T.children(t):
                for d in S.children(s):
                    visit(c, d)

    visit(0, 0)

    def csr(pairs, n, key):
        lists = [[] for _ in range(n)]
        for p in pairs:
            lists[p[key]].append(p[1 - key])
        ptr = np.zeros(n + 1, np.int32)
        for i in range(n):
            ptr[i + 1] = ptr[i] + len(lists[i])
        return ptr, np.array([v for lst in lists for v in sorted(lst)], np.int32)

    nptr, nnodes = csr(near, T.nnodes, 0)
    fptr, fnodes = csr(far, T.nnodes, 0)
    tptr, tnodes = csr(far, S.nnodes, 1)
    return nptr, nnodes, fptr, fnodes, tptr, tnodes


def genradius(T, node):
    p = T.parent[node]
    if p < 0:
        return T.radius[node]
    total = 0.0
    for c in T.children(p):
        total += T.radius[c]
    return min(genradius(T, p), total / T.nchildren[p])


def islf(T, node, k, gamma):
    return k * (2.0 * genradius(T, node)) <= gamma


def directions(diam, k, gamma):
    kd = max(k * diam, 2.0 ** -52)
    ratio = math.acos(1.0 / math.sqrt(3.0)) / math.asin(min(1.0, gamma / kd))
    n = max(6, int(math.ceil(6.0 * math.pow(4.0, math.log(ratio) / math.log(2.0)))))
    ga = math.pi * (3.0 - math.sqrt(5.0))
    out = np.zeros((n, 3))
    for i in range(n):
        z = 1.0 - 2.0 * (i + 0.5) / n
        r = math.sqrt(max(0.0, 1.0 - z * z))
        out[i] = (r * math.cos(i * ga), r * math.sin(i * ga), z)
    return out


def nearest_direction(D, v):
    """1-based index of the direction with the largest dot product, first on ties."""
    dots = D[:, 0] * v[0] + D[:, 1] * v[1] + D[:, 2] * v[2]
    return int(np.argmax(dots)) + 1


class DirectionalData:
    """directionalfardata of one tree plus the basis items of the bottom-up compressor."""

    def __init__(self, T, F, farptr, farnodes, k, etahf=5.0, gamma=1.0):
        nn = T.nnodes
        self.T = T
        self.farptr = np.asarray(farptr).copy()
        self.farnodes = np.asarray(farnodes).copy()
        dirs = [[] for _ in range(nn)]
        dircount = [[] for _ in range(nn)]
        pmap = [[] for _ in range(nn)]
        pcount = [0] * nn
        dirsvec = [None] * nn
        for level in range(T.nlevels):
            for node in np.nonzero(T.level == level)[0]:
                node = int(node)
                p = int(T.parent[node])
                hasfars = self.farptr[node + 1] > self.farptr[node]
                hasparentvecs = p >= 0 and dirsvec[p] is not None
                hasparentdirs = p >= 0 and len(dirs[p]) > 0
                if islf(T, node, k, gamma):
                    inherit = hasparentdirs and level > 0 and islf(T, p, k, gamma)
                    dirs[node] = [0] if (hasfars or inherit) else []
                    pmap[node] = [1] if inherit else []
                    continue
                if not hasfars and not hasparentvecs:
                    dirs[node] = []
                    continue
                total = directions(2.0 * T.radius[node], k, gamma)
                b, e = int(self.farptr[node]), int(self.farptr[node + 1])
                c = T.center[node]
                nodedirs = []
                for f in self.farnodes[b:e]:
                    cf = F.center[f]
                    nodedirs.append(nearest_direction(total, (c[0] - cf[0], c[1] - cf[1], c[2] - cf[2])))
                perm = sorted(range(len(nodedirs)), key=lambda i: nodedirs[i])  # stable
                self.farnodes[b:e] = self.farnodes[b:e][perm]
                uniq = sorted(set(nodedirs))
                noriginal = len(uniq)
                partochddir = []
                if p >= 0:
                    cp = T.center[p]
                    rp2 = 2.0 * T.radius[p]
                    mult = k * rp2 / etahf + rp2
                    for didx in range(len(dirs[p])):
                        pv = dirsvec[p][didx]
                        v = (c[0] - cp[0] + mult * pv[0], c[1] - cp[1] + mult * pv[1], c[2] - cp[2] + mult * pv[2])
                        partochddir.append(nearest_direction(total, v))
                    for idx, cdir in enumerate(partochddir):
                        if cdir in uniq:
                            partochddir[idx] = uniq.index(cdir) + 1
                        else:
                            uniq.append(cdir)
                            partochddir[idx] = len(uniq)
                counts = [0] * len(uniq)
                sd = [nodedirs[i] for i in perm]
                i = 0
                for u in range(noriginal):
                    while i < len(sd) and sd[i] == uniq[u]:
                        counts[u] += 1
                        i += 1
                dirsvec[node] = total[np.array(uniq) - 1]
                pmap[node] = partochddir
                pcount[node] = sum(1 for x in partochddir if x != 0)
                dirs[node] = uniq
                dircount[node] = counts
        for node in range(nn):
            if dirs[node] and not dircount[node]:
                dircount[node] = [max(0, int(self.farptr[node + 1] - self.farptr[node]))]
                pcount[node] = len(pmap[node])
        # CSR
        self.dirptr = np.zeros(nn + 1, np.int32)
        self.chdirptr = np.zeros(nn + 1, np.int32)
        for node in range(nn):
            self.dirptr[node + 1] = self.dirptr[node] + len(dirs[node])
            self.chdirptr[node + 1] = self.chdirptr[node] + pcount[node]
        ni = int(self.dirptr[-1])
        self.dirs = np.zeros(ni, np.int32)
        self.dirvec = np.zeros((ni, 3))
        self.dirfarptr = np.zeros(ni + 1, np.int32)
        self.chdirmap = np.zeros(int(self.chdirptr[-1]), np.int32)
        self.item_node = np.zeros(ni, np.int32)
        for node in range(nn):
            off = int(self.farptr[node])
            for u, d in enumerate(dirs[node]):
                item = int(self.dirptr[node]) + u
                self.dirs[item] = d
                self.item_node[item] = node
                if dirsvec[node] is not None:
                    self.dirvec[item] = dirsvec[node][u]
                self.dirfarptr[item] = off
                off += dircount[node][u]
            self.chdirmap[self.chdirptr[node]:self.chdirptr[node + 1]] = pmap[node]
        self.dirfarptr[ni] = self.farptr[nn]
        self.nitems = ni
        # items: basis or nested in the children's mapped items
        self.item_basis = np.zeros(ni, np.int32)
        chptr, chidx = [0], []
        for item in range(ni):
            node = int(self.item_node[item])
            basis = self.isbasisnode(node, int(self.dirs[item]))
            self.item_basis[item] = basis
            if not basis:
                local = item - int(self.dirptr[node])
                for ch in T.children(node):
                    m = int(self.dirmap(ch)[local])
                    chidx.append(int(self.dirptr[ch]) + m - 1)
            chptr.append(len(chidx))
        self.item_chptr = np.array(chptr, np.int32)
        self.item_chidx = np.array(chidx, np.int32)

    def node_dirs(self, node):
        return list(self.dirs[self.dirptr[node]:self.dirptr[node + 1]])

    def dirmap(self, node):
        return self.chdirmap[self.chdirptr[node]:self.chdirptr[node + 1]]

    def dirfarnodes(self, node, d):
        local = self.node_dirs(node).index(d)
        item = int(self.dirptr[node]) + local
        return list(self.farnodes[self.dirfarptr[item]:self.dirfarptr[item + 1]])

    def isbasisnode(self, node, d):
        T = self.T
        if T.isleaf(node):
            return True
        if d == 0:
            return False
        fc = int(T.firstchild[node])
        return self.node_dirs(fc) in ([0], [])

    def farfield(self, item):
        """dirfarfield of an item."""
        T = self.T
        node = int(self.item_node[item])
        d = int(self.dirs[item])
        ff = []
        if d == 0:
            cur = node
            while cur >= 0:
                cd = self.node_dirs(cur)
                if not cd or 0 not in cd:
                    break
                ff.extend(self.dirfarnodes(cur, 0))
                cur = int(T.parent[cur])
            return np.array(ff, np.int32)
        ff.extend(self.dirfarnodes(node, d))
        cur = node
        diridcs = [item - int(self.dirptr[node]) + 1]
        while T.parent[cur] >= 0:
            cmap = self.dirmap(cur)
            diridcs = [i + 1 for i, x in enumerate(cmap) if x in diridcs]
            par = int(T.parent[cur])
            pardirs = self.node_dirs(par)
            for i in diridcs:
                ff.extend(self.dirfarnodes(par, pardirs[i - 1]))
            cur = par
        return np.array(ff, np.int32)


class DirectionalH2:
    """Oracle directional H^2 matrix, built and applied by the C restatement (nca_oracle.c,
    OpenMP): the directional plan (as DirectionalData above), the bottom-up compressor per
    (cluster, direction) item with IACA (tree-mimicry columns over the item's directional far
    field, maximum-value rows, extrapolated Frobenius stop; src/compressors/bottomup.jl:214-424,
    src/pivoting/pivots.jl:329-364), couplings per directional far pair
    (src/couplingmatrices.jl:55-111), the near field, and the directional product
    (src/nca/{aggregate,couple,disaggregate}.jl, directional methods)."""

    def __init__(self, testpts, trialpts, kernel, k, minvalues=32, tol=1e-4, maxrank=50, etalf=1.0, etahf=5.0,
                 gamma=1.0, nthreads=None):
        import ctypes as C
        import os
        from . import oracle as O
        self.O = O
        L = O.lib()
        self.testpts = np.ascontiguousarray(testpts, dtype=np.float64)
        self.trialpts = np.ascontiguousarray(trialpts, dtype=np.float64)
        self.kernel, self.maxrank, self.tol = kernel, maxrank, tol
        if maxrank > 256:
            raise ValueError("the oracle supports maxrank <= 256")
        self._h = L.oracle_dir_build(O._p(self.testpts), len(self.testpts), O._p(self.trialpts),
                                     len(self.trialpts), int(minvalues), float(k), float(etalf), float(etahf),
                                     float(gamma), *kernel.args(), float(tol), float(tol), int(maxrank),
                                     int(nthreads or os.cpu_count() or 1))
        side, item, npiv, rank = (C.c_int() for _ in range(4))
        st = L.oracle_dir_status(self._h, C.byref(side), C.byref(item), C.byref(npiv), C.byref(rank))
        self.trees = [O.Tree(L.oracle_dir_tree(self._h, s), len(p), self) for s, p in
                      ((0, self.testpts), (1, self.trialpts))]
        if st:
            raise O.SingularBuild(f"singular cross matrix (side {side.value}, item {item.value}, "
                                  f"{npiv.value} pivots, rank {rank.value})")
        self.nitems, self.ranks, self.nrows, self.piv, self.plan = [], [], [], [], []
        for sd in (0, 1):
            ni = L.oracle_dir_nitems(self._h, sd)
            nn = self.trees[sd].nnodes
            nf = L.oracle_dir_nfar(self._h, sd)
            nc = L.oracle_dir_nchildren(self._h, sd)
            plan = {"farnodes": np.zeros(nf, np.int32), "dirptr": np.zeros(nn + 1, np.int32),
                    "dirs": np.zeros(ni, np.int32), "dirvec": np.zeros((ni, 3)),
                    "dirfarptr": np.zeros(ni + 1, np.int32), "item_basis": np.zeros(ni, np.int32),
                    "item_chptr": np.zeros(ni + 1, np.int32), "item_chidx": np.zeros(nc, np.int32)}
            L.oracle_dir_plan(self._h, sd, *[O._p(plan[f]) for f in ("farnodes", "dirptr", "dirs", "dirvec",
                                                                        "dirfarptr", "item_basis", "item_chptr",
                                                                        "item_chidx")])
            rank = np.zeros(max(ni, 1), np.int32)
            nrows = np.zeros(max(ni, 1), np.int32)
            ptr = np.zeros(ni + 1, np.int32)
            idx = np.zeros(max(ni * maxrank, 1), np.int32)
            L.oracle_dir_pivots(self._h, sd, O._p(rank), O._p(nrows), O._p(ptr), O._p(idx))
            self.nitems.append(ni)
            self.ranks.append(rank[:ni])
            self.nrows.append(nrows[:ni])
            self.piv.append([idx[ptr[i]:ptr[i + 1]].copy() for i in range(ni)])
            self.plan.append(plan)
        xe, ce, ne, npairs = (C.c_long() for _ in range(4))
        L.oracle_dir_sizes(self._h, C.byref(xe), C.byref(ce), C.byref(ne), C.byref(npairs))
        self.entries = {"x": xe.value, "coupling": ce.value, "near": ne.value, "pairs": npairs.value}

    def interpolation(self, side):
        """X of every item of one side (nrows x rank)."""
        L = self.O.lib()
        tot = L.oracle_dir_x_total(self._h, side)
        ni = self.nitems[side]
        off = np.zeros(ni + 1, np.int64)
        X = np.zeros(max(tot, 1), np.complex128)
        L.oracle_dir_x(self._h, side, self.O._p(off), self.O._p(X))
        return [X[off[i]:off[i + 1]].reshape((self.nrows[side][i], self.ranks[side][i]), order="F")
                for i in range(ni)]

    @property
    def shape(self):
        return (len(self.testpts), len(self.trialpts))

    def apply(self, x, mode=0):
        """y = op(H) x for a vector or a block of columns; mode 0: H, 1: H^T, 2: H^H."""
        x = np.asarray(x, dtype=np.complex128)
        vec = x.ndim == 1
        X = np.asfortranarray(x.reshape(x.shape[0], -1))
        nin, nout = (self.shape[1], self.shape[0]) if mode == 0 else self.shape
        if X.shape[0] != nin:
            raise ValueError("dimension mismatch")
        Y = np.zeros((nout, X.shape[1]), dtype=np.complex128, order="F")
        self.O.lib().oracle_dir_apply(self._h, int(mode), self.O._p(X), nin, self.O._p(Y), nout, X.shape[1])
        return Y[:, 0] if vec else Y

    def __del__(self):
        if getattr(self, "_h", None):
            self.O.lib().oracle_dir_free(self._h)
            self._h = None
