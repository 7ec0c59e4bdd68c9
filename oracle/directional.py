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
Only the tests import this module. Dot products and sums are written out element by element in
the same order as the library's host code, so ties resolve identically.
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
    """Oracle directional H^2 matrix: the bottom-up compressor per (cluster, direction) item
    (src/compressors/bottomup.jl:214-424) with the project's pivoting rules (tree mimicry over
    the item's directional far field, the sampled fully pivoted ACA on K[rows, far pivots],
    X = K[rows, sigma] K[tau, sigma]^{-1}), couplings per directional far pair
    (src/couplingmatrices.jl:55-111), the near field, and the directional product
    (src/nca/{aggregate,couple,disaggregate}.jl, directional methods)."""

    def __init__(self, testpts, trialpts, kernel, k, minvalues=32, tol=1e-4, maxrank=50, etalf=1.0, etahf=5.0,
                 gamma=1.0):
        from . import oracle as O
        self.O = O
        self.testpts = np.ascontiguousarray(testpts, dtype=np.float64)
        self.trialpts = np.ascontiguousarray(trialpts, dtype=np.float64)
        self.kernel = kernel
        self.trees = [O.OwnedTree(self.testpts, minvalues), O.OwnedTree(self.trialpts, minvalues)]
        T, S = self.trees
        (self.nearptr, self.nearnodes, fptr, fnodes, tptr, tnodes) = interactions_wideband(T, S, k, etalf, etahf, gamma)
        self.tnearptr, self.tnearnodes = self._transpose(self.nearptr, self.nearnodes, S.nnodes)
        self.dirs = [DirectionalData(T, S, fptr, fnodes, k, etahf, gamma),
                     DirectionalData(S, T, tptr, tnodes, k, etahf, gamma)]
        self.maxrank, self.tol = maxrank, tol
        self.piv = [None, None]
        self.X = [None, None]
        for side in (0, 1):
            self._build_side(side)
        self._couplings()

    @staticmethod
    def _transpose(ptr, nodes, n):
        lists = [[] for _ in range(n)]
        for t in range(len(ptr) - 1):
            for s in nodes[ptr[t]:ptr[t + 1]]:
                lists[s].append(t)
        tp = np.zeros(n + 1, np.int32)
        for i in range(n):
            tp[i + 1] = tp[i] + len(lists[i])
        return tp, np.array([v for lst in lists for v in lst], np.int32)

    def _block(self, side, rows, cols):
        """K[rows, cols]; side 0: rows are test points, side 1: rows are trial points."""
        O = self.O
        rows = np.asarray(rows, np.int64)
        cols = np.asarray(cols, np.int64)
        if side == 0:
            ii, jj = np.repeat(rows, len(cols)), np.tile(cols, len(rows))
        else:
            ii, jj = np.tile(cols, len(rows)), np.repeat(rows, len(cols))
        v = O.entries(self.kernel, self.testpts, self.trialpts, ii, jj)
        return v.reshape(len(rows), len(cols))

    def _build_side(self, side):
        O = self.O
        D = self.dirs[side]
        T, F = self.trees[side], self.trees[1 - side]
        own = self.testpts if side == 0 else self.trialpts
        far = self.trialpts if side == 0 else self.testpts
        piv = [np.zeros(0, np.int32)] * D.nitems
        X = [None] * D.nitems
        for level in range(T.nlevels - 1, -1, -1):
            for item in range(D.nitems):
                node = int(D.item_node[item])
                if T.level[node] != level:
                    continue
                ff = D.farfield(item)
                if len(ff) == 0:
                    continue
                if D.item_basis[item]:
                    rows = T.values(node)
                else:
                    rows = np.concatenate([piv[ch] for ch in D.item_chidx[D.item_chptr[item]:D.item_chptr[item + 1]]]
                                          + [np.zeros(0, np.int32)]).astype(np.int32)
                fp = O.select_farpivots(F, own, far, T.values(node), ff, self.maxrank)
                if len(fp) == 0 or len(rows) == 0:
                    continue
                A = self._block(side, rows, fp)
                r, rp, cp = O.aca(A, self.maxrank, self.tol, True)
                if r == 0:
                    continue
                piv[item] = rows[rp]
                X[item] = O.cross_solve(A[:, cp], rp)
        self.piv[side] = piv
        self.X[side] = X

    def _couplings(self):
        Dt, Ds = self.dirs
        pos = {}
        for s in range(self.trees[1].nnodes):
            for q in range(Ds.farptr[s], Ds.farptr[s + 1]):
                pos[(s, int(Ds.farnodes[q]))] = q
        item_of = [np.zeros(len(D.farnodes), np.int32) for D in self.dirs]
        for D, io in zip(self.dirs, item_of):
            for it in range(D.nitems):
                io[D.dirfarptr[it]:D.dirfarptr[it + 1]] = it
        self.C = {}
        for t in range(self.trees[0].nnodes):
            for e in range(Dt.farptr[t], Dt.farptr[t + 1]):
                s = int(Dt.farnodes[e])
                it, is_ = int(item_of[0][e]), int(item_of[1][pos[(s, t)]])
                if len(self.piv[0][it]) and len(self.piv[1][is_]):
                    self.C[(it, is_)] = self._block(0, self.piv[0][it], self.piv[1][is_])

    def apply(self, x, mode=0):
        """y = op(H) x for a vector or a block of columns; mode 0: H, 1: H^T, 2: H^H."""
        x = np.asarray(x, dtype=np.complex128)
        vec = x.ndim == 1
        X = x.reshape(x.shape[0], -1)
        I = 1 if mode == 0 else 0
        O_ = 1 - I
        conj = (lambda a: a.conj()) if mode == 2 else (lambda a: a)
        DI, DO = self.dirs[I], self.dirs[O_]
        TI, TO = self.trees[I], self.trees[O_]
        XI, XO = self.X[I], self.X[O_]
        xhat = [None] * DI.nitems
        for level in range(TI.nlevels - 1, -1, -1):
            for it in range(DI.nitems):
                if XI[it] is None or TI.level[DI.item_node[it]] != level:
                    continue
                if DI.item_basis[it]:
                    xhat[it] = conj(XI[it]).T @ X[TI.values(int(DI.item_node[it]))]
                else:
                    acc, r0 = np.zeros((XI[it].shape[1], X.shape[1]), complex), 0
                    for ch in DI.item_chidx[DI.item_chptr[it]:DI.item_chptr[it + 1]]:
                        rc = 0 if XI[ch] is None else XI[ch].shape[1]
                        if rc:
                            acc = acc + conj(XI[it][r0:r0 + rc]).T @ xhat[ch]
                        r0 += rc
                    xhat[it] = acc
        yhat = [None if XO[it] is None else np.zeros((XO[it].shape[1], X.shape[1]), complex) for it in range(DO.nitems)]
        for (it, is_), Cb in self.C.items():
            if mode == 0:
                yhat[it] += Cb @ xhat[is_]
            else:
                yhat[is_] += conj(Cb).T @ xhat[it]
        Y = np.zeros((TO.perm.shape[0], X.shape[1]), complex)
        for level in range(TO.nlevels):
            for it in range(DO.nitems):
                if XO[it] is None or TO.level[DO.item_node[it]] != level:
                    continue
                if DO.item_basis[it]:
                    Y[TO.values(int(DO.item_node[it]))] += conj(XO[it]) @ yhat[it]
                else:
                    r0 = 0
                    for ch in DO.item_chidx[DO.item_chptr[it]:DO.item_chptr[it + 1]]:
                        rc = 0 if XO[ch] is None else XO[ch].shape[1]
                        if rc:
                            yhat[ch] = yhat[ch] + conj(XO[it][r0:r0 + rc]) @ yhat[it]
                        r0 += rc
        nptr, nnodes = (self.nearptr, self.nearnodes) if mode == 0 else (self.tnearptr, self.tnearnodes)
        for t in range(TO.nnodes):
            for s in nnodes[nptr[t]:nptr[t + 1]]:
                rows, cols = TO.values(t), TI.values(int(s))
                Nb = self._block(0, rows, cols) if mode == 0 else self._block(0, cols, rows).T
                Y[rows] += conj(Nb) @ X[cols]
        return Y[:, 0] if vec else Y
