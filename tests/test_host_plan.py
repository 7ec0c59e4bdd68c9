"""Host side of the library on the CPU: the C ABI loads and exports its declared entry points;
the tree, the partition and phase-1 far pivots equal the oracle's bit for bit; the
reference's structural KATs for CSR helpers, far data, farfield and _selectfarpivots."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, sphere

import nca_b200 as N
from oracle import oracle as O


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "nca_b200.h")).read()
    declared = set(re.findall(r"^(?:int32_t|void)\s+\**(nca_\w+)\(", header, re.M))
    assert len(declared) >= 25
    lib = N.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert set(N._lib.SIGNATURES) == declared
    assert lib.nca_version() == 2


@pytest.mark.parametrize("n,mv,seed", [(1024, 32, 1), (5000, 20, 2), (30000, 64, 3)])
def test_tree_and_partition_match_oracle(n, mv, seed):
    pts = sphere(n, seed) * np.array([1.0, 0.7, 1.3])
    other = sphere(n // 2, seed + 10) + np.array([0.4, 0.0, 0.1])
    tt = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=mv))
    st = N.KMeansTree(other, N.KMeansTreeBuilder(minvalues=mv))
    for tree, p in ((tt, pts), (st, other)):
        ot = O.OwnedTree(p, mv)
        assert tree.nnodes == ot.nnodes
        for name in ("perm", "begin", "end", "nchildren", "level"):
            assert np.array_equal(getattr(tree, name), getattr(ot, name)), name
        assert np.array_equal(tree._center, ot.center) and np.array_equal(tree._radius, ot.radius)
        # invariants: children partition the parent, leaves hold at most minvalues points
        assert np.array_equal(np.sort(tree.perm), np.arange(len(p)))
        for node in range(tree.nnodes):
            if tree.isleaf(node):
                assert tree.numberofvalues(node) <= mv
            else:
                ch = tree.children(node)
                assert tree.begin[ch[0]] == tree.begin[node] and tree.end[ch[-1]] == tree.end[node]
                assert tree.level[ch[0]] == tree.level[node] + 1
    part = N.interactions(N.BlockTree(tt, st), N.isnear())
    H = O.H2(pts, other, O.Kernel(O.KIND_LAPLACE), minvalues=mv, tol=1e-3, maxrank=20)
    for name in ("nearptr", "nearnodes", "farptr", "farnodes", "tfarptr", "tfarnodes"):
        src = {"tfarptr": "trialfarptr", "tfarnodes": "trialfarnodes"}.get(name, name)
        assert np.array_equal(getattr(part, src), getattr(H, name)), name
    # phase 1 for every node of both sides
    fd_test, fd_trial = N.fardata(N.BlockTree(tt, st), N.isnear(), part)
    for side, (own, far, ownp, farp, fd) in enumerate(((tt, st, pts, other, fd_test), (st, tt, other, pts, fd_trial))):
        sel = N.TreeMimicryPivoting(ownp, farp, far)
        for node in range(own.nnodes):
            ff = N.farfield(own, fd, node)
            got = N._selectfarpivots(sel, own.values(node), ff, far, 20) if len(ff) else np.zeros(0, np.int32)
            assert np.array_equal(got, H.farpivots[side][node]), (side, node)


def test_interaction_invariants():
    """test/admissibility/test_farinteractions.jl:44-80."""
    rng = np.random.default_rng(1)
    cases = [(rng.random((300, 3)), rng.random((300, 3)), 10, 10),
             (rng.random((200, 3)), rng.random((200, 3)) + np.array([1.0, 0, 0]), 10, 25),
             (rng.random((40, 3)), rng.random((40, 3)) + np.array([3.0, 0, 0]), 100, 100)]
    isnear = N.isnear()
    for tp, sp, mt, ms in cases:
        tt = N.KMeansTree(tp, N.KMeansTreeBuilder(minvalues=mt))
        st = N.KMeansTree(sp, N.KMeansTreeBuilder(minvalues=ms))
        tree = N.BlockTree(tt, st)
        part = N.interactions(tree, isnear)
        rootsfar = not isnear(tt, st, 0, 0)
        testdata, trialdata = N.fardata(tree, isnear, part)
        testpairs = [(t, int(s)) for t in range(tt.nnodes) for s in N.farnodes(testdata, t)]
        trialpairs = [(int(t), s) for s in range(st.nnodes) for t in N.farnodes(trialdata, s)]
        assert testpairs and len(set(testpairs)) == len(testpairs)
        assert sorted(testpairs) == sorted(trialpairs)
        assert all(not isnear(tt, st, t, s) for t, s in testpairs)
        if not rootsfar:
            assert all(isnear(tt, st, tt.parent(t) if t else 0, st.parent(s) if s else 0)
                       for t, s in testpairs if t and s)
        covered = np.zeros((len(tp), len(sp)), int)
        for t in range(tt.nnodes):
            for s in part.nearnodes[part.nearptr[t]:part.nearptr[t + 1]]:
                covered[np.ix_(tt.values(t), st.values(s))] += 1
        for t, s in testpairs:
            covered[np.ix_(tt.values(t), st.values(s))] += 1
        assert np.all(covered == 1)
        assert rootsfar == (mt == 100)


def test_fardata_kats():
    """FarData accessors and farfield order (test_farinteractions.jl:84-123)."""
    data = N.FarData([0, 2, 2, 4], [7, 8, 9, 10])
    assert list(N.farnodes(data, 0)) == [7, 8] and len(N.farnodes(data, 1)) == 0
    assert list(N.farnodes(data, 2)) == [9, 10]
    pts = np.random.default_rng(3).random((60, 3))
    tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=4))
    leaf = max(n for n in range(tree.nnodes) if tree.isleaf(n))
    chain = [leaf] + tree.parents_upwards(leaf)
    assert len(chain) >= 3
    counts = np.zeros(tree.nnodes, int)
    counts[chain] = 1
    data = N.FarData(N.ptrfromcounts(counts), 10 * np.sort(chain))
    assert list(N.farfield(tree, data, leaf)) == [10 * c for c in chain]
    counts[leaf] = 0
    nofar = N.FarData(N.ptrfromcounts(counts), 10 * np.sort(chain[1:]))
    assert len(N.farnodes(nofar, leaf)) == 0
    assert list(N.farfield(tree, nofar, leaf)) == [10 * c for c in chain[1:]]


def test_csr_helper_kats():
    """test/utils/test_utils.jl:6-52 and test/nca/test_abstractnca.jl:9-24 (0-based)."""
    assert list(N.ptrfromcounts([2, 0, 3, 1])) == [0, 2, 2, 5, 6]
    assert list(N.ptrfromcounts([])) == [0]
    blocks, nodes = N.collect_assigned([None, [1, 2], None, None, [3]])
    assert nodes == [1, 4] and blocks == [[1, 2], [3]]
    assert N.collect_assigned([None] * 3) == ([], [])
    assert list(N.plan_from_pivots([[1, 2], [7, 8, 9], [], [4]]).globalidxtocoeffptr) == [0, 2, 5, 5, 6]
    assert list(N.plan_from_pivots([None, [1, 2], None, []]).globalidxtocoeffptr) == [0, 0, 2, 2, 2]
    assert list(N.plan_from_pivots([]).globalidxtocoeffptr) == [0]


def test_selectfarpivots_kats():
    """test/compressors/test_batchedbottomup.jl:55-114 on the library's host planner."""
    rng = np.random.default_rng(8)
    testpts = rng.random((150, 3))
    trialpts = rng.random((200, 3)) + np.array([3.0, 0, 0])
    ttree = N.KMeansTree(testpts, N.KMeansTreeBuilder(minvalues=15))
    stree = N.KMeansTree(trialpts, N.KMeansTreeBuilder(minvalues=15))
    sel = N.TreeMimicryPivoting(testpts, trialpts, stree)
    cluster = ttree.values(0)
    farnodes = stree.children(0)
    farvalues = np.concatenate([stree.values(n) for n in farnodes])
    for node in range(stree.nnodes):
        for cap in (0, 1, 7, 30, 300):
            assert N._clustersize(stree, node, cap) == min(cap, stree.numberofvalues(node))
    small = [n for n in range(stree.nnodes) if stree.isleaf(n) and 0 < stree.numberofvalues(n) <= 15][:2]
    actual = np.concatenate([stree.values(n) for n in small])
    got = N._selectfarpivots(sel, cluster, small, stree, 25)
    assert sorted(got) == sorted(actual) or len(got) == 25
    piv = N._selectfarpivots(sel, cluster, farnodes, stree, 25)
    assert len(piv) == 25 and len(set(piv)) == 25 and set(piv) <= set(farvalues)
    assert np.array_equal(N._selectfarpivots(sel, cluster, farnodes, stree, 25), piv)
    assert len(N._selectfarpivots(sel, cluster[:7], farnodes, stree, 25)) == 7
    leaf = next(n for n in range(stree.nnodes) if stree.isleaf(n))
    assert stree.numberofvalues(leaf) < 25
    assert sorted(N._selectfarpivots(sel, cluster, [leaf], stree, 25)) == sorted(stree.values(leaf))
    assert len(N._selectfarpivots(sel, np.zeros(0, np.int32), farnodes, stree, 25)) == 0
    assert len(N._selectfarpivots(sel, cluster, farnodes, stree, 0)) == 0
    # the first pivot is the far point closest to the cluster centroid
    c = testpts[cluster].mean(axis=0)
    d = np.linalg.norm(trialpts[farvalues] - c, axis=1)
    assert np.linalg.norm(trialpts[piv[0]] - c) <= d.min() * (1 + 0.5)


def test_batchedbottomup_constructor():
    """test/compressors/test_batchedbottomup.jl:18-41."""
    pts = np.random.default_rng(0).random((50, 3))
    tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=10))
    sel = N.TreeMimicryPivoting(pts, pts, tree)
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-3))
    c = N.BatchedBottomUp(pivotselector=sel, compressor=aca)
    assert c.pivotselector is sel and c.compressor is aca
    assert type(N.BatchedBottomUp(sel, aca)) is type(c)
    for kwargs in ({}, {"pivotselector": sel}, {"compressor": aca}):
        with pytest.raises(TypeError):
            N.BatchedBottomUp(**kwargs)


def test_load_refuses_files_that_are_not_saved_cores(tmp_path):
    """nca_core_load checks the tag, the format number and every array count against the file
    before any device work: a foreign or truncated file is an ArgumentError."""
    p = tmp_path / "junk.nca"
    p.write_bytes(b"not a core at all" * 10)
    with pytest.raises(N.ArgumentError, match="not a saved core"):
        N.load_core(str(p))
    p.write_bytes(b"NCAB200C" + (1).to_bytes(4, "little") + b"\x00" * 6)
    with pytest.raises(N.ArgumentError, match="truncated"):
        N.load_core(str(p))
    with pytest.raises(N.ArgumentError, match="cannot open"):
        N.load_core(str(tmp_path / "missing.nca"))
