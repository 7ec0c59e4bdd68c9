"""Host plan of directional (wideband) H^2 matrices against the oracle restatement.

The wideband partition, the direction sets, the far nodes grouped by direction, the
parent-to-child direction maps, the basis items with their children's items and every item's
far field (dirfarfield) must agree exactly with the oracle (oracle/directional.py, a line-by-line
restatement of src/admissibility/nearinteractions.jl, directionalsubdivision/*.jl and
src/compressors/bottomup.jl:214-320)."""
import numpy as np
import pytest

from conftest import sphere


def _n():
    import nca_b200
    return nca_b200


def _o():
    from oracle import directional, oracle
    return oracle, directional


CASES = [
    ("sphere k=6", lambda: (sphere(3000, 1), None), 6.0, 32),
    ("sphere k=40", lambda: (sphere(3000, 2), None), 40.0, 32),
    ("two spheres k=12", lambda: (sphere(1800, 3), sphere(1500, 4) * 0.7 + np.array([2.5, 0.3, 0.0])), 12.0, 24),
]


@pytest.mark.parametrize("name,make,k,minvalues", CASES, ids=[c[0] for c in CASES])
def test_directional_plan_matches_oracle(name, make, k, minvalues):
    N = _n()
    O, D = _o()
    test, trial = make()
    trial = test if trial is None else trial
    tt = N.KMeansTree(test, N.KMeansTreeBuilder(minvalues=minvalues))
    st = N.KMeansTree(trial, N.KMeansTreeBuilder(minvalues=minvalues))
    bt = N.BlockTree(tt, st)
    P = N.interactions(bt, N.isnearwideband(k))
    ot, os_ = O.OwnedTree(test, minvalues), O.OwnedTree(trial, minvalues)
    nptr, nnodes, fptr, fnodes, tptr, tnodes = D.interactions_wideband(ot, os_, k)
    assert np.array_equal(P.nearptr, nptr) and np.array_equal(P.nearnodes, nnodes)
    assert np.array_equal(P.farptr, fptr) and np.array_equal(P.farnodes, fnodes)
    assert np.array_equal(P.trialfarptr, tptr) and np.array_equal(P.trialfarnodes, tnodes)
    dev = N.directionalfardata(bt, P)
    ref = (D.DirectionalData(ot, os_, fptr, fnodes, k), D.DirectionalData(os_, ot, tptr, tnodes, k))
    nhf = 0
    for side in (0, 1):
        a, b = dev[side], ref[side]
        assert a.nitems == b.nitems, side
        for f in ("farnodes", "dirptr", "dirs", "dirfarptr", "item_basis", "item_chptr", "item_chidx"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), (side, f)
        assert np.array_equal(a.dirvec, b.dirvec)
        for item in range(a.nitems):
            assert np.array_equal(a.farfield(item), b.farfield(item)), (side, item)
        nhf += int((a.dirs != 0).sum())
    if k >= 12:
        assert nhf > 0  # the case exercises high-frequency directions


def test_wideband_reduces_to_lowfrequency_ball_condition():
    """With k = 0 every pair is low frequency: the partition equals isnear(eta_lf)."""
    N = _n()
    pts = sphere(2000, 5)
    t = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=32))
    bt = N.BlockTree(t, t)
    a = N.interactions(bt, N.isnearwideband(0.0, etalf=1.0))
    b = N.interactions(bt, N.isnear(1.0))
    assert np.array_equal(a.farnodes, b.farnodes) and np.array_equal(a.nearnodes, b.nearnodes)
    da, _ = N.directionalfardata(bt, a)
    assert np.all(da.dirs == 0)
