"""The k-means cluster tree built on the device equals the host planner's tree bit for bit
(permutation, node ranges, levels, centres, radii) — and so the oracle's, which the host tree is
checked against in test_host_plan.py — on spheres, a stretched cloud, clusters of repeated points
and sizes around the 256-point summation chunks."""
import os

import numpy as np
import pytest

from conftest import sphere

import nca_b200 as N

pytestmark = pytest.mark.gpu


def _tree(pts, mv, host):
    old = os.environ.get("NCA_TREE_DEVICE")
    if host:
        os.environ.pop("NCA_TREE_DEVICE", None)
    else:
        os.environ["NCA_TREE_DEVICE"] = "1"
    try:
        return N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=mv))
    finally:
        if old is None:
            os.environ.pop("NCA_TREE_DEVICE", None)
        else:
            os.environ["NCA_TREE_DEVICE"] = old


def _cases():
    rng = np.random.default_rng(5)
    stretched = rng.standard_normal((100_000, 3)) * np.array([3.0, 1.0, 0.2])
    repeated = np.repeat(sphere(2_000, 9), 12, axis=0)  # 24,000 points, every one 12 times
    return [
        ("sphere 262144", sphere(262_144, 888), 64),
        ("sphere 20000", sphere(20_000, 3), 32),
        ("stretched 100000", stretched, 64),
        ("repeated 24000", repeated, 20),
        ("sphere 16641", sphere(16_641, 4), 16),
    ]


@pytest.mark.parametrize("name,pts,mv", _cases(), ids=[c[0] for c in _cases()])
def test_device_tree_equals_host_tree(name, pts, mv):
    d = _tree(pts, mv, host=False)
    h = _tree(pts, mv, host=True)
    assert d.nnodes == h.nnodes and d.nlevels == h.nlevels
    for field in ("perm", "begin", "end", "nchildren", "level"):
        assert np.array_equal(getattr(d, field), getattr(h, field)), field
    assert np.array_equal(d._center, h._center)
    assert np.array_equal(d._radius, h._radius)
    assert np.array_equal(np.sort(d.perm), np.arange(len(pts)))
