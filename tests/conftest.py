"""Test configuration: the `gpu` marker, import paths and shared workload builders."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "nestedcrossapproximation.jl_b200"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def grid_c1():
    """1,024 points on a 32 x 32 grid of the unit square at z = 0 (x fastest), trial points
    shifted by (1.1, 0, 0.2): the CPU-runnable plain configuration."""
    g = np.linspace(0.0, 1.0, 32)
    X, Y = np.meshgrid(g, g, indexing="ij")
    test = np.stack([X.ravel(order="F"), Y.ravel(order="F"), np.zeros(1024)], axis=1)
    return test, test + np.array([1.1, 0.0, 0.2])


def sphere(n, seed):
    """n points uniform on the unit sphere (normalised Gaussian triples, seeded)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, 3))
    return g / np.linalg.norm(g, axis=1, keepdims=True)


def cgauss(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def cube_surface(n, seed):
    """n points uniform on the surface of the unit cube [0, 1]^3 (face chosen uniformly, then a
    uniform point on it), seeded."""
    rng = np.random.default_rng(seed)
    face = rng.integers(0, 6, n)
    uv = rng.uniform(0.0, 1.0, (n, 2))
    pts = np.empty((n, 3))
    axis = face // 2
    for a in range(3):
        sel = axis == a
        others = [b for b in range(3) if b != a]
        pts[sel, a] = (face[sel] % 2).astype(float)
        pts[sel, others[0]] = uv[sel, 0]
        pts[sel, others[1]] = uv[sel, 1]
    return pts
