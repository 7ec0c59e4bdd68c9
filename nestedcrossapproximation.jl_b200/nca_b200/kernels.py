"""Point kernels of the device entry generator.

HelmholtzKernel(k) is cis(k r)/(4 pi r) (README.md:100-108); sign=-1 gives exp(-ikr)/(4 pi r)
(test/nca/test_petrovgalerkinnca.jl:14-17); rmin sets entries with r < rmin to zero
(test/testutils.jl:18-21; r == 0 is always zero). MatrixKernel(M) evaluates entry (i, j) of a
given matrix, like AdaptiveCrossApproximation.PointMatrix in test/test_couplingmatrices.jl:15.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import BuildOpts, KernelDesc

KIND_HELMHOLTZ, KIND_LAPLACE, KIND_MATRIX = 0, 1, 2


class PointKernel:
    kind = KIND_HELMHOLTZ
    k = 0.0
    sign = 1
    rmin = 0.0
    matrix = None

    def desc(self) -> KernelDesc:
        d = KernelDesc()
        d.kind, d.sign, d.k, d.rmin = self.kind, self.sign, float(self.k), float(self.rmin)
        if self.matrix is not None:
            d.matrix = self.matrix.ctypes.data_as(C.c_void_p)
            d.ldmatrix = self.matrix.shape[0]
        return d

    def __call__(self, x, y):
        r = float(np.linalg.norm(np.asarray(x) - np.asarray(y)))
        if r == 0.0 or r < self.rmin:
            return 0j
        if self.kind == KIND_LAPLACE:
            return 1.0 / (4 * np.pi * r) + 0j
        return np.exp(1j * self.sign * self.k * r) / (4 * np.pi * r)


class HelmholtzKernel(PointKernel):
    def __init__(self, k: float, sign: int = 1, rmin: float = 0.0):
        self.kind, self.k, self.sign, self.rmin = KIND_HELMHOLTZ, float(k), 1 if sign >= 0 else -1, float(rmin)


class LaplaceKernel(PointKernel):
    def __init__(self, rmin: float = 0.0):
        self.kind, self.rmin = KIND_LAPLACE, float(rmin)


class MatrixKernel(PointKernel):
    """Entries taken from a dense matrix (rows: test indices, columns: trial indices)."""

    def __init__(self, M):
        self.kind = KIND_MATRIX
        self.matrix = np.asfortranarray(M, dtype=np.complex128)

    def __call__(self, i, j):
        return self.matrix[i, j]


__all__ = ["HelmholtzKernel", "LaplaceKernel", "MatrixKernel", "BuildOpts"]
