"""nca_b200: batched bottom-up nested cross approximation and H^2 products on one B200.

The Python face mirrors NestedCrossApproximation.jl's API for this path (PetrovGalerkinNCA,
H2Workspace, BatchedBottomUp, BottomUp, TreeMimicryPivoting, ACA, IACA, KMeansTree, BlockTree, isnear, mul,
transpose, adjoint, storage, farmatrix/nearmatrix stores); all arithmetic runs in
libnca_b200.so (hand-written sm_100a kernels behind a C ABI, include/nca_b200.h).
"""
from . import seams
from ._lib import (ArgumentError, ConcurrentWorkspaceError, CudaError, DimensionMismatch, SingularCrossMatrixError,
                   LIBPATH, lib)
from .admissibility import DirectionalData, FarData, IsNearWideband, directionalfardata, fardata, farfield, farinteractions, farnodes, farptr, interactions, isnear, \
    isnearwideband
from .compressors import ACA, IACA, BatchedBottomUp, BottomUp, FNormEstimator, FNormExtrapolator, FullPivoting, \
    MaximumValue, TreeMimicryPivoting, _clustersize, _selectfarpivots
from .kernels import HelmholtzKernel, LaplaceKernel, MatrixKernel
from .nca import (BatchCore, H2Workspace, LoadedCore, load_core, dHdk, rrule_mul, PetrovGalerkinNCA, PetrovGalerkinNCACore, adjoint, batch, core, farmatrix, mul, nearmatrix,
                  storage, transpose, withworkspace)
from .trees import BlockTree, KMeansTree, KMeansTreeBuilder, testtree, trialtree
from .utils import collect_assigned, plan_from_pivots, ptrfromcounts

__all__ = [n for n in dir() if not n.startswith("__")]
