"""ctypes binding of libnca_b200.so and the mapping of its status codes onto exceptions.

The exception types mirror the reference's: SingularCrossMatrixError
(src/utils/utils.jl:38-54), ConcurrentWorkspaceError (src/nca/petrovgalerkinnca.jl:210-218),
DimensionMismatch and ArgumentError.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libnca_b200.so")

NCA_OK, NCA_ERR_SINGULAR, NCA_ERR_DIM, NCA_ERR_ARG, NCA_ERR_CUDA, NCA_ERR_TIMEOUT, NCA_ERR_OOM, NCA_ERR_BUSY = range(8)


class SingularCrossMatrixError(Exception):
    """The cross matrix A[pivots, cols] of a cluster is singular (coincident points)."""

    def __init__(self, kind, npivots, rank, message=""):
        self.kind, self.npivots, self.rank = kind, npivots, rank
        super().__init__(message or f"SingularCrossMatrixError: the cross matrix for a {kind} is singular - "
                         f"{npivots} pivots were selected but only {rank} of them are linearly independent.")


class ConcurrentWorkspaceError(Exception):
    def __init__(self, message=""):
        super().__init__(message or "ConcurrentWorkspaceError: the workspace is in use by another matrix-vector "
                         "product. Create one H2Workspace per task; they can share the core.")


class DimensionMismatch(ValueError):
    pass


class ArgumentError(ValueError):
    pass


class CudaError(RuntimeError):
    pass


class NCAStruct(C.Structure):
    pass


class KernelDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("sign", C.c_int32), ("k", C.c_double), ("rmin", C.c_double),
                ("matrix", C.c_void_p), ("ldmatrix", C.c_int64)]


class BuildOpts(C.Structure):
    _fields_ = [("tol_test", C.c_double), ("tol_trial", C.c_double), ("maxrank", C.c_int32),
                ("sampled", C.c_int32), ("device", C.c_int32), ("store_f32", C.c_int32),
                ("compressor", C.c_int32)]


class CoreInfo(C.Structure):
    _fields_ = [("ntest", C.c_int64), ("ntrial", C.c_int64), ("nnodes_test", C.c_int32),
                ("nnodes_trial", C.c_int32), ("ncoeff_test", C.c_int64), ("ncoeff_trial", C.c_int64),
                ("near_entries", C.c_int64), ("coupling_entries", C.c_int64),
                ("basis_entries_test", C.c_int64), ("basis_entries_trial", C.c_int64),
                ("transfer_entries_test", C.c_int64), ("transfer_entries_trial", C.c_int64),
                ("nfarpairs", C.c_int64), ("nnearpairs", C.c_int64), ("build_seconds", C.c_double),
                ("build_seconds_host", C.c_double)]


# name -> (restype, argtypes); every entry point of include/nca_b200.h
P, I32, I64, D, SZ = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_size_t
SIGNATURES = {
    "nca_version": (I32, []),
    "nca_last_error": (I32, [C.c_char_p, SZ]),
    "nca_last_singular": (I32, [P, P, P, P]),
    "nca_tree_kmeans": (I32, [P, I64, I32, I32, P]),
    "nca_tree_destroy": (None, [P]),
    "nca_tree_sizes": (I32, [P, P, P, P]),
    "nca_tree_export": (I32, [P] * 10),
    "nca_interactions": (I32, [P, P, D, P]),
    "nca_interactions_wideband": (I32, [P, P, D, D, D, D, P]),
    "nca_partition_destroy": (None, [P]),
    "nca_directional_plan": (I32, [P, P, P, I32, P]),
    "nca_dirplan_destroy": (None, [P]),
    "nca_dirplan_sizes": (I32, [P, P, P, P]),
    "nca_dirplan_export": (I32, [P] * 9),
    "nca_dirplan_farfield": (I32, [P, I32, P, I32, P]),
    "nca_partition_sizes": (I32, [P, P, P]),
    "nca_partition_export": (I32, [P] * 7),
    "nca_select_farpivots": (I32, [P, P, P, P, I32, P, I32, I32, P, P]),
    "nca_core_build": (I32, [P, I64, P, I64, P, P, P, P, P, P]),
    "nca_core_destroy": (None, [P]),
    "nca_core_save": (I32, [P, C.c_char_p]),
    "nca_core_load": (I32, [C.c_char_p, I32, P]),
    "nca_core_batch": (I32, [P, I32, I32, P]),
    "nca_core_get_info": (I32, [P, P]),
    "nca_core_export_pivots": (I32, [P, I32, P, P, P, P]),
    "nca_core_dir_items": (I32, [P, I32, P, P, P, P, P]),
    "nca_core_farpivots_total": (I32, [P, I32, P]),
    "nca_core_export_farpivots": (I32, [P, I32, P, P]),
    "nca_core_export_x": (I32, [P, I32, P, P]),
    "nca_core_export_couplings": (I32, [P, P, P]),
    "nca_core_export_near": (I32, [P, P, P, P]),
    "nca_workspace_create": (I32, [P, I32, P]),
    "nca_workspace_destroy": (None, [P]),
    "nca_apply": (I32, [P, I32, I32, P, I64, P, I64, I64, D, D, D, D, I32]),
    "nca_apply_static": (I32, [P, I32, I32, P, I64, P, I64, I64, D, D, D, D, P]),
    "nca_workspace_last_time": (I32, [P, P]),
    "nca_workspace_last_launches": (I32, [P, P]),
    "nca_workspace_set_parts": (I32, [P, I32, I32]),
    "nca_workspace_set_profiling": (I32, [P, I32]),
    "nca_workspace_stage_times": (I32, [P, P, P, I32]),
    "nca_workspace_set_graphs": (I32, [P, I32]),
    "nca_workspace_autotune": (I32, [P, I32, I32, I64, P]),
    "nca_blocks_aca": (I32, [P, I64, I32, P, P, I32, I32, D, I32, I32, P, P, P]),
    "nca_blocks_factors": (I32, [P, I64, I32, P, I32, P, P, P, I32, I32, P, P]),
    "nca_entries": (I32, [P, P, I64, P, I64, P, P, I64, I32, P]),
    "nca_entries_dk": (I32, [P, P, I64, P, I64, P, P, I64, I32, P]),
    "nca_core_set_wavenumber": (I32, [P, D]),
    "nca_core_prepare_dk": (I32, [P]),
    "nca_apply_dk": (I32, [P, P, I64, P, I64, I64, D, D, D, D, I32]),
}

_lib = None


def lib():
    """The loaded library. Raises if it has not been built: there is no fallback path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise ImportError(
                f"{LIBPATH} is missing: build it with `python nestedcrossapproximation.jl_b200/build.py` "
                "(the library has no CPU fallback)")
        L = C.CDLL(LIBPATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(2048)
    lib().nca_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, kind: str = "cross matrix"):
    if status == NCA_OK:
        return
    msg = last_error()
    if status == NCA_ERR_SINGULAR:
        side, node, npiv, rank = (C.c_int32() for _ in range(4))
        lib().nca_last_singular(C.byref(side), C.byref(node), C.byref(npiv), C.byref(rank))
        err = SingularCrossMatrixError(kind, npiv.value, rank.value, msg)
        err.side, err.node = side.value, node.value
        raise err
    if status == NCA_ERR_DIM:
        raise DimensionMismatch(msg)
    if status == NCA_ERR_ARG:
        raise ArgumentError(msg)
    if status == NCA_ERR_BUSY:
        raise ConcurrentWorkspaceError(msg)
    if status == NCA_ERR_OOM:
        raise MemoryError(msg)
    raise CudaError(f"status {status}: {msg}")


def ptr(a):
    """Address of a numpy array or a torch tensor (device or host)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)
