"""CSR helpers of the reference (src/utils/utils.jl:2-30, src/nca/abstractnca.jl:106-119),
0-based: entry i owns ptr[i]:ptr[i+1]."""
from __future__ import annotations

import numpy as np


def ptrfromcounts(counts):
    counts = np.asarray(counts, dtype=np.int64)
    ptr = np.zeros(len(counts) + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    return ptr


def collect_assigned(v):
    """Compact a list whose unassigned entries are None: (blocks, indices)."""
    nodes = [i for i, b in enumerate(v) if b is not None]
    return [v[i] for i in nodes], nodes


class CoefficientPlan:
    def __init__(self, globalidxtocoeffptr):
        self.globalidxtocoeffptr = np.asarray(globalidxtocoeffptr, dtype=np.int64)


def plan_from_pivots(pivots) -> CoefficientPlan:
    """Coefficient range of every node: as many coefficients as pivots (None counts 0)."""
    return CoefficientPlan(ptrfromcounts([0 if p is None else len(p) for p in pivots]))
