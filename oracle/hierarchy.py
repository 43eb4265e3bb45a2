"""CPU restatement of the smoothed-aggregation level chain (test infrastructure).

ORACLE -- only tests and the CPU baseline may import this module.

The reference's test operators are dumps of an AMG coarsening chain,
lLEV_ac = lLEV_r * l(LEV-1)_ac * lLEV_p (code/scripts/getLevels3MMmatrixes.py:29-38);
the device hierarchy (sp3mm_hierarchy_build) produces such a chain on a box
grid.  This module restates every step on the CPU with the same arithmetic,
so the device levels can be checked bit for bit:

* P0: block^d aggregation of the grid (problems.block_aggregation);
* A P0 with the C oracle's Gustavson product (structural zeros kept, the
  reference's behaviour, code/src/Sp3MM_CSR_OMP_UB_Generic.c:56-124);
* P = [j == agg(i)] - (omega / d_i) * (A P0)_ij with separately rounded
  IEEE operations (numpy float64, no fused multiply-add);
* R = P^T; A_{l+1} = R A P with the oracle's direct product
  (code/src/Sp3MM_CSR_OMP_UB_Generic.c:498-573).

FP32 storage is emulated exactly: a value stored in FP32 is the FP64 result
rounded once (np.float32), and later FP64 arithmetic reads it back widened.
"""
from __future__ import annotations

import numpy as np

from sp3mm4amg_b200.problems import CSR, block_aggregation


def _round(m: CSR, f32: bool) -> CSR:
    if not f32:
        return m
    return CSR(m.indptr, m.indices, m.data.astype(np.float32).astype(np.float64), m.shape)


def diagonal(A: CSR) -> np.ndarray:
    d = np.zeros(A.M)
    rows = np.repeat(np.arange(A.M), np.diff(A.indptr))
    on = A.indices == rows
    d[rows[on]] = A.data[on]
    return d


def block_prolongator(orc, A: CSR, dims, block: int, omega: float, f32: bool = False) -> CSR:
    """P = (I - omega D^-1 A) P0 on the pattern of A*P0 (values rounded to
    FP32 when f32)."""
    P0 = block_aggregation(dims, block)
    AP0 = orc.spmm(A, P0)
    d = diagonal(A)
    if np.any(d == 0.0):
        raise ValueError("a row of A has no diagonal entry")
    s = np.float64(omega) / d
    rows = np.repeat(np.arange(A.M), np.diff(AP0.indptr))
    y = s[rows] * AP0.data
    agg = P0.indices[rows]
    v = np.where(AP0.indices == agg, 1.0 - y, -y)
    return _round(CSR(AP0.indptr, AP0.indices, v, AP0.shape), f32)


def coarse_dims(dims, block: int):
    return tuple(-(-int(d) // block) for d in dims)


def chain(orc, A0: CSR, dims, block: int = 2, omega: float = 2.0 / 3.0,
          min_coarse: int = 64, max_levels: int = 10, coarse_f32: bool = False):
    """[(A_l, P_l, R_l)], P/R None on the last level; same stopping rule as
    the device build (stop at max_levels or when A_l has < min_coarse rows)."""
    levels = []
    A, dims = A0, tuple(dims)
    while len(levels) + 1 < max_levels and A.M >= min_coarse and A.M > 1:
        l = len(levels)
        P = block_prolongator(orc, A, dims, block, omega, f32=coarse_f32 and l > 0)
        R = P.transpose()
        Ac = _round(orc.sp3mm_direct(R, A, P), coarse_f32)
        levels.append((A, P, R))
        A, dims = Ac, coarse_dims(dims, block)
    levels.append((A, None, None))
    return levels
