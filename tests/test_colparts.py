"""2D column-partition utilities (colsOffsetsPartitioningUnifRanges_,
colsPartitioningUnifRanges_, colsPartitioningUnifRangesOffsetsAux_; the
reference's code/src/commons/sparseUtilsGeneric.c:284-400), host code.

Checked against a numpy restatement of the reference's loops on every
golden matrix and grid, in both index bases, and -- where the reference
library was built here (oracle/_ref) -- against the reference's own
functions, array for array.  No GPU is used.
"""
import ctypes
import os

import numpy as np
import pytest

from sp3mm4amg_b200 import capi, problems as pb
from sp3mm4amg_b200.spmat import HostSpMat, SPMAT_P, idx_t, spmat

GRIDS = (1, 2, 3, 7)


def _ranges(n, grid):
    blk, rem = divmod(n, grid)
    starts = [g * blk + min(g, rem) for g in range(grid)]
    widths = [blk + (1 if g < rem else 0) for g in range(grid)]
    return starts, widths


def _want_offsets(A, grid):
    starts, _ = _ranges(A.N, grid)
    off = np.empty(A.M * grid + 1, np.int64)
    for r in range(A.M):
        cols = A.indices[A.indptr[r]:A.indptr[r + 1]]
        for gc in range(grid):
            off[r * grid + gc] = A.indptr[r] + np.searchsorted(cols, starts[gc])
    off[-1] = A.nnz
    return off


def _offsets_array(lib_fn, h, grid, M):
    p = lib_fn(h.ptr, grid)
    assert p
    out = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(idx_t)), shape=(M * grid + 1,))
    out = out.astype(np.int64)
    ctypes.CDLL(None).free(ctypes.c_void_p(p))
    return out


def _parts(p, grid):
    """Copy the gridCols partitions at p (spmat array) and free them."""
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    arr = ctypes.cast(p, ctypes.POINTER(spmat))
    out = []
    for g in range(grid):
        m = arr[g]
        M, N, NZ = int(m.M), int(m.N), int(m.NZ)
        irp = np.ctypeslib.as_array(m.IRP, shape=(M + 1,)).astype(np.int64)
        ja = np.ctypeslib.as_array(m.JA, shape=(NZ,)).astype(np.int64) if NZ else np.zeros(0, np.int64)
        as_ = np.ctypeslib.as_array(m.AS, shape=(NZ,)).copy() if NZ else np.zeros(0)
        out.append((M, N, NZ, irp, ja, as_))
        for a in (m.AS, m.JA, m.IRP):
            libc.free(ctypes.cast(a, ctypes.c_void_p))
    libc.free(ctypes.c_void_p(p))
    return out


def _want_parts(A, grid, off_f):
    offs = _want_offsets(A, grid)
    _, widths = _ranges(A.N, grid)
    out = []
    for g in range(grid):
        lens = np.array([offs[r * grid + g + 1] - offs[r * grid + g] for r in range(A.M)],
                        np.int64)
        irp = np.concatenate([[0], np.cumsum(lens)])
        sel = np.concatenate([np.arange(offs[r * grid + g], offs[r * grid + g + 1])
                              for r in range(A.M)]).astype(np.int64) if A.M else np.zeros(0, np.int64)
        out.append((A.M, widths[g], int(irp[-1]), irp, A.indices[sel] + off_f, A.data[sel]))
    return out


def _same_parts(got, want):
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert a[:3] == b[:3]
        for x, y in zip(a[3:], b[3:]):
            np.testing.assert_array_equal(x, y)


def _ref_lib():
    import oracle
    if not os.path.exists(oracle.REF_SO):
        return None
    lib = ctypes.CDLL(oracle.REF_SO)
    for off in (0, 1):
        for n in ("colsOffsetsPartitioningUnifRanges_", "colsPartitioningUnifRanges_"):
            f = getattr(lib, f"{n}{off}")
            f.restype = ctypes.c_void_p
            f.argtypes = [SPMAT_P, ctypes.c_uint]
        f = getattr(lib, f"colsPartitioningUnifRangesOffsetsAux_{off}")
        f.restype = ctypes.c_void_p
        f.argtypes = [SPMAT_P, ctypes.c_uint, ctypes.c_void_p]
    return lib


@pytest.mark.parametrize("off", [0, 1])
def test_column_partitions(golden, off):
    lib = capi.load()
    ref = _ref_lib()
    for name, g in golden.items():
        for A in (g["A"], g["P"]):
            h = HostSpMat(A, off)
            for grid in GRIDS:
                if grid > A.N:
                    continue
                want_off = _want_offsets(A, grid)
                got_off = _offsets_array(getattr(lib, f"colsOffsetsPartitioningUnifRanges_{off}"),
                                         h, grid, A.M)
                np.testing.assert_array_equal(got_off, want_off, err_msg=f"{name} {grid}")
                want = _want_parts(A, grid, off)
                _same_parts(_parts(getattr(lib, f"colsPartitioningUnifRanges_{off}")(h.ptr, grid),
                                   grid), want)
                po = ctypes.c_void_p()
                p = getattr(lib, f"colsPartitioningUnifRangesOffsetsAux_{off}")(
                    h.ptr, grid, ctypes.byref(po))
                assert p and po.value
                aux_off = np.ctypeslib.as_array(ctypes.cast(po, ctypes.POINTER(idx_t)),
                                                shape=(A.M * grid + 1,)).astype(np.int64)
                ctypes.CDLL(None).free(po)
                np.testing.assert_array_equal(aux_off, want_off)
                _same_parts(_parts(p, grid), want)
                if ref is None:
                    continue
                ro = _offsets_array(getattr(ref, f"colsOffsetsPartitioningUnifRanges_{off}"),
                                    h, grid, A.M)
                np.testing.assert_array_equal(ro, got_off)
                # The reference fails on a range without entries; compare the
                # partitions where every range has some.
                if all(w[2] > 0 for w in want):
                    rp = getattr(ref, f"colsPartitioningUnifRanges_{off}")(h.ptr, grid)
                    _same_parts(_parts(rp, grid), want)


def test_column_partition_errors():
    lib = capi.load()
    A = pb.random_sparse(5, 9, 0.3, seed=3)
    h = HostSpMat(A, 0)
    assert not lib.colsOffsetsPartitioningUnifRanges_0(h.ptr, 0)
    assert not lib.colsPartitioningUnifRanges_0(h.ptr, 0)
    assert not lib.colsPartitioningUnifRanges_0(None, 2)
    # A range with no entries: NULL arrays, zero counts (the reference fails).
    E = pb.CSR(np.zeros(4, np.int64), np.zeros(0, np.int64), np.zeros(0), (3, 6))
    parts = _parts(lib.colsPartitioningUnifRanges_1(HostSpMat(E, 1).ptr, 2), 2)
    assert [p[:3] for p in parts] == [(3, 3, 0), (3, 3, 0)]
