"""ctypes mirrors of the reference's ABI structs and host CSR conversions.

``spmat`` has the layout of the reference's CSR struct
(code/src/include/sparseMatrix.h:41-53, built without ROWLENS):
``{idx_t NZ, M, N; double* AS; idx_t* JA; idx_t* IRP; idx_t MAX_ROW_NZ}``
with ``idx_t = unsigned long`` (code/src/include/config.h:51).

``CONFIG`` has the layout of code/src/include/config.h:42-49.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .problems import CSR

idx_t = ctypes.c_uint64

RBTREE = 0
IDXMAP = 1


class spmat(ctypes.Structure):
    _fields_ = [
        ("NZ", idx_t),
        ("M", idx_t),
        ("N", idx_t),
        ("AS", ctypes.POINTER(ctypes.c_double)),
        ("JA", ctypes.POINTER(idx_t)),
        ("IRP", ctypes.POINTER(idx_t)),
        ("MAX_ROW_NZ", idx_t),
    ]


class CONFIG(ctypes.Structure):
    _fields_ = [
        ("gridRows", ctypes.c_ushort),
        ("gridCols", ctypes.c_ushort),
        ("symbMMRowImplID", ctypes.c_int),
        ("threadNum", ctypes.c_uint),
        ("chunkDistrbFunc", ctypes.c_void_p),
    ]


SPMAT_P = ctypes.POINTER(spmat)
CONFIG_P = ctypes.POINTER(CONFIG)
# SPMM_INTERF: spmat* (*)(spmat*, spmat*, CONFIG*)
SPMM_INTERF = ctypes.CFUNCTYPE(ctypes.c_void_p, SPMAT_P, SPMAT_P, CONFIG_P)


class HostSpMat:
    """A borrowed ``spmat`` over numpy arrays (the caller-owned input side).

    ``off_f`` = 1 stores 1-based IRP/JA as a FORTRAN caller passes them
    (code/src/Fortran_C_indexing.md).
    """

    def __init__(self, csr: CSR, off_f: int = 0, pinned: bool = False):
        self.off_f = int(off_f)
        if pinned:
            # Page-locked host arrays (torch's pinned allocator), so that the
            # library's host->device copies run at full PCIe/C2C speed.
            import torch
            def alloc(n, dt):
                return torch.empty(max(n, 1), dtype=dt, pin_memory=True).numpy()[:n]
            self.irp = alloc(csr.M + 1, torch.int64).view(np.uint64)
            self.ja = alloc(csr.nnz, torch.int64).view(np.uint64)
            self.as_ = alloc(csr.nnz, torch.float64)
            self.irp[:] = csr.indptr.astype(np.uint64) + np.uint64(off_f)
            self.ja[:] = csr.indices.astype(np.uint64) + np.uint64(off_f)
            self.as_[:] = csr.data
        else:
            self.irp = np.ascontiguousarray(csr.indptr, dtype=np.uint64) + np.uint64(off_f)
            self.ja = np.ascontiguousarray(csr.indices, dtype=np.uint64) + np.uint64(off_f)
            self.as_ = np.ascontiguousarray(csr.data, dtype=np.float64)
        rl = np.diff(csr.indptr)
        self.struct = spmat(
            NZ=csr.nnz, M=csr.M, N=csr.N,
            AS=self.as_.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            JA=self.ja.ctypes.data_as(ctypes.POINTER(idx_t)),
            IRP=self.irp.ctypes.data_as(ctypes.POINTER(idx_t)),
            MAX_ROW_NZ=int(rl.max()) if rl.size else 0,
        )

    @property
    def ptr(self):
        return ctypes.pointer(self.struct)


def csr_from_spmat(p, off_f: int = 0) -> CSR:
    """Copy a returned ``spmat*`` (address or pointer) into a 0-based CSR."""
    if isinstance(p, int):
        p = ctypes.cast(p, SPMAT_P)
    m = p.contents
    M, N, NZ = int(m.M), int(m.N), int(m.NZ)
    irp = np.ctypeslib.as_array(m.IRP, shape=(M + 1,)).astype(np.int64) - off_f
    if NZ:
        ja = np.ctypeslib.as_array(m.JA, shape=(NZ,)).astype(np.int64) - off_f
        as_ = np.ctypeslib.as_array(m.AS, shape=(NZ,)).copy()
    else:
        ja = np.zeros(0, np.int64)
        as_ = np.zeros(0, np.float64)
    return CSR(irp, ja, as_, (M, N))


def array_from_idx_ptr(p, n: int) -> np.ndarray:
    """Copy ``n`` idx_t entries from a returned ``idx_t*``."""
    if isinstance(p, int):
        p = ctypes.cast(p, ctypes.POINTER(idx_t))
    return np.ctypeslib.as_array(p, shape=(n,)).astype(np.int64)
