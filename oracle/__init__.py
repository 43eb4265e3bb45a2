"""Parity oracle for the Sp3MM triple product -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product library never calls it.

Two CPU implementations are exposed with one interface:

* :class:`Oracle` -- ``lib/liboracle_sp3mm.so``, the C restatement in
  ``sp3mm_oracle.c`` of the reference's arithmetic (each function there cites
  the reference file:line it follows);
* :class:`Reference` -- ``_ref/libsp3mm_ref.so``, the reference's own
  unmodified sources compiled in place by ``make -C oracle ref``.  It exists
  only where the reference tree was present at build time.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from sp3mm4amg_b200.problems import CSR
from sp3mm4amg_b200.spmat import (CONFIG, CONFIG_P, SPMAT_P, SPMM_INTERF, HostSpMat,
                                  array_from_idx_ptr, csr_from_spmat, idx_t, RBTREE, IDXMAP)

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "liboracle_sp3mm.so")
REF_SO = os.path.join(HERE, "_ref", "libsp3mm_ref.so")
# Root of the reference project's tree, read only by this test
# infrastructure (building _ref, regenerating the golden fixtures): the
# SP3MM_REFERENCE_ROOT environment variable, else the read-only checkout the
# project is developed beside.  Where neither exists, the tests that need the
# tree itself skip and the committed fixtures under tests/golden stand in.
REF_ROOT = os.environ.get("SP3MM_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "code", "src")
REF_TEST_DIR = os.path.join(REF_ROOT, "code", "test")


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference library when its tree exists)."""
    targets = ["all"]
    if ref and os.path.isdir(REF_SRC):
        targets += ["ref", f"REF_SRC={REF_SRC}"]
    subprocess.run(["make", "-s", "-C", HERE, *targets], check=True)


def max_rel_err(x: np.ndarray, y: np.ndarray) -> float:
    """max |x-y| / |y| over entries (|x-y| where y == 0)."""
    if x.size == 0:
        return 0.0
    d = np.abs(x - y)
    den = np.abs(y)
    rel = np.where(den > 0, d / np.where(den > 0, den, 1.0), d)
    return float(rel.max())


def compare(got: CSR, want: CSR, rtol: float = 1e-12) -> dict:
    """Strict comparator: shape, row_ptr and col_idx bit-exact; values within
    rtol relative (absolute where the expected entry is exactly zero)."""
    out = {"shape": got.shape == want.shape, "nnz": got.nnz == want.nnz}
    out["row_ptr"] = out["shape"] and np.array_equal(got.indptr, want.indptr)
    out["col_idx"] = out["row_ptr"] and np.array_equal(got.indices, want.indices)
    if out["col_idx"]:
        out["max_rel_err"] = max_rel_err(got.data, want.data)
        out["bitwise_equal"] = int(np.sum(got.data.view(np.uint64) == want.data.view(np.uint64)))
        out["values"] = out["max_rel_err"] <= rtol
    else:
        out["max_rel_err"] = float("inf")
        out["bitwise_equal"] = 0
        out["values"] = False
    out["ok"] = all(out[k] for k in ("shape", "nnz", "row_ptr", "col_idx", "values"))
    return out


class Oracle:
    """ctypes driver of the C restatement."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        lib = ctypes.CDLL(path)
        self.lib = lib
        for name in ("orc_spmm", "orc_sp3mm_pair", "orc_sp3mm_pair_right", "orc_sp3mm_direct"):
            getattr(lib, name).restype = ctypes.c_void_p
        lib.orc_spmm.argtypes = [SPMAT_P, SPMAT_P, ctypes.c_int]
        for name in ("orc_sp3mm_pair", "orc_sp3mm_pair_right", "orc_sp3mm_direct"):
            getattr(lib, name).argtypes = [SPMAT_P, SPMAT_P, SPMAT_P, ctypes.c_int]
        for name in ("orc_spmm_ub_rowsizes", "orc_spmm_symb_rowsizes"):
            getattr(lib, name).restype = ctypes.c_void_p
            getattr(lib, name).argtypes = [SPMAT_P, SPMAT_P, ctypes.c_int]
        for name in ("orc_sp3mm_direct_ub_rowsizes", "orc_sp3mm_direct_symb_rowsizes"):
            getattr(lib, name).restype = ctypes.c_void_p
            getattr(lib, name).argtypes = [SPMAT_P, SPMAT_P, SPMAT_P, ctypes.c_int]
        lib.orc_free.argtypes = [ctypes.c_void_p]
        lib.orc_set_threads.argtypes = [ctypes.c_int]
        lib.orc_get_threads.restype = ctypes.c_int
        self.libc = ctypes.CDLL(None)
        self.libc.free.argtypes = [ctypes.c_void_p]

    def set_threads(self, n: int) -> None:
        self.lib.orc_set_threads(int(n))

    def threads(self) -> int:
        return int(self.lib.orc_get_threads())

    def _mat(self, p, off):
        if not p:
            raise RuntimeError("oracle returned NULL")
        out = csr_from_spmat(p, off)
        self.lib.orc_free(p)
        return out

    def _sizes(self, p, m):
        if not p:
            raise RuntimeError("oracle returned NULL")
        out = array_from_idx_ptr(p, m + 1)
        self.libc.free(p)
        return out

    def spmm(self, A: CSR, B: CSR, off: int = 0) -> CSR:
        a, b = HostSpMat(A, off), HostSpMat(B, off)
        return self._mat(self.lib.orc_spmm(a.ptr, b.ptr, off), off)

    def sp3mm_pair(self, R, A, P, off: int = 0) -> CSR:
        r, a, p = HostSpMat(R, off), HostSpMat(A, off), HostSpMat(P, off)
        return self._mat(self.lib.orc_sp3mm_pair(r.ptr, a.ptr, p.ptr, off), off)

    def sp3mm_pair_right(self, R, A, P, off: int = 0) -> CSR:
        r, a, p = HostSpMat(R, off), HostSpMat(A, off), HostSpMat(P, off)
        return self._mat(self.lib.orc_sp3mm_pair_right(r.ptr, a.ptr, p.ptr, off), off)

    def sp3mm_direct(self, R, A, P, off: int = 0) -> CSR:
        r, a, p = HostSpMat(R, off), HostSpMat(A, off), HostSpMat(P, off)
        return self._mat(self.lib.orc_sp3mm_direct(r.ptr, a.ptr, p.ptr, off), off)

    def spmm_ub_rowsizes(self, A, B, off: int = 0) -> np.ndarray:
        a, b = HostSpMat(A, off), HostSpMat(B, off)
        return self._sizes(self.lib.orc_spmm_ub_rowsizes(a.ptr, b.ptr, off), A.M)

    def spmm_symb_rowsizes(self, A, B, off: int = 0) -> np.ndarray:
        a, b = HostSpMat(A, off), HostSpMat(B, off)
        return self._sizes(self.lib.orc_spmm_symb_rowsizes(a.ptr, b.ptr, off), A.M)

    def sp3mm_direct_ub_rowsizes(self, R, A, P, off: int = 0) -> np.ndarray:
        r, a, p = HostSpMat(R, off), HostSpMat(A, off), HostSpMat(P, off)
        return self._sizes(self.lib.orc_sp3mm_direct_ub_rowsizes(r.ptr, a.ptr, p.ptr, off), R.M)

    def sp3mm_direct_symb_rowsizes(self, R, A, P, off: int = 0) -> np.ndarray:
        r, a, p = HostSpMat(R, off), HostSpMat(A, off), HostSpMat(P, off)
        return self._sizes(self.lib.orc_sp3mm_direct_symb_rowsizes(r.ptr, a.ptr, p.ptr, off), R.M)


# Reference SpMM entry points by table order (code/src/include/
# Sp3MM_CSR_OMP_UB_Generic.h:86-92 and Sp3MM_CSR_OMP_Num_Generic.h:86-91).
REF_SPMM_UB = ("spmmRowByRow_", "spmmRowByRow1DBlocks_", "spmmRowByRow2DBlocks_",
               "spmmRowByRow2DBlocksAllocated_")
REF_SPMM_SYMBNUM = ("spmmRowByRow_SymbNum_", "spmmRowByRow1DBlocks_SymbNum_")


class Reference:
    """ctypes driver of the reference's own code (oracle/_ref)."""

    def __init__(self, path: str = REF_SO, threads: int = 0):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = ctypes.CDLL(path)
        self.lib = lib
        for off in (0, 1):
            for n in REF_SPMM_UB + REF_SPMM_SYMBNUM + ("spmmSerial_",):
                f = getattr(lib, f"{n}{off}")
                f.restype = ctypes.c_void_p
                f.argtypes = [SPMAT_P, SPMAT_P, CONFIG_P]
            for n in ("sp3mmRowByRowPair_", "sp3mmRowByRowMerged_"):
                f = getattr(lib, f"{n}{off}")
                f.restype = ctypes.c_void_p
                f.argtypes = [SPMAT_P, SPMAT_P, SPMAT_P, CONFIG_P, ctypes.c_void_p]
            for n in ("spMMSizeUpperbound_",):
                f = getattr(lib, f"{n}{off}")
                f.restype = ctypes.c_void_p
                f.argtypes = [SPMAT_P, SPMAT_P]
            f = getattr(lib, f"SpMM_Symb___{off}")
            f.restype = ctypes.c_void_p
            f.argtypes = [ctypes.c_int, SPMAT_P, SPMAT_P]
        lib.freeSpmat.argtypes = [ctypes.c_void_p]
        lib.refshim_chunks_noop.restype = ctypes.c_void_p
        lib.refshim_chunks_fair_folded.restype = ctypes.c_void_p
        lib.refshim_runtime_sched_kind.restype = ctypes.c_int
        lib.refshim_set_threads.argtypes = [ctypes.c_int]
        lib.refshim_max_threads.restype = ctypes.c_int
        lib.refshim_elapsed_internal.restype = ctypes.c_double
        lib.MPI_Dims_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        self.libc = ctypes.CDLL(None)
        self.libc.free.argtypes = [ctypes.c_void_p]
        if threads:
            lib.refshim_set_threads(int(threads))
        self.cfg = CONFIG(gridRows=20, gridCols=2, symbMMRowImplID=RBTREE)
        self.cfg.threadNum = lib.refshim_max_threads()
        # As the reference test driver: dynamic-like schedules get the fair
        # folded chunk division, static gets a no-op (Sp3MM_test.c:296-308).
        kind = lib.refshim_runtime_sched_kind() & 0x7FFFFFFF
        self.cfg.chunkDistrbFunc = (lib.refshim_chunks_noop() if kind == 1
                                    else lib.refshim_chunks_fair_folded())

    def threads(self) -> int:
        return int(self.cfg.threadNum)

    def adapt_grid(self, table_index: int) -> None:
        """The test driver's per-implementation grid (Sp3MM_test.c:172-205)."""
        if table_index == 1:
            self.cfg.gridRows = self.cfg.threadNum * 2
        elif table_index in (2, 3):
            dims = (ctypes.c_int * 2)(0, 0)
            self.lib.MPI_Dims_create(int(self.cfg.threadNum), 2, dims)
            if dims[1] == 1:
                dims = (ctypes.c_int * 2)(0, 0)
                self.lib.MPI_Dims_create(int(self.cfg.threadNum) + 1, 2, dims)
            self.cfg.gridRows, self.cfg.gridCols = dims[0], dims[1]

    def _mat(self, p, off):
        if not p:
            raise RuntimeError("reference returned NULL")
        out = csr_from_spmat(p, off)
        self.lib.freeSpmat(p)
        return out

    def spmm(self, name: str, A: CSR, B: CSR, off: int = 0) -> CSR:
        a, b = HostSpMat(A, off), HostSpMat(B, off)
        f = getattr(self.lib, f"{name}{off}")
        return self._mat(f(a.ptr, b.ptr, ctypes.byref(self.cfg)), off)

    def sp3mm_pair(self, spmm_name: str, R, A, P, off: int = 0) -> CSR:
        r, a, p = HostSpMat(R, off), HostSpMat(A, off), HostSpMat(P, off)
        fp = ctypes.cast(getattr(self.lib, f"{spmm_name}{off}"), ctypes.c_void_p).value
        f = getattr(self.lib, f"sp3mmRowByRowPair_{off}")
        return self._mat(f(r.ptr, a.ptr, p.ptr, ctypes.byref(self.cfg), fp), off)

    def sp3mm_direct(self, R, A, P, off: int = 0) -> CSR:
        r, a, p = HostSpMat(R, off), HostSpMat(A, off), HostSpMat(P, off)
        f = getattr(self.lib, f"sp3mmRowByRowMerged_{off}")
        return self._mat(f(r.ptr, a.ptr, p.ptr, ctypes.byref(self.cfg), None), off)

    def spmm_ub_rowsizes(self, A, B, off: int = 0) -> np.ndarray:
        a, b = HostSpMat(A, off), HostSpMat(B, off)
        p = getattr(self.lib, f"spMMSizeUpperbound_{off}")(a.ptr, b.ptr)
        out = array_from_idx_ptr(p, A.M + 1)
        self.libc.free(p)
        return out

    def spmm_symb_rowsizes(self, A, B, off: int = 0, mode: int = RBTREE) -> np.ndarray:
        a, b = HostSpMat(A, off), HostSpMat(B, off)
        p = getattr(self.lib, f"SpMM_Symb___{off}")(mode, a.ptr, b.ptr)
        out = array_from_idx_ptr(p, A.M + 1)
        self.libc.free(p)
        return out

    def elapsed_internal(self) -> float:
        return float(self.lib.refshim_elapsed_internal())


def load_mm(path: str) -> CSR:
    """Read a MatrixMarket coordinate file (the reference's fixture format)."""
    import scipy.io
    return CSR.from_scipy(scipy.io.mmread(path).tocsr())
