"""The reference test driver's flow (code/test/Sp3MM_test.c:228-247, 318-419):
load R, AC and P from MatrixMarket files with MMtoCSR, hand the returned
`spmat`s to the drop-in products, and compare with the golden results bit for
bit, 0-based and 1-based (indices shifted in place as C_FortranShiftIdxs
does, code/src/include/sparseUtilsGeneric.h:64-67)."""
import ctypes
import os

import numpy as np
import pytest

import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import capi
from sp3mm4amg_b200.spmat import CONFIG, SPMAT_P, csr_from_spmat

pytestmark = pytest.mark.gpu


def _shift(p, by):
    m = ctypes.cast(p, SPMAT_P).contents
    M, NZ = int(m.M), int(m.NZ)
    irp = np.ctypeslib.as_array(m.IRP, shape=(M + 1,))
    ja = np.ctypeslib.as_array(m.JA, shape=(NZ,))
    irp += np.uint64(by)
    ja += np.uint64(by)


def _bits(x):
    return np.asarray(x, np.float64).view(np.int64)


@pytest.mark.parametrize("off", [0, 1])
def test_products_of_files_read_with_mmtocsr(golden, tmp_path, off):
    lib = capi.load()
    name = sorted(golden)[0]
    case = golden[name]
    ptrs = []
    try:
        for k in ("R", "A", "P"):
            path = str(tmp_path / f"{k}.mtx")
            S.write_mm(case[k], path)
            p = lib.MMtoCSR(os.fsencode(path))
            assert p
            ptrs.append(p)
            if off:
                _shift(p, 1)
        cfg = CONFIG(gridRows=1, gridCols=1, symbMMRowImplID=0, threadNum=1,
                     chunkDistrbFunc=None)
        for fname, want in ((f"sp3mmRowByRowPair_{off}", case["pair"]),
                            (f"sp3mmRowByRowMerged_{off}", case["direct"])):
            out = getattr(lib, fname)(*[ctypes.cast(p, SPMAT_P) for p in ptrs],
                                      ctypes.byref(cfg), None)
            assert out, fname
            try:
                got = csr_from_spmat(out, off)
            finally:
                S._free_spmat(out)
            assert got.shape == want.shape
            assert np.array_equal(got.indptr, want.indptr), fname
            assert np.array_equal(got.indices, want.indices), fname
            assert np.array_equal(_bits(got.data), _bits(want.data)), fname
    finally:
        for p in ptrs:
            S._free_spmat(p)
