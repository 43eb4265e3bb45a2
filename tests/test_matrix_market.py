"""MatrixMarket reading and writing (MMtoCSR, sp3mm_write_mm, sp3mm_spmat_sort_rows).

The reader replaces the reference's loader (code/src/lib/parser.c:126-330),
which its test driver uses to load R, AC and P (code/test/Sp3MM_test.c:228-247).
Files here are generated from the committed golden matrices; where the built
reference (oracle/_ref) is present, our reader is compared with the
reference's own MMtoCSR on the same files, array for array.  Host code only:
no GPU is used.
"""
import ctypes
import os

import numpy as np
import pytest

import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import capi
from sp3mm4amg_b200.problems import CSR
from sp3mm4amg_b200.spmat import SPMAT_P

from conftest import REF_TEST_DIR


def _spmat_arrays(p):
    m = ctypes.cast(p, SPMAT_P).contents
    M, N, NZ = int(m.M), int(m.N), int(m.NZ)
    irp = np.ctypeslib.as_array(m.IRP, shape=(M + 1,)).copy()
    ja = np.ctypeslib.as_array(m.JA, shape=(NZ,)).copy() if NZ else np.zeros(0, np.uint64)
    as_ = np.ctypeslib.as_array(m.AS, shape=(NZ,)).copy() if NZ else np.zeros(0)
    return M, N, NZ, irp, ja, as_


def _ours(path):
    lib = capi.load()
    p = lib.MMtoCSR(os.fsencode(path))
    if not p:
        return None
    try:
        return _spmat_arrays(p)
    finally:
        S._free_spmat(p)


@pytest.fixture(scope="module")
def ref_reader():
    """The reference's MMtoCSR from the built reference library, if present."""
    import oracle
    if not os.path.exists(oracle.REF_SO):
        pytest.skip("reference library not built")
    lib = ctypes.CDLL(oracle.REF_SO)
    lib.MMtoCSR.restype = ctypes.c_void_p
    lib.MMtoCSR.argtypes = [ctypes.c_char_p]
    lib.freeSpmat.argtypes = [ctypes.c_void_p]

    def read(path):
        p = lib.MMtoCSR(os.fsencode(path))
        assert p, f"reference MMtoCSR failed on {path}"
        try:
            return _spmat_arrays(p)
        finally:
            lib.freeSpmat(p)
    return read


def _same(a, b):
    assert a[:3] == b[:3]
    assert np.array_equal(a[3], b[3])
    assert np.array_equal(a[4], b[4])
    assert np.array_equal(a[5].view(np.int64), b[5].view(np.int64))


def _entries(csr: CSR, lower=False):
    r = np.repeat(np.arange(csr.M), np.diff(csr.indptr))
    c, v = csr.indices, csr.data
    if lower:
        keep = c <= r
        r, c, v = r[keep], c[keep], v[keep]
    return r, c, v


def _write(path, header, size, items, sep="\n"):
    with open(path, "w", newline="") as f:
        f.write(header + sep)
        f.write(size + sep)
        for it in items:
            f.write(it + sep)


def test_round_trip_golden(golden, tmp_path):
    for name, case in golden.items():
        for k in ("R", "A", "P", "pair"):
            m = case[k]
            path = str(tmp_path / f"{name}_{k}.mtx")
            S.write_mm(m, path)
            back = S.read_mm(path)
            assert back.shape == m.shape
            assert np.array_equal(back.indptr, m.indptr)
            assert np.array_equal(back.indices, m.indices)
            assert np.array_equal(back.data.view(np.int64),
                                  np.asarray(m.data, np.float64).view(np.int64))


def test_reference_fixtures_read_like_the_reference(ref_reader):
    if not os.path.isdir(REF_TEST_DIR):
        pytest.skip("reference tree not present")
    for n in ("r", "ac", "p", "ac_next"):
        path = os.path.join(REF_TEST_DIR, n)
        _same(_ours(path), ref_reader(path))


def test_file_forms_read_like_the_reference(golden, ref_reader, tmp_path):
    A = golden[sorted(golden)[0]]["A"]
    r, c, v = _entries(A, lower=True)
    # Lower triangle in column-major order (the usual symmetric layout), so
    # mirrored entries land out of column order within rows.
    o = np.lexsort((r, c))
    r, c, v = r[o], c[o], v[o]
    nz = len(r)
    items = [f"{i + 1} {j + 1} {x:.17g}" for i, j, x in zip(r, c, v)]
    # Spacing the fscanf-based reader accepts: tabs, a leading '+', an item
    # split across lines, exponent forms.
    items[0] = "\t" + items[0].replace(" ", "\t  ")
    items[1] = items[1].replace(" ", "\n", 1)
    items[2] = "+" + items[2]
    items[3] = f"{r[3] + 1} {c[3] + 1} {v[3]:.17e}"
    size = f"{A.M} {A.N} {nz}"
    cases = {
        "sym.mtx": ("%%MatrixMarket matrix coordinate real symmetric\n% a comment\n%\n",
                    size, items, "\n"),
        "sym_crlf.mtx": ("%%MatrixMarket Matrix Coordinate Real Symmetric\r\n%c\r\n", size,
                         items, "\r\n"),
        "pattern.mtx": ("%%MatrixMarket matrix coordinate pattern general", size,
                        [f"{i + 1} {j + 1}" for i, j in zip(r, c)], "\n"),
        "integer_sym.mtx": ("%%MatrixMarket matrix coordinate integer symmetric", size,
                            [f"{i + 1} {j + 1} {int(k)}" for i, j, k in
                             zip(r, c, np.arange(nz) % 7 - 3)], "\n"),
        "skew.mtx": ("%%MatrixMarket matrix coordinate real skew-symmetric", size,
                     [f"{i + 1} {j + 1} {x:.17g}" for i, j, x in zip(r, c, v) if i != j], "\n"),
    }
    for fname, (hdr, sz, its, sep) in cases.items():
        if fname == "skew.mtx":
            sz = f"{A.M} {A.N} {len(its)}"
        path = str(tmp_path / fname)
        _write(path, hdr.rstrip("\r\n"), "\n" + sz if fname == "pattern.mtx" else sz, its, sep)
        ours, ref = _ours(path), ref_reader(path)
        assert ours is not None, fname
        _same(ours, ref)
    # The symmetric expansion is the full matrix.
    full = S.read_mm(str(tmp_path / "sym.mtx"), sort_rows=True)
    assert np.array_equal(full.indptr, A.indptr)
    assert np.array_equal(full.indices, A.indices)
    assert np.array_equal(full.data, A.data)


def test_sort_rows_is_stable(tmp_path):
    path = str(tmp_path / "dup.mtx")
    _write(path, "%%MatrixMarket matrix coordinate real general", "2 3 5",
           ["1 3 1.0", "1 1 2.0", "1 3 3.0", "2 2 4.0", "1 1 5.0"])
    raw = S.read_mm(path)
    assert list(raw.indices) == [2, 0, 2, 0, 1]
    srt = S.read_mm(path, sort_rows=True)
    assert list(srt.indptr) == [0, 4, 5]
    assert list(srt.indices) == [0, 0, 2, 2, 1]
    assert list(srt.data) == [2.0, 5.0, 1.0, 3.0, 4.0]


@pytest.mark.parametrize("body", [
    ("%%MatrixMarket matrix coordinate real general", "2 2 3", ["1 1 1.0", "2 2 2.0"]),
    ("%%MatrixMarket matrix coordinate real general", "2 2 1", ["1 1 1.0", "2 2 2.0"]),
    ("%%MatrixMarket matrix coordinate real general", "2 2 1", ["0 1 1.0"]),
    ("%%MatrixMarket matrix coordinate real general", "2 2 1", ["3 1 1.0"]),
    ("%%MatrixMarket matrix coordinate real general", "2 2 1", ["1 3 1.0"]),
    ("%%MatrixMarket matrix coordinate real general", "2 2 1", ["1 1 x"]),
    ("%%MatrixMarket matrix coordinate real general", "2 2 2", ["1 1 1.0", "% late", "2 2 1"]),
    ("%%MatrixMarket matrix array real general", "2 2", ["1.0", "2.0", "3.0", "4.0"]),
    ("%%MatrixMarket matrix coordinate complex general", "2 2 1", ["1 1 1.0 0.0"]),
    ("%%MatrixMarket vector coordinate real general", "2 2 1", ["1 1 1.0"]),
    ("%MatrixMarket matrix coordinate real general", "2 2 1", ["1 1 1.0"]),
    ("%%MatrixMarket matrix coordinate real general", "2 x 1", ["1 1 1.0"]),
])
def test_malformed_files_fail(tmp_path, body):
    path = str(tmp_path / "bad.mtx")
    _write(path, *body)
    with pytest.raises(S.Sp3mmError):
        S.read_mm(path)


def test_missing_file_fails(tmp_path):
    with pytest.raises(S.Sp3mmError):
        S.read_mm(str(tmp_path / "absent.mtx"))


def test_write_rejects_invalid_csr(tmp_path):
    bad = CSR(np.array([0, 2, 1]), np.array([0, 1]), np.array([1.0, 2.0]), (2, 2))
    with pytest.raises(S.Sp3mmError):
        S.write_mm(bad, str(tmp_path / "x.mtx"))
    out_of_range = CSR(np.array([0, 1]), np.array([5]), np.array([1.0]), (1, 2))
    with pytest.raises(S.Sp3mmError):
        S.write_mm(out_of_range, str(tmp_path / "y.mtx"))
    assert not os.path.exists(str(tmp_path / "y.mtx"))
