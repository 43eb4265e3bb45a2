"""The C-ABI library loads and exports every symbol include/*.h declares;
host-side logic (struct layouts, conversions, generators).  No GPU calls."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from sp3mm4amg_b200 import capi, problems as pb
from sp3mm4amg_b200.spmat import CONFIG, HostSpMat, csr_from_spmat, spmat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    """Names declared with SP3MM_API in include/*.h."""
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = "\n".join(ln for ln in open(h).read().splitlines()
                         if not ln.lstrip().startswith("#"))
        for decl in re.findall(r"SP3MM_API\s+([^;]+);", text, flags=re.S):
            decl = " ".join(decl.split())
            if decl.startswith("extern double"):
                names.update(n.strip() for n in decl[len("extern double"):].split(","))
            elif decl.startswith(("SP3MM ", "SPMM ")):
                names.update(n.strip() for n in decl.split(" ", 1)[1].split(","))
            else:
                m = re.search(r"(\w+)\s*\(", decl)
                assert m, decl
                names.add(m.group(1))
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_library_loads_and_exports_declared_symbols():
    lib = capi.load()
    decl = declared_symbols()
    # 2 x (5 UB + 4 SymbNum SpMMs, 5 triple products, 3 size functions),
    # the device-layer functions, 3 MatrixMarket and 6 column-partition host
    # functions, 4 timing globals.
    assert len(decl) == 34 + len(capi.DEVICE_API) + 3 + 6 + 4 == 96
    exported = exported_symbols(capi.LIB_PATH)
    missing = sorted(decl - exported)
    assert not missing, missing
    for name in decl:
        assert hasattr(lib, name) or name in exported
    # The Python binding covers the same set.
    assert set(capi.all_symbols()) == decl


def test_library_exports_nothing_undeclared():
    exported = exported_symbols(capi.LIB_PATH)
    ours = {s for s in exported if not s.startswith("_")}
    assert ours <= declared_symbols()


def test_library_targets_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", capi.LIB_PATH], capture_output=True,
                         text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_struct_layouts():
    # code/src/include/sparseMatrix.h:41-53 and config.h:42-49.
    assert ctypes.sizeof(spmat) == 56
    assert [f[0] for f in spmat._fields_] == ["NZ", "M", "N", "AS", "JA", "IRP", "MAX_ROW_NZ"]
    assert ctypes.sizeof(CONFIG) == 24
    assert CONFIG.chunkDistrbFunc.offset == 16
    assert ctypes.sizeof(capi.sp3mm_dcsr) == 48


def test_host_spmat_roundtrip():
    m = pb.random_sparse(17, 23, 0.2, seed=5, empty_rows=0.2)
    for off in (0, 1):
        h = HostSpMat(m, off)
        assert h.irp[0] == off and h.struct.NZ == m.nnz
        back = csr_from_spmat(ctypes.pointer(h.struct), off)
        assert np.array_equal(back.indptr, m.indptr)
        assert np.array_equal(back.indices, m.indices)
        assert np.array_equal(back.data, m.data)


def test_generator_sizes():
    p = pb.config0()
    assert (p.A.nnz, p.P.nnz, p.R.nnz) == (20224, 12032, 12032)
    assert p.R.shape == (1024, 4096) and p.P.shape == (4096, 1024)
    # Ordered CSR: strictly ascending columns per row.
    for m in (p.A, p.P, p.R):
        d = np.diff(m.indices)
        starts = m.indptr[1:-1]
        ok = np.ones(d.shape, bool)
        ok[starts[(starts > 0) & (starts < m.nnz)] - 1] = True
        inner = np.ones(m.nnz, bool)
        inner[m.indptr[:-1][m.indptr[:-1] < m.nnz]] = False
        assert np.all(d[inner[1:]] > 0)


def test_compulsory_bytes_config1_formula():
    # bytes(X) = (rows+1)*s_idx + nnz*(s_idx+8), summed over R, A, P and C.
    p = pb.stencil_problem(3, 8)
    c_nnz = 1192
    b8 = p.compulsory_bytes(nnz_c=c_nnz, idx_bytes=8)
    want = sum((m.M + 1) * 8 + m.nnz * 16 for m in (p.R, p.A, p.P)) + 65 * 8 + c_nnz * 16
    assert b8 == want


def test_oracle_not_imported_by_product():
    # The product package never imports the oracle.
    for path in glob.glob(os.path.join(ROOT, "sp3mm4amg_b200", "**", "*.py"), recursive=True):
        text = open(path).read()
        assert "import oracle" not in text and "from oracle" not in text, path
