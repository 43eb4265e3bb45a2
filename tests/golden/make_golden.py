"""Generate tests/golden/golden_cases.npz from the reference's own code.

Run from the repository root where the reference tree is present:

    make -C oracle all ref
    python tests/golden/make_golden.py

For every case it stores the inputs (R, A, P as 0-based CSR) and the outputs
of the reference library built from the unmodified reference sources
(oracle/_ref/libsp3mm_ref.so):

* ``pair``   -- sp3mmRowByRowPair_0 with spmmRowByRow_SymbNum_0 (every
  reference pair-wise SpMM gives the same bits; the script checks that);
* ``direct`` -- sp3mmRowByRowMerged_0;
* ``symb_ra`` / ``ub_ra`` -- SpMM_Symb___0 (RBTREE) and spMMSizeUpperbound_0
  of R*A.

It also checks that the 1-based (_1) functions on the shifted inputs return
the same matrices shifted by one, and records that check.

It also writes ``reference_fixture.npz``: the reference's only bundled golden
quadruple, ``code/test/{r,ac,p,ac_next}`` (R, AC, P and the externally
computed next-level operator), read with the reference library's own
MatrixMarket loader (MMtoCSR), plus that library's pair-wise and direct
results on it (``ref_pair``, ``ref_direct``).  The GPU box has no reference
tree, so its tests read the quadruple from this file.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from sp3mm4amg_b200 import problems as pb  # noqa: E402


def cases():
    yield "poisson2d_64_agg2", pb.config0()
    yield "poisson3d_8_agg2", pb.stencil_problem(3, 8)
    yield "poisson2d_13x7_agg2", pb.stencil_problem(2, (13, 7))
    # Rectangular random operators with empty rows.
    R = pb.random_sparse(40, 70, 0.08, seed=11, empty_rows=0.2)
    A = pb.random_sparse(70, 90, 0.06, seed=12, empty_rows=0.1)
    P = pb.random_sparse(90, 30, 0.10, seed=13, empty_rows=0.1)
    yield "random_rect_empty_rows", pb.Problem("random_rect_empty_rows", R, A, P)


def pack(prefix, m, out):
    out[f"{prefix}_indptr"] = m.indptr
    out[f"{prefix}_indices"] = m.indices
    out[f"{prefix}_data"] = m.data
    out[f"{prefix}_shape"] = np.array(m.shape, np.int64)


def write_reference_fixture(ref):
    import ctypes
    from sp3mm4amg_b200.spmat import csr_from_spmat
    lib = ctypes.CDLL(O.REF_SO)
    lib.MMtoCSR.restype = ctypes.c_void_p
    lib.MMtoCSR.argtypes = [ctypes.c_char_p]
    lib.freeSpmat.argtypes = [ctypes.c_void_p]
    out, mats = {}, {}
    for n in ("r", "ac", "p", "ac_next"):
        p = lib.MMtoCSR(os.fsencode(os.path.join(O.REF_TEST_DIR, n)))
        assert p, n
        m = csr_from_spmat(p, 0)
        lib.freeSpmat(p)
        # The device CSR contract: strictly ascending columns in every row.
        for i in range(m.M):
            c = m.indices[m.indptr[i]:m.indptr[i + 1]]
            assert np.all(np.diff(c) > 0), (n, i)
        mats[n] = m
        pack(n, m, out)
    R, AC, P = mats["r"], mats["ac"], mats["p"]
    pack("ref_pair", ref.sp3mm_pair("spmmRowByRow_SymbNum_", R, AC, P, 0), out)
    pack("ref_direct", ref.sp3mm_direct(R, AC, P, 0), out)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixture.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main():
    ref = O.Reference()
    write_reference_fixture(ref)
    out = {}
    names = []
    for name, prob in cases():
        names.append(name)
        R, A, P = prob.R, prob.A, prob.P
        pair = None
        for i, f in enumerate(O.REF_SPMM_UB + O.REF_SPMM_SYMBNUM):
            ref.adapt_grid(i if i < 4 else i - 4)
            c = ref.sp3mm_pair(f, R, A, P, 0)
            if pair is None:
                pair = c
            else:
                assert O.compare(c, pair, 0.0)["bitwise_equal"] == pair.nnz, (name, f)
        direct = ref.sp3mm_direct(R, A, P, 0)
        for off in (1,):
            assert O.compare(ref.sp3mm_pair("spmmRowByRow_SymbNum_", R, A, P, off), pair, 0.0)[
                "bitwise_equal"] == pair.nnz
            assert O.compare(ref.sp3mm_direct(R, A, P, off), direct, 0.0)["bitwise_equal"] == \
                direct.nnz
        symb = ref.spmm_symb_rowsizes(R, A, 0)
        ub = ref.spmm_ub_rowsizes(R, A, 0)
        for k, m in (("R", R), ("A", A), ("P", P), ("pair", pair), ("direct", direct)):
            pack(f"{name}__{k}", m, out)
        out[f"{name}__symb_ra"] = symb
        out[f"{name}__ub_ra"] = ub
        print(f"{name}: C {pair.shape} nnz {pair.nnz}; direct max rel diff vs pair "
              f"{O.max_rel_err(direct.data, pair.data):.2e}")
    out["cases"] = np.array(names)
    out["one_based_checked"] = np.array(True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_cases.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
