"""The oracle (CPU restatement) pinned against the reference: its bundled
fixture, golden vectors generated by the reference's own code, and -- where
the reference library was built here -- the reference called side by side."""
import os

import numpy as np
import pytest

import oracle as O
from sp3mm4amg_b200 import problems as pb


@pytest.mark.parametrize("off", [0, 1])
def test_oracle_matches_reference_fixture(orc, reference_fixture, off):
    # code/test/{r,ac,p,ac_next}: AC_next is an external (AMG4PSBLAS) result;
    # the reference's own test accepts it at 7e-4 absolute
    # (code/src/include/config.h:147); we require the exact pattern and 1e-12
    # relative.
    R, AC, P, ACN = reference_fixture
    C = orc.sp3mm_pair(R, AC, P, off)
    cmp = O.compare(C, ACN, rtol=1e-12)
    assert cmp["ok"], cmp
    D = orc.sp3mm_direct(R, AC, P, off)
    assert O.compare(D, ACN, rtol=1e-12)["ok"]


def test_oracle_matches_reference_fixture_results(orc, reference_fixture):
    """Bit for bit against the reference library's own results on its fixture
    (stored beside the quadruple by tests/golden/make_golden.py)."""
    from conftest import REF_FIXTURE, _unpack
    z = np.load(REF_FIXTURE)
    R, AC, P, _ = reference_fixture
    for got, key in ((orc.sp3mm_pair(R, AC, P), "ref_pair"),
                     (orc.sp3mm_direct(R, AC, P), "ref_direct")):
        want = _unpack(z, key)
        cmp = O.compare(got, want, rtol=0.0)
        assert cmp["ok"] and cmp["bitwise_equal"] == want.nnz, (key, cmp)


def test_reference_fixture_file_matches_the_tree(reference_fixture):
    """Where the reference tree is present, the committed quadruple equals its
    files (read here with scipy, an independent MatrixMarket reader)."""
    from conftest import REF_TEST_DIR
    if not os.path.isdir(REF_TEST_DIR):
        pytest.skip("reference tree not present")
    for got, n in zip(reference_fixture, ("r", "ac", "p", "ac_next")):
        want = O.load_mm(os.path.join(REF_TEST_DIR, n))
        cmp = O.compare(got, want, rtol=0.0)
        assert cmp["ok"] and cmp["bitwise_equal"] == want.nnz, (n, cmp)


def test_oracle_matches_golden(orc, golden):
    for name, g in golden.items():
        for off in (0, 1):
            C = orc.sp3mm_pair(g["R"], g["A"], g["P"], off)
            cmp = O.compare(C, g["pair"], rtol=0.0)
            assert cmp["ok"] and cmp["bitwise_equal"] == C.nnz, (name, off, cmp)
            D = orc.sp3mm_direct(g["R"], g["A"], g["P"], off)
            cmp = O.compare(D, g["direct"], rtol=0.0)
            assert cmp["ok"] and cmp["bitwise_equal"] == D.nnz, (name, off, cmp)
            np.testing.assert_array_equal(orc.spmm_symb_rowsizes(g["R"], g["A"], off), g["symb_ra"])
            np.testing.assert_array_equal(orc.spmm_ub_rowsizes(g["R"], g["A"], off), g["ub_ra"])


def test_oracle_internal_consistency(orc, golden):
    for name, g in golden.items():
        R, A, P = g["R"], g["A"], g["P"]
        RA = orc.spmm(R, A)
        sizes = orc.spmm_symb_rowsizes(R, A)
        np.testing.assert_array_equal(sizes[:-1], RA.row_lengths())
        assert sizes[-1] == RA.nnz
        ub = orc.spmm_ub_rowsizes(R, A)
        assert np.all(ub[:-1] >= sizes[:-1])
        dsz = orc.sp3mm_direct_symb_rowsizes(R, A, P)
        np.testing.assert_array_equal(dsz[:-1], g["direct"].row_lengths())
        dub = orc.sp3mm_direct_ub_rowsizes(R, A, P)
        assert np.all(dub[:-1] >= dsz[:-1])
        # R*(A*P) has the pair's pattern; values agree to rounding.
        RR = orc.sp3mm_pair_right(R, A, P)
        cmp = O.compare(RR, g["pair"], rtol=1e-12)
        assert cmp["col_idx"] and cmp["max_rel_err"] < 1e-13, (name, cmp)


def test_oracle_vs_scipy(orc):
    prob = pb.stencil_problem(3, 10)
    C = orc.sp3mm_pair(prob.R, prob.A, prob.P)
    S = (prob.R.to_scipy() @ prob.A.to_scipy() @ prob.P.to_scipy()).tocsr()
    S.sort_indices()
    assert np.array_equal(C.indptr, S.indptr)
    assert np.array_equal(C.indices, S.indices)
    assert O.max_rel_err(C.data, S.data) < 1e-13


def test_oracle_empty_and_degenerate(orc):
    Z = pb.CSR(np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0), (0, 5))
    B = pb.random_sparse(5, 4, 0.5, seed=3)
    C = orc.spmm(Z, B)
    assert C.shape == (0, 4) and C.nnz == 0
    E = pb.CSR(np.zeros(4, np.int64), np.zeros(0, np.int64), np.zeros(0), (3, 5))
    C = orc.spmm(E, B)
    assert C.nnz == 0 and np.array_equal(C.indptr, np.zeros(4))


@pytest.mark.skipif(not os.path.exists(O.REF_SO), reason="reference library not built")
@pytest.mark.parametrize("off", [0, 1])
def test_every_reference_pair_function_is_bit_identical(orc, off):
    # The property the restatement relies on: all six pair-wise SpMMs (and
    # both symbolic modes) return the same bits, and the direct product has
    # the same pattern.
    ref = O.Reference()
    prob = pb.config0()
    want = orc.sp3mm_pair(prob.R, prob.A, prob.P, off)
    for mode in (O.RBTREE, O.IDXMAP):
        ref.cfg.symbMMRowImplID = mode
        for i, f in enumerate(O.REF_SPMM_UB + O.REF_SPMM_SYMBNUM):
            ref.adapt_grid(i if i < 4 else i - 4)
            got = ref.sp3mm_pair(f, prob.R, prob.A, prob.P, off)
            cmp = O.compare(got, want, rtol=0.0)
            assert cmp["ok"] and cmp["bitwise_equal"] == want.nnz, (f, mode, cmp)
    d = ref.sp3mm_direct(prob.R, prob.A, prob.P, off)
    cmp = O.compare(d, orc.sp3mm_direct(prob.R, prob.A, prob.P, off), rtol=0.0)
    assert cmp["ok"] and cmp["bitwise_equal"] == d.nnz
    cmp = O.compare(d, want, rtol=1e-12)
    assert cmp["col_idx"] and cmp["max_rel_err"] < 1e-14


def test_comparator_detects_planted_errors(orc, golden):
    # A mistake planted in the oracle's output must be caught.
    g = golden["poisson2d_64_agg2"]
    C = orc.sp3mm_pair(g["R"], g["A"], g["P"])
    bad = pb.CSR(C.indptr.copy(), C.indices.copy(), C.data.copy(), C.shape)
    bad.data[100] *= 1 + 1e-11
    assert not O.compare(bad, g["pair"])["ok"]
    bad = pb.CSR(C.indptr.copy(), C.indices.copy(), C.data.copy(), C.shape)
    bad.indices[5], bad.indices[6] = bad.indices[6], bad.indices[5]
    assert not O.compare(bad, g["pair"])["ok"]
