"""GPU parity: every entry point of libsp3mm_b200.so against the oracle and
the reference's golden vectors.  Pattern (row_ptr, col_idx) bit-exact; values
within RTOL relative -- and in practice bit-identical, which is asserted for
the pair-wise and direct products since the kernels keep the reference's
summation order."""
import numpy as np
import pytest

import oracle as O
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import capi, problems as pb

pytestmark = pytest.mark.gpu

RTOL = 1e-12   # FP64, summation order only

UB_SPMM = capi.SPMM_UB_NAMES
SN_SPMM = capi.SPMM_SYMBNUM_NAMES


def assert_same(got, want, exact=True, rtol=RTOL, what=""):
    cmp = O.compare(got, want, rtol=rtol)
    assert cmp["ok"], (what, cmp)
    if exact:
        assert cmp["bitwise_equal"] == want.nnz, (what, cmp)


@pytest.fixture(scope="module")
def cases(golden):
    out = dict(golden)
    return out


@pytest.mark.parametrize("off", [0, 1])
@pytest.mark.parametrize("name", UB_SPMM + SN_SPMM)
def test_spmm_entry_points_golden(cases, orc, name, off):
    for cname, g in cases.items():
        RA = orc.spmm(g["R"], g["A"])
        got = S.spmm(g["R"], g["A"], name, off_f=off)
        assert_same(got, RA, what=(cname, name, off))
        C = S.spmm(got, g["P"], name, off_f=off)
        assert_same(C, g["pair"], what=(cname, name, off, "second"))


@pytest.mark.parametrize("off", [0, 1])
@pytest.mark.parametrize("spmm", UB_SPMM + SN_SPMM + (None,))
def test_pair_driver_golden(cases, spmm, off):
    for cname, g in cases.items():
        C = S.sp3mm(g["R"], g["A"], g["P"], "sp3mmRowByRowPair_", spmm=spmm, off_f=off)
        assert_same(C, g["pair"], what=(cname, spmm, off))
        C = S.sp3mm(g["R"], g["A"], g["P"], "sp3mmRowByRowPair_SymbNum_", spmm=spmm, off_f=off)
        assert_same(C, g["pair"], what=(cname, spmm, off, "symbnum driver"))


@pytest.mark.parametrize("off", [0, 1])
@pytest.mark.parametrize("name", ["sp3mmRowByRowMerged_", "sp3mmRowByRowMerged_SymbNum_"])
def test_direct_golden(cases, name, off):
    for cname, g in cases.items():
        C = S.sp3mm(g["R"], g["A"], g["P"], name, off_f=off)
        assert_same(C, g["direct"], what=(cname, name, off))


@pytest.mark.parametrize("off", [0, 1])
@pytest.mark.parametrize("spmm", [None, "spmmRowByRow_", "spmmRowByRow_SymbNum_"])
def test_pair_right(cases, orc, spmm, off):
    for cname, g in cases.items():
        want = orc.sp3mm_pair_right(g["R"], g["A"], g["P"])
        C = S.sp3mm(g["R"], g["A"], g["P"], "sp3mmRowByRowPairRight_", spmm=spmm, off_f=off)
        assert_same(C, want, what=(cname, spmm, off))
        # Same pattern as (R*A)*P, values to rounding.
        assert_same(C, g["pair"], exact=False, what=(cname, "vs pair"))


@pytest.mark.parametrize("off", [0, 1])
def test_row_sizes(cases, off):
    for cname, g in cases.items():
        np.testing.assert_array_equal(S.symb_rowsizes(g["R"], g["A"], off_f=off), g["symb_ra"])
        np.testing.assert_array_equal(S.ub_rowsizes(g["R"], g["A"], off_f=off), g["ub_ra"])


def _col_offsets(B, grid_cols):
    """B's column-partition offsets (code/src/commons/sparseUtilsGeneric.c:284-311)."""
    n = B.N
    blk, rem = divmod(n, grid_cols)
    starts = [g * blk + min(g, rem) for g in range(grid_cols)]
    off = np.empty(B.M * grid_cols + 1, np.int64)
    for r in range(B.M):
        cols = B.indices[B.indptr[r]:B.indptr[r + 1]]
        for gc in range(grid_cols):
            off[r * grid_cols + gc] = B.indptr[r] + np.searchsorted(cols, starts[gc])
    off[-1] = B.nnz
    return off


@pytest.mark.parametrize("off", [0, 1])
def test_colparts_upper_bound(off):
    A = pb.random_sparse(30, 40, 0.1, seed=21)
    B = pb.random_sparse(40, 50, 0.1, seed=22)
    gc = 3
    offs = _col_offsets(B, gc)
    got = S.ub_colparts_rowsizes(A, B, gc, offs, off_f=off)
    want = np.zeros(A.M * gc + 1, np.int64)
    for r in range(A.M):
        for jj in range(A.indptr[r], A.indptr[r + 1]):
            j = A.indices[jj]
            for g in range(gc):
                want[r * gc + g] += offs[j * gc + g + 1] - offs[j * gc + g]
    want[-1] = want[:-1].sum()
    np.testing.assert_array_equal(got, want)


def _random_triple(seed, n_c=60, n=200, m=300, dens=0.03, empty=0.1):
    R = pb.random_sparse(n_c, n, dens, seed=seed, empty_rows=empty)
    A = pb.random_sparse(n, m, dens, seed=seed + 1, empty_rows=empty)
    P = pb.random_sparse(m, 50, dens * 2, seed=seed + 2, empty_rows=empty)
    return R, A, P


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_rectangular_all_variants(orc, seed):
    R, A, P = _random_triple(seed * 10)
    pair = orc.sp3mm_pair(R, A, P)
    direct = orc.sp3mm_direct(R, A, P)
    with S.Context() as ctx:
        dR, dA, dP = ctx.upload(R), ctx.upload(A), ctx.upload(P)
        for fl in (S.UB, S.SYMBNUM):
            assert_same(ctx.rap(dR, dA, dP, S.PAIR, fl).download(), pair, what=("pair", fl))
            assert_same(ctx.rap(dR, dA, dP, S.DIRECT, fl).download(), direct, what=("dir", fl))
            right = orc.sp3mm_pair_right(R, A, P)
            assert_same(ctx.rap(dR, dA, dP, S.PAIR_RIGHT, fl).download(), right)


@pytest.mark.parametrize("lanes", [4, 8, 16, 32, 512])
def test_results_do_not_depend_on_tuning(golden, orc, lanes):
    # Every lanes-per-row instantiation (512: a CTA per direct row), and
    # table shifts from generous to tiny (d1 = 8 forces nearly every row
    # through the overflow/retry path).
    g = golden["poisson2d_64_agg2"]
    R, A, P = _random_triple(7)
    want_r = (orc.sp3mm_pair(R, A, P), orc.sp3mm_direct(R, A, P))
    with S.Context() as ctx:
        for d1, d2 in ((0, 0), (1, 1), (3, 2), (8, 4)):
            ctx.set_tuning(lanes, d1, d2)
            for (r, a, p), (pair, direct) in (((g["R"], g["A"], g["P"]), (g["pair"], g["direct"])),
                                              ((R, A, P), want_r)):
                dR, dA, dP = ctx.upload(r), ctx.upload(a), ctx.upload(p)
                for fl in (S.UB, S.SYMBNUM):
                    assert_same(ctx.rap(dR, dA, dP, S.PAIR, fl).download(), pair,
                                what=(lanes, d1, d2, fl, "pair"))
                    assert_same(ctx.rap(dR, dA, dP, S.DIRECT, fl).download(), direct,
                                what=(lanes, d1, d2, fl, "direct"))
                for m in (dR, dA, dP):
                    m.free()


def test_fp32_value_storage(golden, orc):
    # FP32 storage, FP64 accumulation: the pattern stays exact, values carry
    # the FP32 rounding of the stored operands and result.
    g = golden["poisson2d_64_agg2"]
    with S.Context() as ctx:
        d64 = [ctx.upload(m) for m in (g["R"], g["A"], g["P"])]
        d32 = [ctx.upload(m, S.F32) for m in (g["R"], g["A"], g["P"])]
        for variant, want in ((S.DIRECT, g["direct"]), (S.PAIR, g["pair"]),
                              (S.PAIR_RIGHT, g["pair"])):
            for fl in (S.UB, S.SYMBNUM):
                # FP64 operands, FP32 result (the finest level of a mixed hierarchy).
                C = ctx.rap(*d64, variant, fl, S.F32).download()
                cmp = O.compare(C, want, rtol=1e-6)
                assert cmp["col_idx"] and cmp["max_rel_err"] < 2 ** -23, (variant, fl, cmp)
                # FP32 operands and result: errors of the FP32 operands,
                # bounded relative to the largest entry (entries that cancel
                # lose relative accuracy).
                scale = np.abs(want.data).max()
                for out in (S.F32, S.F64):
                    C = ctx.rap(*d32, variant, fl, out).download()
                    cmp = O.compare(C, want, rtol=1.0)
                    assert cmp["col_idx"], (variant, fl, out, cmp)
                    assert np.abs(C.data - want.data).max() <= 1e-5 * scale
        with pytest.raises(S.Sp3mmError):
            ctx.rap(d64[0], d32[1], d64[2], S.DIRECT, S.UB)


@pytest.mark.parametrize("flavour", [0, 1])
def test_long_rows_use_large_and_global_tables(orc, flavour):
    # Dense-ish rows push bounds past the shared-memory levels (up to 4096
    # slots) into the global-memory tables.
    A = pb.random_sparse(40, 3000, 0.3, seed=31)
    B = pb.random_sparse(3000, 9000, 0.02, seed=32)
    want = orc.spmm(A, B)
    assert want.row_lengths().max() > 4096
    name = "spmmRowByRow_" if flavour == 0 else "spmmRowByRow_SymbNum_"
    assert_same(S.spmm(A, B, name), want)
    # Mixed: some short, some long rows in one product.
    A2 = pb.random_sparse(300, 3000, 0.01, seed=33)
    A2 = pb.CSR.from_scipy(__import__("scipy.sparse", fromlist=["vstack"]).vstack(
        [A2.to_scipy(), A.to_scipy()]).tocsr())
    assert_same(S.spmm(A2, B, name), orc.spmm(A2, B))


def test_direct_long_rows(orc):
    R = pb.random_sparse(20, 500, 0.2, seed=41)
    A = pb.random_sparse(500, 2000, 0.05, seed=42)
    P = pb.random_sparse(2000, 6000, 0.01, seed=43)
    want = orc.sp3mm_direct(R, A, P)
    for name in ("sp3mmRowByRowMerged_", "sp3mmRowByRowMerged_SymbNum_"):
        assert_same(S.sp3mm(R, A, P, name), want, what=name)


def test_empty_and_degenerate_inputs(orc):
    Z = pb.CSR(np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0), (0, 5))
    B = pb.random_sparse(5, 4, 0.5, seed=3)
    E = pb.CSR(np.zeros(4, np.int64), np.zeros(0, np.int64), np.zeros(0), (3, 5))
    for name in ("spmmRowByRow_", "spmmRowByRow_SymbNum_"):
        C = S.spmm(Z, B, name)
        assert C.shape == (0, 4) and C.nnz == 0
        C = S.spmm(E, B, name)
        assert C.shape == (3, 4) and C.nnz == 0 and np.all(C.indptr == 0)
        E2 = pb.CSR(np.zeros(5, np.int64), np.zeros(0, np.int64), np.zeros(0), (4, 7))
        C = S.spmm(B, E2, name)
        assert C.shape == (5, 7) and C.nnz == 0
    one = pb.CSR(np.array([0, 1]), np.array([0]), np.array([3.0]), (1, 1))
    for name in ("sp3mmRowByRowPair_", "sp3mmRowByRowMerged_", "sp3mmRowByRowMerged_SymbNum_"):
        C = S.sp3mm(one, one, one, name)
        assert C.nnz == 1 and C.data[0] == 27.0


def test_malformed_inputs_return_null():
    good = pb.random_sparse(6, 6, 0.5, seed=4)
    bad_order = pb.CSR(good.indptr.copy(), good.indices.copy(), good.data.copy(), good.shape)
    r = int(np.argmax(good.row_lengths()))
    s = good.indptr[r]
    bad_order.indices[s], bad_order.indices[s + 1] = bad_order.indices[s + 1], bad_order.indices[s]
    bad_col = pb.CSR(good.indptr.copy(), good.indices.copy(), good.data.copy(), good.shape)
    bad_col.indices[-1] = 99
    bad_rp = pb.CSR(good.indptr.copy(), good.indices.copy(), good.data.copy(), good.shape)
    bad_rp.indptr[2], bad_rp.indptr[3] = bad_rp.indptr[3] + 1, bad_rp.indptr[2]
    for bad in (bad_order, bad_col, bad_rp):
        with pytest.raises(S.Sp3mmError):
            S.spmm(bad, good, "spmmRowByRow_")
        with pytest.raises(S.Sp3mmError):
            S.sp3mm(good, bad, good, "sp3mmRowByRowMerged_")
        # Page-locked inputs take the other upload route; same checks.
        with pytest.raises(S.Sp3mmError):
            S.sp3mm(good, bad, good, "sp3mmRowByRowMerged_", pinned=True)
    # Dimension mismatch.
    with pytest.raises(S.Sp3mmError):
        S.spmm(good, pb.random_sparse(7, 3, 0.5, seed=5), "spmmRowByRow_")
    # The library still works after the errors.
    assert S.spmm(good, good, "spmmRowByRow_").shape == (6, 6)


def test_device_roundtrip_and_transpose():
    m = pb.random_sparse(300, 200, 0.05, seed=8, empty_rows=0.2)
    with S.Context() as ctx:
        d = ctx.upload(m)
        back = d.download()
        assert np.array_equal(back.indptr, m.indptr)
        assert np.array_equal(back.indices, m.indices)
        assert np.array_equal(back.data, m.data)
        assert d.max_row == int(m.row_lengths().max())
        t = ctx.transpose(d).download()
        want = m.transpose()
        assert np.array_equal(t.indptr, want.indptr)
        assert np.array_equal(t.indices, want.indices)
        assert np.array_equal(t.data, want.data)


def test_elapsed_internal_set():
    g = pb.config0()
    S.sp3mm(g.R, g.A, g.P, "sp3mmRowByRowMerged_")
    t = S.elapsed_internal()
    assert 0.0 < t < 10.0


def test_reference_fixture_on_gpu(reference_fixture):
    """The reference's bundled quadruple code/test/{r,ac,p,ac_next}: every
    variant within 1e-12 of the external AC_next, and bit for bit equal to the
    reference library's own pair-wise / direct result on the same inputs."""
    from conftest import REF_FIXTURE, _unpack
    R, AC, P, ACN = reference_fixture
    z = np.load(REF_FIXTURE)
    ref_pair, ref_direct = _unpack(z, "ref_pair"), _unpack(z, "ref_direct")
    for off in (0, 1):
        for name, sp, want in (("sp3mmRowByRowPair_", None, ref_pair),
                               ("sp3mmRowByRowMerged_", None, ref_direct),
                               ("sp3mmRowByRowPair_", "spmmRowByRow_SymbNum_", ref_pair),
                               ("sp3mmRowByRowMerged_SymbNum_", None, ref_direct)):
            C = S.sp3mm(R, AC, P, name, spmm=sp, off_f=off)
            assert O.compare(C, ACN, rtol=RTOL)["ok"], (name, sp, off)
            assert_same(C, want, what=f"{name} {sp} off={off}")


@pytest.mark.parametrize("off", [0, 1])
def test_pinned_and_pageable_inputs_agree(golden, off):
    """Inputs in page-locked host memory are copied as they are and narrowed
    on the device; pageable inputs are narrowed by host threads into pinned
    staging.  Both routes give the reference's result bit for bit."""
    g = golden["poisson2d_64_agg2"]
    for name, want in (("sp3mmRowByRowMerged_", g["direct"]), ("sp3mmRowByRowPair_", g["pair"])):
        a = S.sp3mm(g["R"], g["A"], g["P"], name, off_f=off, pinned=True)
        b = S.sp3mm(g["R"], g["A"], g["P"], name, off_f=off, pinned=False)
        assert_same(a, want, what=f"{name} pinned")
        assert_same(b, want, what=f"{name} pageable")


def test_trim_releases_staging_and_transfers_continue(golden):
    # Page-locked staging given back by a destroyed context is cached for the
    # next one; trim frees it (and the context's own) and later transfers
    # allocate staging again, with the same results.
    A = golden[sorted(golden)[0]]["A"]
    with S.Context() as first:
        d = first.upload(A)
        d.download()
        d.free()
    with S.Context() as ctx:
        for _ in range(2):
            ctx.trim()
            d = ctx.upload(A)
            got = d.download()
            d.free()
            assert np.array_equal(got.indptr, A.indptr)
            assert np.array_equal(got.indices, A.indices)
            assert np.array_equal(np.asarray(got.data).view(np.int64),
                                  np.asarray(A.data, np.float64).view(np.int64))
