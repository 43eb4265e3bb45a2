"""The CTA-per-row direct kernel (rowdense.cuh): column ranges split across a
CTA's warps, dense shared-memory accumulators, first-touch order rebuilt by
sorting flat product positions.  Its results must be bit-identical to the
reference's direct product (the oracle) and to the warp-per-row kernels, in
every flavour and value type, including rows it cannot hold (an R*A row of
more than 4096 columns, or a C row spanning more than 8192 columns), which go
to the retry launch, and in both of its configurations (rows that outgrow
the smaller one run again on the default one)."""
import numpy as np
import pytest

import oracle as O
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import problems as pb

pytestmark = pytest.mark.gpu

DENSE = 512


def _same(got, want, what):
    cmp = O.compare(got, want, rtol=1e-12)
    assert cmp["ok"], (what, cmp)
    assert cmp["bitwise_equal"] == want.nnz, (what, cmp)


def _direct_all_ways(ctx, orc, R, A, P, what, vt=S.F64):
    want = orc.sp3mm_direct(R, A, P)
    d = [ctx.upload(m, val_type=vt) for m in (R, A, P)]
    got = {}
    for lanes in (0, 32, DENSE):
        ctx.set_tuning(lanes, -1, -1)
        for fl in (S.UB, S.SYMBNUM):
            C = ctx.rap(*d, S.DIRECT, fl)
            got[(lanes, fl)] = C.download()
            C.free()
    ctx.set_tuning(0, -1, -1)
    for m in d:
        m.free()
    if vt == S.F64:
        for k, c in got.items():
            _same(c, want, (what, k))
    base = got[(32, S.UB)]
    for k, c in got.items():
        assert np.array_equal(c.indptr, base.indptr), (what, k)
        assert np.array_equal(c.indices, base.indices), (what, k)
        assert np.array_equal(np.asarray(c.data).view(np.int64),
                              np.asarray(base.data).view(np.int64)), (what, k)


def test_golden_and_random(golden, orc):
    with S.Context() as ctx:
        for name, g in golden.items():
            _direct_all_ways(ctx, orc, g["R"], g["A"], g["P"], name)
        for seed in (3, 4):
            R = pb.random_sparse(40, 300, 0.2, seed=seed, empty_rows=0.1)
            A = pb.random_sparse(300, 900, 0.05, seed=seed + 1, empty_rows=0.1)
            P = pb.random_sparse(900, 120, 0.06, seed=seed + 2, empty_rows=0.1)
            _direct_all_ways(ctx, orc, R, A, P, ("random", seed))


def test_coarse_level_of_a_hierarchy(orc):
    # The second level of a 32^3 hierarchy: 512 rows whose R*A rows have
    # about 2,000 of 4,096 columns -- the case the kernel is for.
    dims = (32, 32, 32)
    A0 = pb.poisson3d(*dims)
    with S.Context() as ctx:
        dA0 = ctx.upload(A0)
        h = ctx.hierarchy(dA0, dims, min_coarse=64)
        A1, P1, R1 = h.level(1)
        R, A, P = R1.download(), A1.download(), P1.download()
        h.free()
        dA0.free()
        _direct_all_ways(ctx, orc, R, A, P, "level1")
        _direct_all_ways(ctx, orc, R, A, P, "level1 f32", vt=S.F32)


def test_rows_beyond_the_slice_are_retried(orc):
    rng = np.random.default_rng(5)
    # Wide: R*A rows with more than 4096 distinct columns.
    R = pb.random_sparse(6, 400, 0.9, seed=11)
    A = pb.random_sparse(400, 20000, 0.02, seed=12)
    P = pb.random_sparse(20000, 64, 0.05, seed=13)
    # R*A rows spanning several 8192-column slices but holding fewer than
    # 4096 columns: the slices are walked one after another.
    Rm = pb.random_sparse(6, 400, 0.5, seed=16)
    Am = pb.random_sparse(400, 30000, 0.0005, seed=17)
    Pm_ = pb.random_sparse(30000, 64, 0.05, seed=18)
    with S.Context() as ctx:
        _direct_all_ways(ctx, orc, R, A, P, "wide R*A")
        _direct_all_ways(ctx, orc, Rm, Am, Pm_, "multi-slice R*A")
    # Far apart: C rows spanning more than 8192 columns (and R*A spans of
    # several slices).
    n = 3000
    cols = np.stack([rng.integers(0, 50, n), rng.integers(20000, 20050, n)], 1)
    import scipy.sparse as sp
    Pm = sp.csr_matrix((rng.uniform(0.5, 1.5, 2 * n), cols.ravel(),
                        np.arange(0, 2 * n + 1, 2)), shape=(n, 20050))
    Pm.sort_indices()
    P2 = pb.CSR(Pm.indptr, Pm.indices, Pm.data, Pm.shape)
    A2 = pb.random_sparse(n, n, 0.01, seed=14)
    R2 = pb.random_sparse(20, n, 0.3, seed=15)
    with S.Context() as ctx:
        _direct_all_ways(ctx, orc, R2, A2, P2, "wide C span")


def test_rows_with_more_products_than_columns_run_one_cta_per_row(orc):
    # The coarsest levels' shape (93^3 level 3: 216 rows, 270k products and
    # all 1,728 columns each): every R*A row has more products than A has
    # columns.  Such rows are binned by their bound (here 2,000 columns, a
    # table of 4,096 slots), not the bound shifted right, so the default
    # routing sends them to the CTA-per-row kernel.
    R = pb.random_sparse(20, 2000, 0.3, seed=21)
    A = pb.random_sparse(2000, 2000, 0.1, seed=22)
    P = pb.random_sparse(2000, 60, 0.1, seed=23)
    want = orc.sp3mm_direct(R, A, P)
    with S.Context() as ctx:
        d = [ctx.upload(m) for m in (R, A, P)]
        for fl in (S.UB, S.SYMBNUM):
            ctx.set_profiling(True)
            C = ctx.rap(*d, S.DIRECT, fl)
            got = C.download()
            prof = ctx.profile()
            ctx.set_profiling(False)
            C.free()
            _same(got, want, ("dense rows", fl))
            assert any(k.startswith("direct.dense") for k in prof), prof
        for m in d:
            m.free()


def test_wide_operands_run_the_small_configuration_then_the_default(orc):
    # A with 20,000 columns: heavy rows run first on the configuration with
    # half the slice and list (two CTAs per SM); rows whose R*A row holds
    # more than its 2,048 columns (rows 0-3: about 2,950) run again on the
    # default configuration, the others (rows 4-7: about 790) stay.
    rng = np.random.default_rng(31)
    import scipy.sparse as sp
    rows = [np.sort(rng.choice(3000, 80 if i < 4 else 20, replace=False)) for i in range(8)]
    Rm = sp.csr_matrix((rng.uniform(0.5, 1.5, sum(len(r) for r in rows)),
                        np.concatenate(rows), np.cumsum([0] + [len(r) for r in rows])),
                       shape=(8, 3000))
    R = pb.CSR(Rm.indptr, Rm.indices, Rm.data, Rm.shape)
    A = pb.random_sparse(3000, 20000, 0.002, seed=32)
    P = pb.random_sparse(20000, 64, 0.05, seed=33)
    with S.Context() as ctx:
        _direct_all_ways(ctx, orc, R, A, P, "small then default")
        want = orc.sp3mm_direct(R, A, P)
        d = [ctx.upload(m) for m in (R, A, P)]
        ctx.set_tuning(DENSE, -1, -1)
        for fl in (S.UB, S.SYMBNUM):
            ctx.set_profiling(True)
            C = ctx.rap(*d, S.DIRECT, fl)
            got = C.download()
            prof = ctx.profile()
            ctx.set_profiling(False)
            C.free()
            _same(got, want, ("small then default", fl))
            assert any(k.startswith("direct.dense2") for k in prof), prof
            assert any(k.startswith("direct.dense.") for k in prof), prof
        ctx.set_tuning(0, -1, -1)
        for m in d:
            m.free()
