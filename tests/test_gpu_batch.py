"""Batches (sp3mm_batch_*): many independent products planned together and
executed as one captured graph.  Every result is checked bit for bit
against the oracle (direct R*A*P: sp3mmRowByRowMerged_; SpMM: the
reference's Gustavson SpMM), across tunings, value types, replays with new
values, empty and long-row products."""
import numpy as np
import pytest

import oracle as O
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import problems as pb

pytestmark = pytest.mark.gpu


def _same(got, want):
    cmp = O.compare(got, want, rtol=0.0)
    assert cmp["ok"], cmp
    assert cmp["bitwise_equal"] == want.nnz


def _f32(m):
    return pb.CSR(m.indptr, m.indices, m.data.astype(np.float32).astype(np.float64), m.shape)


def _problems():
    """Uneven stencil problems, 2D and 3D, tiny to mid-size."""
    out = []
    for dims in [(6, 5), (64, 64), (12, 12, 12), (31, 17), (24, 20, 9), (3, 3, 3), (200, 150)]:
        A = pb.poisson3d(*dims) if len(dims) == 3 else pb.poisson2d(*dims)
        P = pb.jacobi_smooth(A, pb.block_aggregation(dims, 2))
        out.append((P.transpose(), A, P))
    return out


@pytest.fixture(scope="module")
def mixed(orc):
    """Direct R*A*P products and SpMM products (A*P, R*A) with oracles."""
    probs = _problems()
    specs, wants = [], []
    for R, A, P in probs:
        specs.append((R, A, P))
        wants.append(orc.sp3mm_direct(R, A, P))
    for R, A, P in probs[:4]:
        specs.append((A, P))
        wants.append(orc.spmm(A, P))
        specs.append((R, A))
        wants.append(orc.spmm(R, A))
    return specs, wants


def _run(ctx, specs, tuning=None, out_vt=S.F64, in_vt=S.F64, flavour=S.UB):
    dev = [tuple(ctx.upload(m, in_vt) for m in s) for s in specs]
    b = ctx.batch(dev, out_vt, flavour)
    if tuning is not None:
        b.set_tuning(**tuning)
    b.run()
    got = [b.result(i).download() for i in range(len(specs))]
    info = b.info()
    b.free()
    for t in dev:
        for m in t:
            m.free()
    return got, info


@pytest.mark.parametrize("flavour", [S.UB, S.SYMBNUM])
def test_batch_mixed_bit_exact(mixed, flavour):
    specs, wants = mixed
    with S.Context() as ctx:
        got, info = _run(ctx, specs, flavour=flavour)
    assert info["nnz"] == sum(w.nnz for w in wants)
    for g, w in zip(got, wants):
        _same(g, w)


@pytest.mark.parametrize("tuning", [
    dict(d1=0, d2=0, slack=0, splits=None),
    dict(d1=3, d2=3, slack=1, splits=[]),
    dict(d1=1, d2=2, slack=0, splits=[2]),
    dict(d1=6, d2=6, slack=2, splits=[1, 3]),
])
def test_batch_tuning_invariance(mixed, tuning):
    specs, wants = mixed
    with S.Context() as ctx:
        for flavour in (S.UB, S.SYMBNUM):
            got, _ = _run(ctx, specs, tuning, flavour=flavour)
            for g, w in zip(got, wants):
                _same(g, w)


def test_batch_value_types(mixed, orc):
    specs, _ = mixed
    specs32 = [tuple(_f32(m) for m in s) for s in specs]
    wants = [orc.sp3mm_direct(*s) if len(s) == 3 else orc.spmm(*s) for s in specs32]
    with S.Context() as ctx:
        got_ff, _ = _run(ctx, specs32, out_vt=S.F32, in_vt=S.F32)
        got_fd, _ = _run(ctx, specs32, out_vt=S.F64, in_vt=S.F32)
        got_df, _ = _run(ctx, specs, out_vt=S.F32, in_vt=S.F64)
    for g, w in zip(got_ff, wants):
        _same(g, _f32(w))
    for g, w in zip(got_fd, wants):
        _same(g, w)
    want64 = [orc.sp3mm_direct(*s) if len(s) == 3 else orc.spmm(*s) for s in specs]
    for g, w in zip(got_df, want64):
        _same(g, _f32(w))


def test_batch_replay_new_values(orc):
    """Execute replays the captured numeric graph on the operands' current
    values; patterns stay those of the plan."""
    probs = _problems()[:4]
    rng = np.random.default_rng(5)
    with S.Context() as ctx:
        dev = [tuple(ctx.upload(m) for m in s) for s in probs]
        b = ctx.batch(dev)
        b.run()
        for _ in range(2):
            newA = []
            for (R, A, P), (dR, dA, dP) in zip(probs, dev):
                A2 = pb.CSR(A.indptr, A.indices, A.data * rng.uniform(0.5, 2.0, A.nnz), A.shape)
                dA.set_values(A2.data)
                newA.append(A2)
            b.execute()
            ctx.sync()
            for i, ((R, _, P), A2) in enumerate(zip(probs, newA)):
                _same(b.result(i).download(), orc.sp3mm_direct(R, A2, P))
        b.free()


def test_batch_autotune_keeps_results(mixed):
    specs, wants = mixed
    with S.Context() as ctx:
        dev = [tuple(ctx.upload(m) for m in s) for s in specs]
        b = ctx.batch(dev)
        b.plan()
        report = b.autotune(reps=2)
        assert "ms=" in report and len(report.splitlines()) >= 2
        b.execute()
        ctx.sync()
        for i, w in enumerate(wants):
            _same(b.result(i).download(), w)
        b.free()


def test_batch_replay_after_booked_plan(mixed):
    """A booked plan computes the values; the first execute builds the exact
    replay graph and reproduces them."""
    specs, wants = mixed
    with S.Context() as ctx:
        dev = [tuple(ctx.upload(m) for m in s) for s in specs]
        b = ctx.batch(dev)
        b.run()
        first = [b.result(i).download() for i in range(len(specs))]
        b.execute()
        ctx.sync()
        for i, w in enumerate(wants):
            _same(first[i], w)
            _same(b.result(i).download(), w)
        b.free()


@pytest.mark.parametrize("flavour", [S.UB, S.SYMBNUM])
def test_batch_long_rows_global_tables(orc, flavour):
    """Rows with thousands of distinct columns exceed every shared-memory
    tier: symbolic retries and the global-memory tiers take them."""
    X = pb.random_sparse(40, 2000, 0.12, seed=11)
    Y = pb.random_sparse(2000, 20000, 0.002, seed=12)
    Z = pb.random_sparse(20000, 3000, 0.0015, seed=13)
    small = _problems()[1]
    specs = [(X, Y), (X, Y, Z), small]
    wants = [orc.spmm(X, Y), orc.sp3mm_direct(X, Y, Z), orc.sp3mm_direct(*small)]
    assert int(np.diff(wants[0].indptr).max()) > 4000
    with S.Context() as ctx:
        got, info = _run(ctx, specs, flavour=flavour)
        if flavour == S.SYMBNUM:
            assert info["global_tiers"] >= 1
    for g, w in zip(got, wants):
        _same(g, w)


def test_batch_degenerate(orc):
    Z0 = pb.CSR(np.zeros(4, np.int64), np.zeros(0, np.int64), np.zeros(0), (3, 5))
    E = pb.CSR(np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0), (0, 3))
    B = pb.random_sparse(5, 4, 0.5, seed=3)
    A = pb.random_sparse(3, 3, 0.6, seed=4, empty_rows=0.3)
    specs = [(Z0, B), (E, A), (A, A, A), (A, A)]
    wants = [orc.spmm(Z0, B), orc.spmm(E, A), orc.sp3mm_direct(A, A, A), orc.spmm(A, A)]
    with S.Context() as ctx:
        for flavour in (S.UB, S.SYMBNUM):
            got, _ = _run(ctx, specs, flavour=flavour)
            for g, w in zip(got, wants):
                _same(g, w)
        empty = ctx.batch([])
        empty.run()
        assert empty.info()["nnz"] == 0
        empty.free()


def test_batch_rejects_bad_inputs():
    A = pb.poisson2d(8, 8)
    with S.Context() as ctx:
        dA, dA32 = ctx.upload(A), ctx.upload(A, S.F32)
        dB = ctx.upload(pb.random_sparse(10, 4, 0.3, seed=1))
        with pytest.raises(S.Sp3mmError):
            ctx.batch([(dA, dB)])                 # X.N != Y.M
        with pytest.raises(S.Sp3mmError):
            ctx.batch([(dA, dA), (dA32, dA32)])   # mixed value types
        with pytest.raises(S.Sp3mmError):
            ctx.batch([(dA, dA, dB)])             # Y.N != Z.M


@pytest.mark.parametrize("flavour", [S.UB, S.SYMBNUM])
@pytest.mark.parametrize("in_vt", [S.F64, S.F32])
def test_batch_heavy_direct_rows(orc, flavour, in_vt):
    # An all-direct batch holding a coarse-level product (the second level of
    # a 32^3 hierarchy: R*A rows of about 2,000 columns), whose rows run on
    # the CTA-per-row kernel, next to small products on the warp kernels --
    # and a product whose R*A rows exceed the CTA's 4096-entry list (retried).
    dims = (32, 32, 32)
    A0 = pb.poisson3d(*dims)
    with S.Context() as ctx:
        dA0 = ctx.upload(A0)
        h = ctx.hierarchy(dA0, dims, min_coarse=64)
        A1, P1, R1 = h.level(1)
        heavy = (R1.download(), A1.download(), P1.download())
        h.free()
        dA0.free()
    wide = (pb.random_sparse(6, 400, 0.9, seed=11), pb.random_sparse(400, 20000, 0.02, seed=12),
            pb.random_sparse(20000, 64, 0.05, seed=13))
    specs = [heavy, wide] + [s for s in _problems()[:3]]
    if in_vt == S.F32:
        specs = [tuple(_f32(m) for m in s) for s in specs]
    wants = [orc.sp3mm_direct(*s) for s in specs]
    with S.Context() as ctx:
        got, info = _run(ctx, specs, in_vt=in_vt, out_vt=in_vt, flavour=flavour)
    for g, w in zip(got, wants):
        if in_vt == S.F64:
            _same(g, w)
        else:
            assert np.array_equal(g.indptr, w.indptr) and np.array_equal(g.indices, w.indices)
            assert np.array_equal(np.asarray(g.data, np.float32),
                                  np.asarray(w.data, np.float64).astype(np.float32))


def test_batch_heavy_rows_replay_new_values(orc):
    # The exact numeric graph (replays) runs the heavy levels on the
    # CTA-per-row kernel too; new operand values, same patterns.
    dims = (32, 32, 32)
    A0 = pb.poisson3d(*dims)
    rng = np.random.default_rng(9)
    with S.Context() as ctx:
        dA0 = ctx.upload(A0)
        h = ctx.hierarchy(dA0, dims, min_coarse=64)
        A1, P1, R1 = h.level(1)
        heavy = (R1.download(), A1.download(), P1.download())
        h.free()
        dA0.free()
        probs = [heavy] + _problems()[:2]
        dev = [tuple(ctx.upload(m) for m in s) for s in probs]
        b = ctx.batch(dev)
        b.run()
        for _ in range(2):
            newA = []
            for (R, A, P), (dR, dA, dP) in zip(probs, dev):
                A2 = pb.CSR(A.indptr, A.indices, A.data * rng.uniform(0.5, 2.0, A.nnz), A.shape)
                dA.set_values(A2.data)
                newA.append(A2)
            b.execute()
            ctx.sync()
            for i, ((R, _, P), A2) in enumerate(zip(probs, newA)):
                _same(b.result(i).download(), orc.sp3mm_direct(R, A2, P))
        b.free()
