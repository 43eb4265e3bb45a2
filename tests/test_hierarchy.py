"""Smoothed-aggregation hierarchy: the CPU chain (oracle) pinned to the
host generators, and the device build (sp3mm_hierarchy_build,
sp3mm_block_prolongator) checked level by level against it, bit for bit,
in FP64 and with FP32 coarse storage."""
import numpy as np
import pytest

import oracle as O
from oracle import hierarchy as H
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import problems as pb


def _same(got, want):
    cmp = O.compare(got, want, rtol=0.0)
    assert cmp["ok"], cmp
    assert cmp["bitwise_equal"] == want.nnz


# ---------------------------------------------------------------- CPU only

@pytest.mark.parametrize("dims,block", [((12, 12, 12), 2), ((13, 9, 7), 2), ((20, 17), 3),
                                        ((9, 9, 9), 3)])
def test_oracle_prolongator_matches_generator(orc, dims, block):
    A = pb.poisson3d(*dims) if len(dims) == 3 else pb.poisson2d(*dims)
    want = pb.jacobi_smooth(A, pb.block_aggregation(dims, block))
    got = H.block_prolongator(orc, A, dims, block, 2.0 / 3.0)
    # The generator (scipy) drops explicit zeros; stencils produce none
    # outside P0's pattern, so patterns and values agree exactly.
    _same(got, want)


def test_oracle_chain_levels(orc):
    dims = (16, 16, 16)
    levels = H.chain(orc, pb.poisson3d(*dims), dims, block=2, min_coarse=64)
    sizes = [lv[0].M for lv in levels]
    assert sizes == [4096, 512, 64, 8]
    for A, P, R in levels[:-1]:
        assert P.shape == (A.M, -(-A.M // 8))
        _same(R, P.transpose())
    for A, _, _ in levels:
        a = A.to_scipy()
        assert abs(a - a.T).max() <= 1e-12 * abs(a).max()


def test_oracle_chain_fp32_storage_is_rounded(orc):
    dims = (12, 12, 12)
    lv = H.chain(orc, pb.poisson3d(*dims), dims, coarse_f32=True, min_coarse=8)
    for l, (A, P, _) in enumerate(lv):
        if l > 0:
            assert np.array_equal(A.data, A.data.astype(np.float32).astype(np.float64))
        if P is not None and l > 0:
            assert np.array_equal(P.data, P.data.astype(np.float32).astype(np.float64))


def test_oracle_prolongator_needs_diagonal(orc):
    A = pb.poisson2d(6, 6)
    a = A.to_scipy().tolil()
    a[3, 3] = 0.0
    a = a.tocsr()
    a.eliminate_zeros()
    with pytest.raises(ValueError):
        H.block_prolongator(orc, pb.CSR.from_scipy(a), (6, 6), 2, 2.0 / 3.0)


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("dims,block", [((24, 24, 24), 2), ((13, 9, 7), 2), ((40, 33), 3)])
@pytest.mark.parametrize("vt", [S.F64, S.F32])
def test_device_prolongator(orc, dims, block, vt):
    A = pb.poisson3d(*dims) if len(dims) == 3 else pb.poisson2d(*dims)
    want = H.block_prolongator(orc, A, dims, block, 2.0 / 3.0, f32=(vt == S.F32))
    with S.Context() as ctx:
        dA = ctx.upload(A)
        P = ctx.block_prolongator(dA, dims, block, out_val_type=vt)
        assert P.val_type == vt
        got = P.download()
        P.free()
        dA.free()
    _same(got, want)


@pytest.mark.gpu
def test_device_prolongator_rejects_missing_diagonal():
    a = pb.poisson2d(6, 6).to_scipy().tolil()
    a[5, 5] = 0.0
    a = a.tocsr()
    a.eliminate_zeros()
    with S.Context() as ctx:
        dA = ctx.upload(pb.CSR.from_scipy(a))
        with pytest.raises(S.Sp3mmError):
            ctx.block_prolongator(dA, (6, 6), 2)
        with pytest.raises(S.Sp3mmError):
            ctx.block_prolongator(dA, (6, 5), 2)   # grid does not match A


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [S.DIRECT, S.PAIR])
@pytest.mark.parametrize("flavour", [S.UB, S.SYMBNUM])
def test_device_hierarchy_fp64(orc, variant, flavour):
    dims = (32, 32, 32)
    A0 = pb.poisson3d(*dims)
    want = H.chain(orc, A0, dims, min_coarse=64)
    with S.Context() as ctx:
        dA0 = ctx.upload(A0)
        h = ctx.hierarchy(dA0, dims, min_coarse=64, variant=variant, flavour=flavour)
        assert len(h) == len(want)
        for l, (wA, wP, wR) in enumerate(want):
            A, P, R = h.level(l)
            if variant == S.DIRECT or l == 0:
                _same(A.download(), wA)
            else:
                # pair-wise association: same pattern, values within rounding
                cmp = O.compare(A.download(), wA, rtol=1e-12)
                assert cmp["ok"], cmp
            if wP is None:
                assert P is None and R is None
                continue
            if variant == S.DIRECT:
                _same(P.download(), wP)
                _same(R.download(), wR)
        h.free()
        dA0.free()


@pytest.mark.gpu
def test_device_hierarchy_fp32_coarse(orc):
    """FP32 coarse storage: bit-exact to the emulated chain; the error of
    each level against the FP64 chain stays at FP32 rounding scale."""
    dims = (40, 40, 40)
    A0 = pb.poisson3d(*dims)
    want32 = H.chain(orc, A0, dims, min_coarse=64, coarse_f32=True)
    want64 = H.chain(orc, A0, dims, min_coarse=64)
    with S.Context() as ctx:
        dA0 = ctx.upload(A0)
        h = ctx.hierarchy(dA0, dims, min_coarse=64, coarse_val_type=S.F32)
        assert len(h) == len(want32) == len(want64)
        for l in range(len(h)):
            A, P, _ = h.level(l)
            assert A.val_type == (S.F64 if l == 0 else S.F32)
            got = A.download()
            _same(got, want32[l][0])
            if P is not None:
                assert P.val_type == (S.F64 if l == 0 else S.F32)
                _same(P.download(), want32[l][1])
            # Norm-relative error vs the FP64 chain (on the CPU chain at
            # 40^3: 0, 4.3e-8, 6.3e-8, 8.0e-8, 1.2e-6 for levels 0..4).
            ref = want64[l][0]
            err = np.abs(got.data - ref.data).max() / np.abs(ref.data).max()
            assert err <= 1e-5, (l, err)
        h.free()
        dA0.free()


@pytest.mark.gpu
def test_device_hierarchy_max_levels_and_grid_check(orc):
    dims = (20, 20)
    A0 = pb.poisson2d(*dims)
    with S.Context() as ctx:
        dA0 = ctx.upload(A0)
        h = ctx.hierarchy(dA0, dims, max_levels=2, min_coarse=1)
        assert len(h) == 2
        A1, P1, R1 = h.level(1)
        assert A1.shape == (100, 100) and P1 is None and R1 is None
        h.free()
        with pytest.raises(S.Sp3mmError):
            ctx.hierarchy(dA0, (20, 21))
        dA0.free()


# ---------------------------------------------------------------- batched build

def _instances():
    return [(12, 12, 12), (40, 33), (7, 9, 5), (64, 64), (3, 4), (21, 18, 10)]


@pytest.mark.gpu
@pytest.mark.parametrize("coarse", [S.F64, S.F32])
def test_device_hierarchies_batched(orc, coarse):
    """Level-synchronous batched build: every level of every hierarchy
    equals the oracle chain bit for bit (and so the single build)."""
    dims_list = _instances()
    A0s = [pb.poisson3d(*d) if len(d) == 3 else pb.poisson2d(*d) for d in dims_list]
    wants = [H.chain(orc, A, d, min_coarse=30, max_levels=5, coarse_f32=(coarse == S.F32))
             for A, d in zip(A0s, dims_list)]
    with S.Context() as ctx:
        dA0 = [ctx.upload(A) for A in A0s]
        hs = ctx.hierarchies(dA0, dims_list, min_coarse=30, max_levels=5,
                             coarse_val_type=coarse)
        for h, want in zip(hs, wants):
            assert len(h) == len(want)
            for l, (wA, wP, wR) in enumerate(want):
                A, P, R = h.level(l)
                _same(A.download(), wA)
                if wP is None:
                    assert P is None
                    continue
                _same(P.download(), wP)
                _same(R.download(), wR)
        # Freeing in any order keeps the others' shared arrays valid.
        hs[1].free()
        A, _, _ = hs[0].level(len(hs[0]) - 1)
        _same(A.download(), wants[0][-1][0])
        for h in hs:
            h.free()
        for a in dA0:
            a.free()


@pytest.mark.gpu
def test_device_hierarchies_batched_errors():
    A = pb.poisson2d(6, 6)
    a = A.to_scipy().tolil()
    a[2, 2] = 0.0
    a = a.tocsr()
    a.eliminate_zeros()
    with S.Context() as ctx:
        good, bad = ctx.upload(A), ctx.upload(pb.CSR.from_scipy(a))
        with pytest.raises(S.Sp3mmError):
            ctx.hierarchies([good, good], [(6, 6), (6, 5)])
        with pytest.raises(S.Sp3mmError):
            ctx.hierarchies([good, bad], [(6, 6), (6, 6)], min_coarse=2)
        hs = ctx.hierarchies([good], [(6, 6)], min_coarse=2)
        assert len(hs[0]) >= 2
        hs[0].free()


def test_workload_generators():
    specs = pb.config3_specs(seed=3, count=256)
    assert len(specs) == 256
    ns = [int(np.prod(s)) for s in specs]
    assert min(ns) >= 500 and max(ns) <= 2.2e5
    assert 0.3 < np.mean([len(s) == 3 for s in specs]) < 0.7
    s4 = pb.config4_specs(seed=4, count=400)
    big = [s for s in s4 if len(s) == 3 and s[0] >= 64]
    assert 0.04 < len(big) / len(s4) < 0.2
    t = pb.poisson_arrivals(50.0, 2000, seed=1)
    assert np.all(np.diff(t) > 0)
    assert abs(np.mean(np.diff(t)) - 1 / 50.0) < 0.003
