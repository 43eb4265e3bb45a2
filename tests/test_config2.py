"""The irregular workload (kNN graph Laplacian, greedy aggregation): the
generator's properties on the CPU, parity against the oracle at a reduced
size and at the full million points (every variant and flavour bit for
bit), and size-independent properties at the full size on the GPU."""
import numpy as np
import pytest

import oracle as O
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import problems as pb


@pytest.fixture(scope="module")
def small():
    return pb.knn_problem(20000, seed=7)


def test_knn_laplacian_properties():
    A, pts = pb.knn_laplacian(5000, seed=3)
    a = A.to_scipy()
    assert abs(a - a.T).max() == 0.0
    deg = np.diff(A.indptr) - 1
    assert deg.min() >= 16 and deg.max() <= 40
    import scipy.sparse as sp
    off = (a - sp.diags(a.diagonal())).tocsr()
    off.eliminate_zeros()
    assert np.all(off.data < 0) and np.all(-off.data >= 0.5) and np.all(-off.data <= 1.5)
    margin = a.diagonal() - np.asarray(abs(off).sum(axis=1)).ravel()
    assert np.allclose(margin, 1e-3)


def test_greedy_aggregation_properties():
    A, _ = pb.knn_laplacian(20000, seed=3)
    lab = pb.greedy_aggregation(A, seed=3)
    assert np.array_equal(lab, pb.greedy_aggregation(A, seed=3))   # seeded
    sizes = np.bincount(lab)
    assert lab.min() == 0 and sizes.min() >= 1
    assert 7.0 < sizes.mean() < 9.0
    # every aggregate of two or more vertices is connected in the graph
    a = A.to_scipy().tocsr()
    for g in np.flatnonzero(sizes >= 2)[:200]:
        members = np.flatnonzero(lab == g)
        sub = a[members][:, members]
        assert (np.asarray((sub != 0).sum(axis=1)).ravel() >= 2).all()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [S.PAIR, S.DIRECT, S.PAIR_RIGHT])
@pytest.mark.parametrize("flavour", [S.UB, S.SYMBNUM])
def test_config2_small_parity(small, orc, variant, flavour):
    want = (orc.sp3mm_direct if variant == S.DIRECT else
            orc.sp3mm_pair_right if variant == S.PAIR_RIGHT else orc.sp3mm_pair)(
        small.R, small.A, small.P)
    with S.Context() as ctx:
        d = [ctx.upload(m) for m in (small.R, small.A, small.P)]
        C = ctx.rap(*d, variant, flavour).download()
    cmp = O.compare(C, want, rtol=1e-12)
    assert cmp["ok"], cmp
    assert cmp["bitwise_equal"] == want.nnz


@pytest.fixture(scope="module")
def full():
    """The benchmarked problem: 1,000,000 points, seed 2."""
    return pb.knn_problem(1_000_000, seed=2)


@pytest.fixture(scope="module")
def full_oracle(full, orc):
    return {S.PAIR: orc.sp3mm_pair(full.R, full.A, full.P),
            S.DIRECT: orc.sp3mm_direct(full.R, full.A, full.P),
            S.PAIR_RIGHT: orc.sp3mm_pair_right(full.R, full.A, full.P)}


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [S.PAIR, S.DIRECT, S.PAIR_RIGHT])
@pytest.mark.parametrize("flavour", [S.UB, S.SYMBNUM])
def test_config2_full_size_parity(full, full_oracle, variant, flavour):
    """The million-point product against the oracle (which resets only the
    entries it touched, so it finishes in seconds here): pattern bit-exact,
    every value bit-identical."""
    want = full_oracle[variant]
    with S.Context() as ctx:
        d = [ctx.upload(m) for m in (full.R, full.A, full.P)]
        C = ctx.rap(*d, variant, flavour).download()
    cmp = O.compare(C, want, rtol=1e-12)
    assert cmp["ok"], cmp
    assert cmp["bitwise_equal"] == want.nnz


@pytest.mark.gpu
def test_config2_full_size_properties(full):
    """1,000,000 points: direct and pair-wise agree in pattern (values within
    1e-12), the upper-bound and symbolic-numeric flavours agree bit for bit,
    C is symmetric, and 1'C1 equals (P1)'A(P1)."""
    prob = full
    with S.Context() as ctx:
        d = [ctx.upload(m) for m in (prob.R, prob.A, prob.P)]
        Cd = ctx.rap(*d, S.DIRECT, S.UB).download()
        Cs = ctx.rap(*d, S.DIRECT, S.SYMBNUM).download()
        Cp = ctx.rap(*d, S.PAIR, S.UB).download()
    assert O.compare(Cs, Cd, rtol=0.0)["bitwise_equal"] == Cd.nnz
    # (R*A)*P and the direct order differ by association: entries with
    # cancellation differ relatively, so the bound is relative to max |C|.
    assert np.array_equal(Cp.indptr, Cd.indptr) and np.array_equal(Cp.indices, Cd.indices)
    assert np.abs(Cp.data - Cd.data).max() <= 1e-12 * np.abs(Cd.data).max()
    c = Cd.to_scipy()
    assert abs(c - c.T).max() <= 1e-12 * abs(c).max()
    p1 = prob.P.to_scipy() @ np.ones(prob.P.N)
    want = p1 @ (prob.A.to_scipy() @ p1)
    assert abs(Cd.data.sum() - want) <= 1e-9 * np.abs(Cd.data).sum()
    assert 100_000 < prob.P.N < 160_000
