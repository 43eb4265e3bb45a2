"""GPU parity at the headline size: the 128^3 7-point smoothed-aggregation
product (configuration of the benchmark), all variants and flavours, against
the oracle (bit-exact pattern, values bit-identical) plus size-independent
properties."""
import numpy as np
import pytest

import oracle as O
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import problems as pb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    prob = pb.config1()
    orc = O.Oracle()
    pair = orc.sp3mm_pair(prob.R, prob.A, prob.P)
    direct = orc.sp3mm_direct(prob.R, prob.A, prob.P)
    return prob, pair, direct


def test_config1_sizes(big):
    prob, pair, direct = big
    assert prob.A.nnz == 14_581_760 and prob.P.nnz == 8_290_304
    assert pair.nnz == 8_382_712 and direct.nnz == pair.nnz


@pytest.mark.parametrize("variant", [S.PAIR, S.DIRECT, S.PAIR_RIGHT])
@pytest.mark.parametrize("flavour", [S.UB, S.SYMBNUM])
def test_config1_device(big, variant, flavour):
    prob, pair, direct = big
    with S.Context() as ctx:
        dR, dA, dP = ctx.upload(prob.R), ctx.upload(prob.A), ctx.upload(prob.P)
        C = ctx.rap(dR, dA, dP, variant, flavour).download()
    want = direct if variant == S.DIRECT else pair
    cmp = O.compare(C, want, rtol=1e-12)
    assert cmp["ok"], cmp
    if variant != S.PAIR_RIGHT:
        assert cmp["bitwise_equal"] == want.nnz
    # Size-independent properties: Galerkin product of a symmetric A with
    # R = P^T is symmetric; row sums of A vanish in the interior.
    Cs = C.to_scipy()
    assert abs(Cs - Cs.T).max() <= 1e-12 * abs(Cs).max()


def test_config1_one_based_drop_in(big):
    prob, pair, direct = big
    C = S.sp3mm(prob.R, prob.A, prob.P, "sp3mmRowByRowMerged_", off_f=1)
    cmp = O.compare(C, direct, rtol=0.0)
    assert cmp["ok"] and cmp["bitwise_equal"] == direct.nnz
