"""Request server (continuous batching of hierarchy setups): every result is
the same alone and in the mix (bit for bit, and equal to the oracle chain),
admission honours slots and memory, late requests join in-flight steps,
and a failing request does not take the others down."""
import numpy as np
import pytest

import oracle as O
from oracle import hierarchy as H
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import problems as pb
from sp3mm4amg_b200 import serving

pytestmark = pytest.mark.gpu

SPECS = [(12, 12, 12), (40, 33), (9, 7, 5), (64, 64), (20, 20, 20), (30, 31)]


def _same(got, want):
    cmp = O.compare(got, want, rtol=0.0)
    assert cmp["ok"], cmp
    assert cmp["bitwise_equal"] == want.nnz


def _levels(h):
    out = []
    for l in range(len(h)):
        A, P, R = h.level(l)
        out.append(tuple(m.download() if m is not None else None for m in (A, P, R)))
    return out


def _serve_all(ctx, specs, modes, max_active=64, mem_fraction=0.5, min_coarse=30):
    srv = S.Server(ctx, max_active, mem_fraction)
    ids = [srv.submit(pb.stencil_operator(d), d, min_coarse=min_coarse, coarse_val_type=m)
           for d, m in zip(specs, modes)]
    while srv.step():
        pass
    for rid in ids:
        assert srv.poll(rid)[0] == S.Server.DONE
    hs = [srv.take(rid) for rid in ids]
    st = srv.stats()
    srv.free()
    return hs, st


def test_server_mix_equals_alone_and_oracle(orc):
    modes = [S.F64, S.F32, S.F64, S.F32, S.F64, S.F64]
    with S.Context() as ctx:
        mix, st = _serve_all(ctx, SPECS, modes)
        assert st["completed"] == len(SPECS) and st["peak_active"] == len(SPECS)
        for d, m, h in zip(SPECS, modes, mix):
            alone, _ = _serve_all(ctx, [d], [m])
            got, ref = _levels(h), _levels(alone[0])
            assert len(got) == len(ref)
            for a, b in zip(got, ref):
                for x, y in zip(a, b):
                    if y is None:
                        assert x is None
                    else:
                        _same(x, y)
            want = H.chain(orc, pb.stencil_operator(d), d, min_coarse=30, max_levels=20,
                           coarse_f32=(m == S.F32))
            for (x, _, _), (w, _, _) in zip(got, want):
                _same(x, w)
            alone[0].free()
            h.free()


def test_server_late_arrivals_join_in_flight(orc):
    """Requests submitted between steps are admitted while earlier ones are
    mid-hierarchy; their results are unaffected."""
    with S.Context() as ctx:
        srv = S.Server(ctx)
        first = [srv.submit(pb.stencil_operator(d), d, min_coarse=30) for d in SPECS[:2]]
        srv.step()
        assert all(srv.poll(r)[0] == S.Server.ACTIVE for r in first)
        late = [srv.submit(pb.stencil_operator(d), d, min_coarse=30) for d in SPECS[2:4]]
        srv.step()
        states = [srv.poll(r)[0] for r in first + late]
        assert all(s in (S.Server.ACTIVE, S.Server.DONE) for s in states)
        while srv.step():
            pass
        for rid, d in zip(first + late, SPECS[:4]):
            h = srv.take(rid)
            want = H.chain(orc, pb.stencil_operator(d), d, min_coarse=30, max_levels=20)
            for l, (w, _, _) in enumerate(want):
                _same(h.level(l)[0].download(), w)
            h.free()
        assert srv.stats()["completed"] == 4
        srv.free()


def test_server_slots_and_memory_admission():
    with S.Context() as ctx:
        _, st = _serve_all(ctx, SPECS, [S.F64] * len(SPECS), max_active=2)
        assert st["peak_active"] <= 2 and st["completed"] == len(SPECS)
        # A budget that holds one small request at a time.
        srv = S.Server(ctx, 64, 1e-6)
        rid = srv.submit(pb.stencil_operator((8, 8)), (8, 8), min_coarse=4)
        big = srv.submit(pb.stencil_operator((60, 60, 60)), (60, 60, 60))
        while srv.step():
            pass
        st = srv.stats()
        srv.free()
        assert st["completed"] <= 1
    # the 60^3 request never fits this budget: refused, not blocking
    with S.Context() as ctx:
        srv = S.Server(ctx, 64, 1e-6)
        big = srv.submit(pb.stencil_operator((60, 60, 60)), (60, 60, 60))
        srv.step()
        assert srv.poll(big)[0] == S.Server.FAILED
        srv.free()


def test_server_failure_is_isolated(orc):
    a = pb.poisson2d(10, 10).to_scipy().tolil()
    a[7, 7] = 0.0
    a = a.tocsr()
    a.eliminate_zeros()
    bad = pb.CSR.from_scipy(a)
    with S.Context() as ctx:
        srv = S.Server(ctx)
        good = [srv.submit(pb.stencil_operator(d), d, min_coarse=30) for d in SPECS[:3]]
        wrong = srv.submit(bad, (10, 10), min_coarse=4)
        while srv.step():
            pass
        assert srv.poll(wrong)[0] == S.Server.FAILED
        for rid, d in zip(good, SPECS[:3]):
            assert srv.poll(rid)[0] == S.Server.DONE
            h = srv.take(rid)
            want = H.chain(orc, pb.stencil_operator(d), d, min_coarse=30, max_levels=20)
            _same(h.level(len(h) - 1)[0].download(), want[-1][0])
            h.free()
        srv.free()


def test_serving_driver_reports_latency():
    specs = pb.config4_specs(seed=9, count=12, large_fraction=0.0)
    arrivals = pb.poisson_arrivals(200.0, len(specs), seed=9)
    with S.Context() as ctx:
        st, _ = serving.serve_batched(ctx, specs, arrivals)
        assert st["completed"] == len(specs) and st["failed"] == 0
        assert 0 < st["p50_s"] <= st["p99_s"] and st["products"] > 0
        plain = serving.serve_plain(ctx, specs, arrivals)
        assert plain["products"] == st["products"]


def test_serving_level_errors_on_device():
    """FP32 coarse storage against FP64, compared on the device: level 0 is
    FP64 in both modes (no error), coarse levels err at FP32 rounding scale,
    patterns agree."""
    specs = [(20, 20, 20), (64, 64)]
    with S.Context() as ctx:
        _, h64 = serving.serve_batched(ctx, specs, np.zeros(2), S.F64, keep=True, min_coarse=30)
        _, h32 = serving.serve_batched(ctx, specs, np.zeros(2), S.F32, keep=True, min_coarse=30)
        for a, b in zip(h32, h64):
            errs = serving.level_errors(a, b)
            assert errs[0][:3] == (0.0, 0.0, 0) and errs[0][3] > 0 and len(errs) >= 2
            for rel, norm, over, n in errs[1:]:
                assert 0.0 < norm <= 1e-5 and rel < 1e-2
                assert 0 <= over <= n and n > 0
            a.free()
            b.free()


def _explicit_chain(npoints, seed, orc):
    """A kNN operator with its caller-side prolongators for two levels (greedy
    aggregation + one Jacobi step on each level, as an AMG caller with its
    own aggregation rules would pass them) and the oracle's level chain."""
    prob = pb.knn_problem(npoints, seed=seed)
    A0, P0 = prob.A, prob.P
    A1 = orc.sp3mm_direct(P0.transpose(), A0, P0)
    P1 = pb.jacobi_smooth(A1, pb.aggregates_from_labels(pb.greedy_aggregation(A1, seed)))
    A2 = orc.sp3mm_direct(P1.transpose(), A1, P1)
    return A0, [P0, P1], [A0, A1, A2]


def test_server_given_prolongators_alone_and_in_mix(orc):
    """Requests that carry their own prolongators (irregular, greedy
    aggregation): every level equals the oracle chain bit for bit, served
    alone and mixed with block-aggregation requests."""
    chains = [_explicit_chain(3000, 5, orc), _explicit_chain(7000, 6, orc)]
    with S.Context() as ctx:
        for mix in (False, True):
            srv = S.Server(ctx)
            ids = []
            for A0, Ps, _ in chains:
                ids.append(srv.submit_ops(A0, Ps))
                if mix:
                    srv.submit(pb.stencil_operator((20, 20, 20)), (20, 20, 20), min_coarse=30)
            while srv.step():
                pass
            for rid, (_, Ps, want) in zip(ids, chains):
                assert srv.poll(rid)[0] == S.Server.DONE
                h = srv.take(rid)
                assert len(h) == len(Ps) + 1
                for l, (A, P, R) in enumerate(_levels(h)):
                    _same(A, want[l])
                    if l < len(Ps):
                        _same(P, Ps[l])
                        _same(R, Ps[l].transpose())
                h.free()
            srv.free()


def test_server_given_prolongators_fp32_coarse(orc):
    """FP32 coarse storage with given prolongators: level 0 and the pattern of
    every level exact, coarse values at FP32 rounding scale."""
    A0, Ps, want = _explicit_chain(3000, 7, orc)
    with S.Context() as ctx:
        srv = S.Server(ctx)
        rid = srv.submit_ops(A0, Ps, coarse_val_type=S.F32)
        while srv.step():
            pass
        assert srv.poll(rid)[0] == S.Server.DONE
        h = srv.take(rid)
        got = _levels(h)
        _same(got[0][0], want[0])
        for l in (1, 2):
            A = got[l][0]
            assert np.array_equal(A.indptr, want[l].indptr)
            assert np.array_equal(A.indices, want[l].indices)
            scale = np.abs(want[l].data).max()
            assert np.abs(A.data - want[l].data).max() <= 1e-5 * scale
        h.free()
        srv.free()


def test_server_given_prolongators_rejects_mismatched_sizes():
    A0 = pb.stencil_operator((6, 6))
    P = pb.aggregates_from_labels(np.arange(36) // 4)
    bad = pb.aggregates_from_labels(np.arange(5) % 2)   # 5 rows after 9 coarse columns
    with S.Context() as ctx:
        srv = S.Server(ctx)
        with pytest.raises(S.Sp3mmError):
            srv.submit_ops(A0, [P, bad])
        srv.free()
