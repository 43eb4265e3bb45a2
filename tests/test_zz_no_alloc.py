"""sp3mm_rap_direct_noalloc: the direct R*A*P that allocates no device memory.

Callers whose device memory belongs to another allocator (a solver or
framework that reserved the GPU's memory up front), or that cannot afford a
trip to the CUDA allocator inside a timed loop, cannot use an entry point
that allocates its temporaries.  This one keeps them in a fixed array inside
the library and writes C into arrays the caller owns.  The test compares it,
through the C ABI, with the allocating entry point (sp3mm_rap, direct,
symbolic-numeric) on two calls in a row and on a second problem, and checks
its size and capacity errors.  It is collected last so that a failure here
leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import sp3mm4amg_b200 as S
from sp3mm4amg_b200 import capi, problems as pb

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _noalloc(lib, dR, dA, dP, capacity):
    import torch
    M = dR.shape[0]
    rp = torch.zeros(M + 1, dtype=torch.int32, device="cuda")
    col = torch.zeros(max(capacity, 1), dtype=torch.int32, device="cuda")
    val = torch.zeros(max(capacity, 1), dtype=torch.float64, device="cuda")
    nnz = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    rc = lib.sp3mm_rap_direct_noalloc(dR.ref, dA.ref, dP.ref, rp.data_ptr(), col.data_ptr(),
                                      val.data_ptr(), capacity, ctypes.byref(nnz), None)
    torch.cuda.synchronize()
    n = int(nnz.value)
    out = None
    if rc == 0:
        out = pb.CSR(rp.cpu().numpy().astype(np.int64), col[:n].cpu().numpy().astype(np.int64),
                     val[:n].cpu().numpy(), dR.shape[:1] + dP.shape[1:])
    return rc, n, out


def test_noalloc_matches_allocating_entry_point_twice():
    lib = capi.load()
    problems = [pb.config0(), pb.stencil_problem(3, 24)]
    with S.Context() as ctx:
        for prob in problems:
            dR, dA, dP = ctx.upload(prob.R), ctx.upload(prob.A), ctx.upload(prob.P)
            want = ctx.rap(dR, dA, dP, S.DIRECT, S.SYMBNUM).download()
            ctx.sync()
            for _ in range(2):
                rc, n, got = _noalloc(lib, dR, dA, dP, want.nnz + 17)
                assert rc == 0 and n == want.nnz
                cmp = O.compare(got, want, rtol=RTOL)
                assert cmp["ok"], cmp
                assert cmp["bitwise_equal"] == want.nnz


def test_noalloc_reports_capacity_and_size_limits():
    lib = capi.load()
    prob = pb.config0()
    with S.Context() as ctx:
        dR, dA, dP = ctx.upload(prob.R), ctx.upload(prob.A), ctx.upload(prob.P)
        ctx.sync()
        rc, n, _ = _noalloc(lib, dR, dA, dP, 100)
        assert rc == capi.SP3MM_ENOMEM and n == 12676
        # Enough rows to exceed the fixed scratch array.
        M, K = 4_000_000, 10
        eye = pb.CSR(np.arange(K + 1, dtype=np.int64), np.arange(K, dtype=np.int64),
                     np.ones(K), (K, K))
        empty = pb.CSR(np.zeros(M + 1, np.int64), np.zeros(0, np.int64), np.zeros(0), (M, K))
        dE, dI = ctx.upload(empty), ctx.upload(eye)
        ctx.sync()
        rc, _, _ = _noalloc(lib, dE, dI, dI, 10)
        assert rc == capi.SP3MM_ELIMIT
        # Still correct after the errors.
        want = ctx.rap(dR, dA, dP, S.DIRECT, S.SYMBNUM).download()
        rc, n, got = _noalloc(lib, dR, dA, dP, want.nnz)
        assert rc == 0 and O.compare(got, want, rtol=RTOL)["ok"]
