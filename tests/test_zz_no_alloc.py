"""sp3mm_rap_direct_noalloc: the direct R*A*P that allocates no device memory.

Callers whose device memory belongs to another allocator (a solver or
framework that reserved the GPU's memory up front), or that cannot afford a
trip to the CUDA allocator inside a timed loop, cannot use an entry point
that allocates its temporaries.  This one keeps them in a fixed array inside
the library and writes C into arrays the caller owns.  The tests call it
through the C ABI and check, on two calls in a row, that its result equals
both the oracle (bit for bit, within the tests' 1e-12 tolerance) and the
allocating entry point (sp3mm_rap, direct, symbolic-numeric); that a call
leaves the device memory pool and the free device memory unchanged; that
operands with unknown longest rows (max_row = -1) are handled; and its size
and capacity errors.  The file is collected last so that a failure here
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


class _Out:
    """Caller-owned device arrays for C (allocated before any measured call)."""

    def __init__(self, M, capacity):
        import torch
        self.rp = torch.zeros(M + 1, dtype=torch.int32, device="cuda")
        self.col = torch.zeros(max(capacity, 1), dtype=torch.int32, device="cuda")
        self.val = torch.zeros(max(capacity, 1), dtype=torch.float64, device="cuda")
        self.capacity = capacity


def _noalloc(lib, dR, dA, dP, out):
    import torch
    nnz = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    rc = lib.sp3mm_rap_direct_noalloc(dR.ref, dA.ref, dP.ref, out.rp.data_ptr(),
                                      out.col.data_ptr(), out.val.data_ptr(), out.capacity,
                                      ctypes.byref(nnz), None)
    torch.cuda.synchronize()
    n = int(nnz.value)
    got = None
    if rc == 0:
        got = pb.CSR(out.rp.cpu().numpy().astype(np.int64),
                     out.col[:n].cpu().numpy().astype(np.int64), out.val[:n].cpu().numpy(),
                     dR.shape[:1] + dP.shape[1:])
    return rc, n, got


def _memory_state():
    """(bytes in use in the device's default memory pool, free device bytes)."""
    from cuda.bindings import runtime as cudart
    err, dev = cudart.cudaGetDevice()
    assert err == cudart.cudaError_t.cudaSuccess
    err, pool = cudart.cudaDeviceGetDefaultMemPool(dev)
    assert err == cudart.cudaError_t.cudaSuccess
    err, used = cudart.cudaMemPoolGetAttribute(
        pool, cudart.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == cudart.cudaError_t.cudaSuccess
    err, free, _total = cudart.cudaMemGetInfo()
    assert err == cudart.cudaError_t.cudaSuccess
    return int(used), int(free)


def _check(got, want, label):
    cmp = O.compare(got, want, rtol=RTOL)
    assert cmp["ok"], (label, cmp)
    assert cmp["bitwise_equal"] == want.nnz, (label, cmp)


def test_noalloc_matches_oracle_and_allocating_entry_point_twice():
    lib = capi.load()
    orc = O.Oracle()
    problems = [pb.config0(), pb.stencil_problem(3, 24)]
    with S.Context() as ctx:
        for prob in problems:
            oracle_c = orc.sp3mm_direct(prob.R, prob.A, prob.P)
            dR, dA, dP = ctx.upload(prob.R), ctx.upload(prob.A), ctx.upload(prob.P)
            alloc_c = ctx.rap(dR, dA, dP, S.DIRECT, S.SYMBNUM).download()
            ctx.sync()
            out = _Out(prob.R.M, oracle_c.nnz + 17)
            for call in range(2):
                rc, n, got = _noalloc(lib, dR, dA, dP, out)
                assert rc == 0 and n == oracle_c.nnz
                _check(got, oracle_c, f"oracle, call {call}")
                _check(got, alloc_c, f"sp3mm_rap, call {call}")


def test_noalloc_allocates_nothing():
    lib = capi.load()
    prob = pb.stencil_problem(3, 24)
    with S.Context() as ctx:
        dR, dA, dP = ctx.upload(prob.R), ctx.upload(prob.A), ctx.upload(prob.P)
        want = ctx.rap(dR, dA, dP, S.DIRECT, S.SYMBNUM).download()
        out = _Out(prob.R.M, want.nnz)
        ctx.sync()
        # The first call loads the kernels and looks up the scratch array;
        # the calls after it must not touch either allocator.
        assert _noalloc(lib, dR, dA, dP, out)[0] == 0
        before = _memory_state()
        for _ in range(2):
            rc, n, got = _noalloc(lib, dR, dA, dP, out)
            assert rc == 0 and n == want.nnz
        assert _memory_state() == before
        _check(got, want, "after the measured calls")


def test_noalloc_operands_without_max_row():
    """P with many columns and rows that overflow the optimistic tables: with
    max_row unknown the retry tables must come from the measured longest
    row, not from P's column count (which would not fit shared memory)."""
    lib = capi.load()
    orc = O.Oracle()
    R = pb.random_sparse(300, 2000, 0.004, seed=11)
    A = pb.random_sparse(2000, 2000, 0.0025, seed=12)
    P = pb.random_sparse(2000, 20000, 0.0002, seed=13)
    want = orc.sp3mm_direct(R, A, P)
    with S.Context() as ctx:
        d = [ctx.upload(m) for m in (R, A, P)]
        for m in d:
            m.d.max_row = -1
        out = _Out(R.M, want.nnz)
        ctx.sync()
        for call in range(2):
            rc, n, got = _noalloc(lib, *d, out)
            assert rc == 0 and n == want.nnz
            _check(got, want, f"call {call}")


def test_noalloc_reports_capacity_and_size_limits():
    lib = capi.load()
    prob = pb.config0()
    with S.Context() as ctx:
        dR, dA, dP = ctx.upload(prob.R), ctx.upload(prob.A), ctx.upload(prob.P)
        ctx.sync()
        small = _Out(prob.R.M, 100)
        rc, n, _ = _noalloc(lib, dR, dA, dP, small)
        assert rc == capi.SP3MM_ENOMEM and n == 12676
        # On ENOMEM the row pointers are written, so the caller can size C.
        assert int(small.rp[-1]) == 12676
        # Enough rows to exceed the fixed scratch array.
        M, K = 4_000_000, 10
        eye = pb.CSR(np.arange(K + 1, dtype=np.int64), np.arange(K, dtype=np.int64),
                     np.ones(K), (K, K))
        empty = pb.CSR(np.zeros(M + 1, np.int64), np.zeros(0, np.int64), np.zeros(0), (M, K))
        dE, dI = ctx.upload(empty), ctx.upload(eye)
        ctx.sync()
        rc, _, _ = _noalloc(lib, dE, dI, dI, _Out(M, 10))
        assert rc == capi.SP3MM_ELIMIT
        # Still correct after the errors.
        want = ctx.rap(dR, dA, dP, S.DIRECT, S.SYMBNUM).download()
        rc, n, got = _noalloc(lib, dR, dA, dP, _Out(prob.R.M, want.nnz))
        assert rc == 0
        _check(got, want, "after the errors")
