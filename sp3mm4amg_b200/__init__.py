"""sp3mm4amg_b200 -- B200 (sm_100a) Galerkin triple product C = R*A*P.

Python mirror of the reference's Sp3MM entry points (andreadiiorio/Sp3MM4AMG,
code/src/include/Sp3MM_CSR_OMP_UB_Generic.h and Sp3MM_CSR_OMP_Num_Generic.h)
over the C ABI of ``lib/libsp3mm_b200.so``, plus the device-resident layer
(:class:`Context`, :class:`DeviceCSR`).  Every product runs on the GPU.

Host API (layer 1, reference names, host CSR in and out)::

    C = sp3mm(R, A, P, "sp3mmRowByRowPair_", spmm="spmmRowByRow_SymbNum_")
    C = sp3mm(R, A, P, "sp3mmRowByRowMerged_")          # direct, upper bound
    C = spmm(A, B, "spmmRowByRow_")                       # SpMM, upper bound

Device API (layer 2, operands resident in HBM)::

    with Context() as ctx:
        dR, dA, dP = ctx.upload(R), ctx.upload(A), ctx.upload(P)
        dC = ctx.rap(dR, dA, dP, variant=DIRECT, flavour=UB)
        C = dC.download()
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import capi
from .capi import (BATCH_RAP, BATCH_SPMM, DIRECT, F32, F64, PAIR, PAIR_RIGHT, SYMBNUM, UB,
                   sp3mm_dcsr)
from .problems import CSR, Problem
from .spmat import (CONFIG, HostSpMat, IDXMAP, RBTREE, SPMAT_P, array_from_idx_ptr,
                    csr_from_spmat, idx_t, spmat)

__all__ = [
    "CSR", "Problem", "Context", "DeviceCSR", "Sp3mmError", "spmm", "sp3mm",
    "symb_rowsizes", "ub_rowsizes", "ub_colparts_rowsizes", "elapsed_internal",
    "UB", "SYMBNUM", "PAIR", "DIRECT", "PAIR_RIGHT", "F64", "F32", "RBTREE", "IDXMAP",
    "BATCH_SPMM", "BATCH_RAP", "Batch", "Hierarchy", "Server", "read_mm", "write_mm",
]


class Sp3mmError(RuntimeError):
    """A library call failed (the C layer returned NULL or an error code)."""


_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def _free_spmat(p: int) -> None:
    m = ctypes.cast(p, SPMAT_P).contents
    for arr in (m.AS, m.JA, m.IRP):
        _libc.free(ctypes.cast(arr, ctypes.c_void_p))
    _libc.free(p)


def _take_spmat(p, off_f: int) -> CSR:
    if not p:
        raise Sp3mmError("libsp3mm_b200 returned NULL (see stderr)")
    try:
        return csr_from_spmat(p, off_f)
    finally:
        _free_spmat(p)


def _config(cfg: CONFIG | None) -> CONFIG:
    if cfg is not None:
        return cfg
    return CONFIG(gridRows=20, gridCols=2, symbMMRowImplID=RBTREE, threadNum=1,
                  chunkDistrbFunc=None)


def spmm(A: CSR, B: CSR, name: str = "spmmRowByRow_SymbNum_", off_f: int = 0,
         cfg: CONFIG | None = None) -> CSR:
    """C = A*B through the reference-named SpMM entry point ``name``."""
    lib = capi.load()
    a, b = HostSpMat(A, off_f), HostSpMat(B, off_f)
    c = _config(cfg)
    f = getattr(lib, f"{name}{off_f}")
    return _take_spmat(f(a.ptr, b.ptr, ctypes.byref(c)), off_f)


def sp3mm(R: CSR, A: CSR, P: CSR, name: str = "sp3mmRowByRowPair_", spmm: str | None = None,
          off_f: int = 0, cfg: CONFIG | None = None, pinned: bool = False) -> CSR:
    """C = R*A*P through the reference-named triple-product entry point.

    ``spmm`` names this library's SpMM entry point handed to the driver
    (``None`` passes NULL, the driver's default); ``pinned`` passes the
    inputs in page-locked host memory.
    """
    lib = capi.load()
    r, a, p = (HostSpMat(m, off_f, pinned=pinned) for m in (R, A, P))
    c = _config(cfg)
    fp = None
    if spmm is not None:
        fp = ctypes.cast(getattr(lib, f"{spmm}{off_f}"), ctypes.c_void_p).value
    f = getattr(lib, f"{name}{off_f}")
    return _take_spmat(f(r.ptr, a.ptr, p.ptr, ctypes.byref(c), fp), off_f)


def _sizes(p, n: int) -> np.ndarray:
    if not p:
        raise Sp3mmError("libsp3mm_b200 returned NULL (see stderr)")
    try:
        return array_from_idx_ptr(p, n)
    finally:
        _libc.free(p)


def symb_rowsizes(A: CSR, B: CSR, off_f: int = 0, mode: int = RBTREE) -> np.ndarray:
    """Exact row sizes of A*B with the total at [M] (SpMM_Symb___)."""
    lib = capi.load()
    a, b = HostSpMat(A, off_f), HostSpMat(B, off_f)
    return _sizes(getattr(lib, f"SpMM_Symb___{off_f}")(mode, a.ptr, b.ptr), A.M + 1)


def ub_rowsizes(A: CSR, B: CSR, off_f: int = 0) -> np.ndarray:
    """Upper-bound row sizes of A*B with the total at [M] (spMMSizeUpperbound_)."""
    lib = capi.load()
    a, b = HostSpMat(A, off_f), HostSpMat(B, off_f)
    return _sizes(getattr(lib, f"spMMSizeUpperbound_{off_f}")(a.ptr, b.ptr), A.M + 1)


def ub_colparts_rowsizes(A: CSR, B: CSR, grid_cols: int, b_col_offsets: np.ndarray,
                         off_f: int = 0) -> np.ndarray:
    """Upper bounds per (row, column partition) (spMMSizeUpperboundColParts_)."""
    lib = capi.load()
    a, b = HostSpMat(A, off_f), HostSpMat(B, off_f)
    offs = np.ascontiguousarray(b_col_offsets, dtype=np.uint64)
    f = getattr(lib, f"spMMSizeUpperboundColParts_{off_f}")
    return _sizes(f(a.ptr, b.ptr, grid_cols, offs.ctypes.data_as(ctypes.POINTER(idx_t))),
                  A.M * grid_cols + 1)


def read_mm(path: str, sort_rows: bool = False) -> CSR:
    """Read a MatrixMarket coordinate file with the library's MMtoCSR (the
    reference's loader, code/src/lib/parser.c): 0-based CSR, symmetric files
    expanded, rows in the file's entry order unless ``sort_rows``."""
    lib = capi.load()
    p = lib.MMtoCSR(os.fsencode(path))
    if not p:
        raise Sp3mmError(f"MMtoCSR failed for {path} (see stderr)")
    try:
        if sort_rows:
            rc = lib.sp3mm_spmat_sort_rows(ctypes.cast(p, SPMAT_P), 0)
            if rc:
                raise Sp3mmError(f"sp3mm_spmat_sort_rows failed ({rc})")
        return csr_from_spmat(p, 0)
    finally:
        _free_spmat(p)


def write_mm(csr: CSR, path: str) -> None:
    """Write a CSR as a MatrixMarket "coordinate real general" file
    (sp3mm_write_mm; 1-based indices, values that round-trip exactly)."""
    lib = capi.load()
    h = HostSpMat(csr, 0)
    rc = lib.sp3mm_write_mm(h.ptr, 0, os.fsencode(path))
    if rc:
        raise Sp3mmError(f"sp3mm_write_mm failed for {path} ({rc})")


def elapsed_internal() -> float:
    """Device seconds of the last layer-1 product (the ElapsedInternal global)."""
    return capi.global_double(capi.load(), "ElapsedInternal")


# ---------------------------------------------------------------------------
# Layer 2.

class DeviceCSR:
    """A CSR matrix resident in device memory (owned by its context)."""

    def __init__(self, ctx: "Context", d: sp3mm_dcsr, owned: bool = True):
        self.ctx = ctx
        self.d = d
        self.owned = owned   # False: a view into a hierarchy, freed with it

    @property
    def shape(self):
        return (int(self.d.M), int(self.d.N))

    @property
    def nnz(self) -> int:
        return int(self.d.nnz)

    @property
    def val_type(self) -> int:
        return int(self.d.val_type)

    @property
    def max_row(self) -> int:
        return int(self.d.max_row)

    @property
    def ref(self):
        return ctypes.byref(self.d)

    def download(self) -> CSR:
        M, nnz = self.shape[0], self.nnz
        rp = np.empty(M + 1, np.int64)
        ci = np.empty(max(nnz, 1), np.int64)
        v = np.empty(max(nnz, 1), np.float64)
        self.ctx._check(self.ctx.lib.sp3mm_dcsr_download_arrays(
            self.ctx.h, self.ref, rp.ctypes.data, ci.ctypes.data, v.ctypes.data))
        return CSR(rp, ci[:nnz], v[:nnz], self.shape)

    def set_values(self, values: np.ndarray) -> None:
        """Overwrite the values (same pattern) from host FP64 values."""
        v = np.ascontiguousarray(values, np.float64)
        if v.size != self.nnz:
            raise ValueError("values must have one entry per nonzero")
        self.ctx._check(self.ctx.lib.sp3mm_dcsr_set_values(self.ctx.h, self.ref, v.ctypes.data))

    def free(self) -> None:
        if self.owned and (self.d.row_ptr or self.d.col or self.d.val):
            self.ctx.lib.sp3mm_dcsr_free(self.ctx.h, self.ref)

    def bytes(self, idx_bytes: int = 4) -> int:
        vb = 4 if self.val_type == F32 else 8
        return (self.shape[0] + 1) * idx_bytes + self.nnz * (idx_bytes + vb)


class Context:
    """A device context: CUDA device, stream and the library's workspace."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.lib = capi.load()
        h = ctypes.c_void_p()
        rc = self.lib.sp3mm_ctx_create(device, ctypes.byref(h))
        if rc:
            raise Sp3mmError(f"sp3mm_ctx_create failed ({rc})")
        self.h = h
        if stream is not None:
            self.set_stream(stream)

    def _check(self, rc: int) -> None:
        if rc:
            msg = self.lib.sp3mm_ctx_last_error(self.h)
            raise Sp3mmError(f"error {rc}: {msg.decode() if msg else ''}")

    def set_stream(self, stream: int | None) -> None:
        self._check(self.lib.sp3mm_ctx_set_stream(self.h, stream))

    @property
    def stream(self) -> int:
        return int(self.lib.sp3mm_ctx_stream(self.h) or 0)

    def sync(self) -> None:
        self._check(self.lib.sp3mm_ctx_sync(self.h))

    def launches(self) -> int:
        return int(self.lib.sp3mm_ctx_launches(self.h))

    def set_tuning(self, lanes_per_row: int = 0, d1: int = -1, d2: int = -1) -> None:
        """Row-kernel tuning (lanes per row, table-size shifts); results never
        depend on it -- rows whose tables overflow are recomputed."""
        self._check(self.lib.sp3mm_ctx_set_tuning(self.h, lanes_per_row, d1, d2))

    def trim(self) -> None:
        """Release cached workspace: the device pool's idle memory and the
        page-locked staging (this context's and the process-wide cache)."""
        self._check(self.lib.sp3mm_ctx_trim(self.h))

    def set_profiling(self, on: bool) -> None:
        """Time every kernel launch with CUDA events on the context stream."""
        self._check(self.lib.sp3mm_ctx_set_profiling(self.h, 1 if on else 0))

    def profile(self) -> dict:
        """{label: (launches, total_ms, max_ms)} since profiling was switched on."""
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self.lib.sp3mm_ctx_profile_report(self.h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            label, n, tot, mx = line.split()
            out[label] = (int(n), float(tot), float(mx))
        return out

    def upload(self, m: CSR, val_type: int = F64) -> DeviceCSR:
        d = sp3mm_dcsr()
        rp = np.ascontiguousarray(m.indptr, np.int64)
        ci = np.ascontiguousarray(m.indices, np.int64)
        v = np.ascontiguousarray(m.data, np.float64)
        self._check(self.lib.sp3mm_dcsr_upload_arrays(
            self.h, m.M, m.N, m.nnz, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, val_type,
            ctypes.byref(d)))
        return DeviceCSR(self, d)

    def spmm(self, A: DeviceCSR, B: DeviceCSR, flavour: int = SYMBNUM,
             out_val_type: int = F64) -> DeviceCSR:
        d = sp3mm_dcsr()
        self._check(self.lib.sp3mm_spmm(self.h, A.ref, B.ref, flavour, out_val_type,
                                        ctypes.byref(d)))
        return DeviceCSR(self, d)

    def rap(self, R: DeviceCSR, A: DeviceCSR, P: DeviceCSR, variant: int = DIRECT,
            flavour: int = UB, out_val_type: int = F64) -> DeviceCSR:
        d = sp3mm_dcsr()
        self._check(self.lib.sp3mm_rap(self.h, R.ref, A.ref, P.ref, variant, flavour,
                                       out_val_type, ctypes.byref(d)))
        return DeviceCSR(self, d)

    def transpose(self, A: DeviceCSR) -> DeviceCSR:
        d = sp3mm_dcsr()
        self._check(self.lib.sp3mm_transpose(self.h, A.ref, ctypes.byref(d)))
        return DeviceCSR(self, d)

    def rowsizes(self, A: DeviceCSR, B: DeviceCSR, exact: bool = True):
        """(per-row sizes as int64 numpy array, total)."""
        import torch  # device buffer for the row sizes
        M = A.shape[0]
        buf = torch.empty(max(M, 1), dtype=torch.int32, device="cuda")
        tot = ctypes.c_int64()
        self._check(self.lib.sp3mm_spmm_rowsizes(self.h, A.ref, B.ref, 1 if exact else 0,
                                                 buf.data_ptr(), ctypes.byref(tot)))
        self.sync()
        return buf[:M].cpu().numpy().astype(np.int64), int(tot.value)

    def rap_memory_estimate(self, R: DeviceCSR, A: DeviceCSR, P: DeviceCSR,
                            variant: int = DIRECT, flavour: int = UB) -> int:
        b = ctypes.c_size_t()
        self._check(self.lib.sp3mm_rap_memory_estimate(R.ref, A.ref, P.ref, variant, flavour,
                                                       ctypes.byref(b)))
        return int(b.value)

    def block_prolongator(self, A: DeviceCSR, dims, block: int = 2, omega: float = 2.0 / 3.0,
                          out_val_type: int = F64) -> DeviceCSR:
        """P = (I - omega D^-1 A) P0 for the block^d aggregation of A's grid."""
        dd = (ctypes.c_int32 * 3)(*(list(dims) + [1, 1])[:3])
        d = sp3mm_dcsr()
        self._check(self.lib.sp3mm_block_prolongator(self.h, A.ref, dd, len(dims), block,
                                                     float(omega), out_val_type,
                                                     ctypes.byref(d)))
        return DeviceCSR(self, d)

    def hierarchy(self, A0: DeviceCSR, dims, block: int = 2, omega: float = 2.0 / 3.0,
                  min_coarse: int = 64, max_levels: int = 10, variant: int = DIRECT,
                  flavour: int = UB, coarse_val_type: int = F64) -> "Hierarchy":
        """Device-resident smoothed-aggregation hierarchy over A0 (borrowed)."""
        dd = (ctypes.c_int32 * 3)(*(list(dims) + [1, 1])[:3])
        h = ctypes.c_void_p()
        self._check(self.lib.sp3mm_hierarchy_build(
            self.h, A0.ref, dd, len(dims), block, float(omega), min_coarse, max_levels,
            variant, flavour, coarse_val_type, ctypes.byref(h)))
        return Hierarchy(self, h)

    def hierarchies(self, A0s, dims_list, block: int = 2, omega: float = 2.0 / 3.0,
                    min_coarse: int = 64, max_levels: int = 10,
                    coarse_val_type: int = F64) -> list:
        """Hierarchies over each A0 (borrowed), built level-synchronously with
        batched launches (direct products)."""
        n = len(A0s)
        arr = (sp3mm_dcsr * max(n, 1))(*[a.d for a in A0s])
        dims = (ctypes.c_int32 * max(3 * n, 1))()
        nd = (ctypes.c_int32 * max(n, 1))()
        for i, dm in enumerate(dims_list):
            nd[i] = len(dm)
            for j, x in enumerate((list(dm) + [1, 1])[:3]):
                dims[3 * i + j] = x
        out = (ctypes.c_void_p * max(n, 1))()
        self._check(self.lib.sp3mm_hierarchy_build_batch(
            self.h, n, arr, dims, nd, block, float(omega), min_coarse, max_levels,
            coarse_val_type, out))
        return [Hierarchy(self, ctypes.c_void_p(out[i])) for i in range(n)]

    def batch(self, products, out_val_type: int = F64, flavour: int = UB) -> "Batch":
        """A batch of independent products: (X, Y) for X*Y, (X, Y, Z) for
        the direct X*Y*Z."""
        b = Batch(self, products, out_val_type)
        if flavour != UB:
            b.set_flavour(flavour)
        return b

    def close(self) -> None:
        if self.h:
            self.lib.sp3mm_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Hierarchy:
    """Levels (A_l, P_l, R_l) of a device hierarchy; P/R are None on the last."""

    def __init__(self, ctx: Context, h: ctypes.c_void_p):
        self.ctx = ctx
        self.h = h

    def __len__(self) -> int:
        return int(self.ctx.lib.sp3mm_hierarchy_levels(self.h))

    def level(self, l: int):
        a, p, r = sp3mm_dcsr(), sp3mm_dcsr(), sp3mm_dcsr()
        self.ctx._check(self.ctx.lib.sp3mm_hierarchy_get(self.h, l, ctypes.byref(a),
                                                         ctypes.byref(p), ctypes.byref(r)))
        view = (lambda d: DeviceCSR(self.ctx, d, owned=False) if d.row_ptr else None)
        return view(a), view(p), view(r)

    def free(self) -> None:
        if self.h:
            self.ctx.lib.sp3mm_hierarchy_free(self.ctx.h, self.h)
            self.h = None


class Batch:
    """Many independent products planned together and executed as one
    captured CUDA graph (sp3mm_batch_*)."""

    def __init__(self, ctx: Context, products, out_val_type: int = F64):
        self.ctx = ctx
        self.products = list(products)   # keep the operands alive
        n = len(self.products)
        kinds = (ctypes.c_int * max(n, 1))()
        X = (sp3mm_dcsr * max(n, 1))()
        Y = (sp3mm_dcsr * max(n, 1))()
        Z = (sp3mm_dcsr * max(n, 1))()
        for i, p in enumerate(self.products):
            kinds[i] = BATCH_RAP if len(p) == 3 else BATCH_SPMM
            X[i] = p[0].d
            Y[i] = p[1].d
            if len(p) == 3:
                Z[i] = p[2].d
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.sp3mm_batch_create(ctx.h, n, kinds, X, Y, Z, out_val_type,
                                              ctypes.byref(h)))
        self.h = h

    def __len__(self) -> int:
        return len(self.products)

    def set_tuning(self, d1: int = 2, d2: int = 1, slack: int = 0, splits=None) -> None:
        """splits None: one numeric tier per table level; [] one tier; else
        a new tier starts at each listed level."""
        if splits is None:
            arr, ns = None, -1
        else:
            ns = len(splits)
            arr = (ctypes.c_int32 * max(ns, 1))(*splits)
        self.ctx._check(self.ctx.lib.sp3mm_batch_set_tuning(self.h, d1, d2, slack, ns, arr))

    def set_flavour(self, flavour: int) -> None:
        """UB: booked single numeric pass in the plan; SYMBNUM: symbolic plan."""
        self.ctx._check(self.ctx.lib.sp3mm_batch_set_flavour(self.h, flavour))

    def plan(self) -> None:
        self.ctx._check(self.ctx.lib.sp3mm_batch_plan(self.h))

    def execute(self) -> None:
        self.ctx._check(self.ctx.lib.sp3mm_batch_execute(self.h))

    def run(self) -> None:
        self.ctx._check(self.ctx.lib.sp3mm_batch_run(self.h))

    def autotune(self, reps: int = 3) -> str:
        buf = ctypes.create_string_buffer(1 << 14)
        self.ctx._check(self.ctx.lib.sp3mm_batch_autotune(self.h, reps, buf, len(buf)))
        return buf.value.decode()

    def result(self, i: int) -> DeviceCSR:
        d = sp3mm_dcsr()
        self.ctx._check(self.ctx.lib.sp3mm_batch_result(self.h, i, ctypes.byref(d)))
        return DeviceCSR(self.ctx, d, owned=False)

    def info(self) -> dict:
        rows, nnz, retried = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        tiers, gt = ctypes.c_int(), ctypes.c_int()
        self.ctx._check(self.ctx.lib.sp3mm_batch_info(self.h, ctypes.byref(rows),
                                                      ctypes.byref(nnz), ctypes.byref(tiers),
                                                      ctypes.byref(gt), ctypes.byref(retried)))
        return {"rows": rows.value, "nnz": nnz.value, "tiers": tiers.value,
                "global_tiers": gt.value, "retried": retried.value}

    def free(self) -> None:
        if self.h:
            self.ctx.lib.sp3mm_batch_free(self.h)
            self.h = None


class Server:
    """Continuous-batching hierarchy-setup server (sp3mm_server_*)."""

    QUEUED, ACTIVE, DONE, FAILED, TAKEN = range(5)

    def __init__(self, ctx: Context, max_active: int = 64, mem_fraction: float = 0.5):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.sp3mm_server_create(ctx.h, max_active, float(mem_fraction),
                                               ctypes.byref(h)))
        self.h = h
        self._inputs = {}   # host arrays must outlive admission

    def now(self) -> float:
        return float(self.ctx.lib.sp3mm_server_now(self.h))

    def submit(self, A0: CSR, dims, block: int = 2, omega: float = 2.0 / 3.0,
               min_coarse: int = 1000, max_levels: int = 20, coarse_val_type: int = F64,
               arrival: float = -1.0) -> int:
        rp = np.ascontiguousarray(A0.indptr, np.int64)
        ci = np.ascontiguousarray(A0.indices, np.int64)
        v = np.ascontiguousarray(A0.data, np.float64)
        dd = (ctypes.c_int32 * 3)(*(list(dims) + [1, 1])[:3])
        rid = ctypes.c_int64()
        self.ctx._check(self.ctx.lib.sp3mm_server_submit(
            self.h, A0.M, A0.nnz, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, dd, len(dims),
            block, float(omega), min_coarse, max_levels, coarse_val_type, float(arrival),
            ctypes.byref(rid)))
        self._inputs[rid.value] = (rp, ci, v)
        return rid.value

    def submit_ops(self, A0: CSR, Ps, coarse_val_type: int = F64, arrival: float = -1.0) -> int:
        """A request with the caller's prolongators P_0, P_1, ... (host CSR);
        the server builds R_l = P_l^T and A_{l+1} = R_l A_l P_l."""
        rp = np.ascontiguousarray(A0.indptr, np.int64)
        ci = np.ascontiguousarray(A0.indices, np.int64)
        v = np.ascontiguousarray(A0.data, np.float64)
        prp = [np.ascontiguousarray(P.indptr, np.int64) for P in Ps]
        pci = [np.ascontiguousarray(P.indices, np.int64) for P in Ps]
        pv = [np.ascontiguousarray(P.data, np.float64) for P in Ps]
        n = len(Ps)
        rows = (ctypes.c_int64 * n)(*[P.M for P in Ps])
        cols = (ctypes.c_int64 * n)(*[P.N for P in Ps])
        nnz = (ctypes.c_int64 * n)(*[P.nnz for P in Ps])
        a_rp = (ctypes.c_void_p * n)(*[a.ctypes.data for a in prp])
        a_ci = (ctypes.c_void_p * n)(*[a.ctypes.data for a in pci])
        a_v = (ctypes.c_void_p * n)(*[a.ctypes.data for a in pv])
        rid = ctypes.c_int64()
        self.ctx._check(self.ctx.lib.sp3mm_server_submit_ops(
            self.h, A0.M, A0.nnz, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, n, rows, cols,
            nnz, a_rp, a_ci, a_v, coarse_val_type, float(arrival), ctypes.byref(rid)))
        self._inputs[rid.value] = (rp, ci, v, prp, pci, pv, rows, cols, nnz, a_rp, a_ci, a_v)
        return rid.value

    def step(self) -> int:
        pending = ctypes.c_int()
        self.ctx._check(self.ctx.lib.sp3mm_server_step(self.h, ctypes.byref(pending)))
        # The loader threads read a request's host arrays until its upload is
        # done; drop them once the request has finished.
        for rid in [r for r in self._inputs
                    if self.poll(r)[0] in (self.DONE, self.FAILED, self.TAKEN)]:
            del self._inputs[rid]
        return pending.value

    def poll(self, rid: int):
        """(status, latency_s, queued_s)."""
        st, lat, q = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        self.ctx.lib.sp3mm_server_poll(self.h, rid, ctypes.byref(st), ctypes.byref(lat),
                                       ctypes.byref(q))
        return st.value, lat.value, q.value

    def take(self, rid: int) -> Hierarchy:
        h = ctypes.c_void_p()
        self.ctx._check(self.ctx.lib.sp3mm_server_take(self.h, rid, ctypes.byref(h)))
        return Hierarchy(self.ctx, h)

    def stats(self) -> dict:
        c, pr, st, de = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        p50, p99, busy = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        peak = ctypes.c_int()
        self.ctx._check(self.ctx.lib.sp3mm_server_stats(
            self.h, ctypes.byref(c), ctypes.byref(pr), ctypes.byref(p50), ctypes.byref(p99),
            ctypes.byref(busy), ctypes.byref(st), ctypes.byref(peak), ctypes.byref(de)))
        return {"completed": c.value, "products": pr.value, "p50_s": p50.value,
                "p99_s": p99.value, "busy_s": busy.value, "steps": st.value,
                "peak_active": peak.value, "deferred": de.value}

    def free(self) -> None:
        if self.h:
            self.ctx.lib.sp3mm_server_free(self.h)
            self.h = None
