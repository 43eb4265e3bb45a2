"""Serving driver: a seeded Poisson stream of hierarchy-setup requests fed
to the continuous-batching server (Server) or, for comparison, served one
request at a time by the single hierarchy build."""
from __future__ import annotations

import time

import numpy as np

from . import F32, F64, Context, Server
from .problems import stencil_operator


def _pct(x, q):
    if not len(x):
        return 0.0
    s = np.sort(np.asarray(x))
    return float(s[min(len(s) - 1, int(q * (len(s) - 1) + 0.5))])


def serve_batched(ctx: Context, specs, arrivals, coarse_val_type: int = F64,
                  max_active: int = 64, mem_fraction: float = 0.5, min_coarse: int = 1000,
                  keep: bool = False, operators=None):
    """Feed the requests at their arrival times to a Server and step it
    until all are done.  Returns (stats, hierarchies or None)."""
    ops = operators if operators is not None else [stencil_operator(d) for d in specs]
    srv = Server(ctx, max_active, mem_fraction)
    t0 = srv.now()
    ids, i = [], 0
    n = len(specs)
    while True:
        now = srv.now() - t0
        while i < n and arrivals[i] <= now:
            ids.append(srv.submit(ops[i], specs[i], min_coarse=min_coarse,
                                  coarse_val_type=coarse_val_type, arrival=t0 + arrivals[i]))
            i += 1
        pending = srv.step()
        if pending == 0:
            if i == n:
                break
            time.sleep(max(0.0, arrivals[i] - (srv.now() - t0)))
    makespan = srv.now() - t0
    st = srv.stats()
    st["makespan_s"] = makespan
    st["products_per_s"] = st["products"] / makespan if makespan > 0 else 0.0
    failed = [rid for rid in ids if srv.poll(rid)[0] == Server.FAILED]
    st["failed"] = len(failed)
    hs = [srv.take(rid) for rid in ids] if keep else None
    srv.free()
    return st, hs


def serve_plain(ctx: Context, specs, arrivals, coarse_val_type: int = F64,
                min_coarse: int = 1000, operators=None):
    """First come first served, one request at a time: upload, single
    hierarchy build (one product per call), sync."""
    ops = operators if operators is not None else [stencil_operator(d) for d in specs]
    lat, products = [], 0
    t0 = time.perf_counter()
    for i, (op, dims) in enumerate(zip(ops, specs)):
        now = time.perf_counter() - t0
        if arrivals[i] > now:
            time.sleep(arrivals[i] - now)
        dA = ctx.upload(op)
        h = ctx.hierarchy(dA, dims, min_coarse=min_coarse, max_levels=20,
                          coarse_val_type=coarse_val_type)
        ctx.sync()
        lat.append(time.perf_counter() - t0 - arrivals[i])
        products += len(h) - 1
        h.free()
        dA.free()
    makespan = time.perf_counter() - t0
    return {"completed": len(lat), "products": products, "p50_s": _pct(lat, 0.5),
            "p99_s": _pct(lat, 0.99), "makespan_s": makespan,
            "products_per_s": products / makespan if makespan > 0 else 0.0}


def _device_view(ptr: int, n: int, typestr: str):
    """A torch tensor over n elements of device memory at ptr (no copy)."""
    import torch

    class _Mem:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                    "version": 3}
    return torch.as_tensor(_Mem(), device="cuda")


def level_errors(h32, h64):
    """Per level of two hierarchies of the same request (FP32 coarse storage
    and FP64): (max entrywise relative error over nonzero FP64 entries, max
    error over max |FP64 value|, entries whose relative error exceeds 1e-3,
    entries), computed on the device.  Raises if the patterns differ (they
    must not, in any mode)."""
    import torch
    out = []
    if len(h32) != len(h64):
        raise RuntimeError("hierarchies differ in depth")
    for lvl in range(len(h64)):
        a, b = h32.level(lvl)[0], h64.level(lvl)[0]
        if a.shape != b.shape or a.nnz != b.nnz:
            raise RuntimeError("hierarchies differ in shape or nonzeros")
        n = a.nnz
        if n == 0:
            out.append((0.0, 0.0, 0, 0))
            continue
        rows = a.shape[0] + 1
        for pa, pb, m in ((a.d.row_ptr, b.d.row_ptr, rows), (a.d.col, b.d.col, n)):
            if not torch.equal(_device_view(pa, m, "<i4"), _device_view(pb, m, "<i4")):
                raise RuntimeError("hierarchies differ in pattern")
        va = _device_view(a.d.val, n, "<f4" if a.val_type == F32 else "<f8").double()
        vb = _device_view(b.d.val, n, "<f4" if b.val_type == F32 else "<f8").double()
        diff = (va - vb).abs()
        ref = vb.abs()
        nz = ref > 0
        rels = diff[nz] / ref[nz]
        rel = float(rels.max()) if bool(nz.any()) else 0.0
        over = int((rels > 1e-3).sum()) + int((diff[~nz] > 0).sum())
        norm = float(diff.max() / ref.max()) if float(ref.max()) > 0 else 0.0
        out.append((rel, norm, over, n))
    return out
