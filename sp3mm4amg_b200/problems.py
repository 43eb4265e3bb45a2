"""Seeded synthetic AMG setup problems: the inputs R, A, P of C = R*A*P.

The reference measured on AMG4PSBLAS operator dumps (its thesis data set,
absent from the reference tree); these generators stand in for them with the
same shapes and value distributions:

* ``poisson2d`` / ``poisson3d``: 5-point / 7-point Laplacians (diag 4 / 6,
  off-diagonal -1), FP64, 0-based ordered CSR, lexicographic numbering with x
  fastest.
* ``block_aggregation``: tentative prolongator P0 of non-overlapping 2x2
  (2x2x2) grid blocks, one entry of value 1.0 per fine row.
* ``jacobi_smooth``: P = (I - omega D^-1 A) P0 with omega = 2/3.
* ``galerkin_problem``: the triple (R = P^T, A, P) of a named workload.

All matrices are returned as :class:`CSR` with int64 indices, columns strictly
ascending in every row (the ordered CSR the reference's parser produces,
code/src/lib/parser.c:126-216).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.sparse as sp


@dataclasses.dataclass
class CSR:
    """A host CSR matrix: ``indptr[M+1]``, ``indices[nnz]``, ``data[nnz]``."""

    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    shape: tuple

    @property
    def M(self) -> int:
        return int(self.shape[0])

    @property
    def N(self) -> int:
        return int(self.shape[1])

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    @classmethod
    def from_scipy(cls, m) -> "CSR":
        m = sp.csr_matrix(m)
        m.sum_duplicates()
        m.sort_indices()
        return cls(np.ascontiguousarray(m.indptr, dtype=np.int64),
                   np.ascontiguousarray(m.indices, dtype=np.int64),
                   np.ascontiguousarray(m.data, dtype=np.float64),
                   (int(m.shape[0]), int(m.shape[1])))

    def to_scipy(self):
        return sp.csr_matrix((self.data, self.indices, self.indptr), shape=self.shape)

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.indptr)

    def transpose(self) -> "CSR":
        return CSR.from_scipy(self.to_scipy().T.tocsr())

    def rows(self, start: int, stop: int) -> "CSR":
        """Rows [start, stop) as a CSR of the same column count."""
        s, e = int(self.indptr[start]), int(self.indptr[stop])
        return CSR(self.indptr[start:stop + 1] - s, self.indices[s:e].copy(),
                   self.data[s:e].copy(), (stop - start, self.N))

    def nbytes(self, idx_bytes: int = 8) -> int:
        """Compulsory bytes of the matrix: row pointers, column indices, values."""
        return (self.M + 1) * idx_bytes + self.nnz * (idx_bytes + 8)


def _stencil(dims, diag: float) -> CSR:
    """Lexicographic (x fastest) 2*d+1 point Laplacian on a box grid."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    idx = np.arange(n, dtype=np.int64)
    coords = []
    rem = idx
    for d in dims:
        coords.append(rem % d)
        rem = rem // d
    rows = [idx]
    cols = [idx]
    vals = [np.full(n, diag)]
    stride = 1
    for axis, d in enumerate(dims):
        c = coords[axis]
        for step in (-1, 1):
            ok = (c + step >= 0) & (c + step < d)
            rows.append(idx[ok])
            cols.append(idx[ok] + step * stride)
            vals.append(np.full(int(ok.sum()), -1.0))
        stride *= d
    m = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    return CSR.from_scipy(m)


def poisson2d(nx: int, ny: int | None = None) -> CSR:
    return _stencil((nx, ny or nx), 4.0)


def poisson3d(nx: int, ny: int | None = None, nz: int | None = None) -> CSR:
    return _stencil((nx, ny or nx, nz or nx), 6.0)


def block_aggregation(dims, block: int = 2) -> CSR:
    """P0 of non-overlapping block^d grid blocks (partial blocks at odd edges)."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    idx = np.arange(n, dtype=np.int64)
    cdims = [-(-d // block) for d in dims]
    agg = np.zeros(n, dtype=np.int64)
    rem = idx
    cstride = 1
    for d, cd in zip(dims, cdims):
        agg += ((rem % d) // block) * cstride
        rem = rem // d
        cstride *= cd
    nc = int(np.prod(cdims))
    return CSR(np.arange(n + 1, dtype=np.int64), agg, np.ones(n), (n, nc))


def jacobi_smooth(A: CSR, P0: CSR, omega: float = 2.0 / 3.0) -> CSR:
    """P = (I - omega D^-1 A) P0, one damped-Jacobi smoothing step."""
    a = A.to_scipy()
    d = a.diagonal()
    scale = sp.diags(omega / d)
    p = (P0.to_scipy() - scale @ (a @ P0.to_scipy())).tocsr()
    return CSR.from_scipy(p)


def aggregates_from_labels(labels: np.ndarray) -> CSR:
    """P0 with one 1.0 per fine row at column labels[i]."""
    n = labels.shape[0]
    nc = int(labels.max()) + 1 if n else 0
    return CSR(np.arange(n + 1, dtype=np.int64), labels.astype(np.int64), np.ones(n), (n, nc))


@dataclasses.dataclass
class Problem:
    """One Galerkin product C = R*A*P with its provenance."""

    name: str
    R: CSR
    A: CSR
    P: CSR

    def compulsory_bytes(self, C: CSR | None = None, nnz_c: int | None = None,
                         idx_bytes: int = 8) -> int:
        """R, A and P read once plus C written once."""
        if C is not None:
            cb = C.nbytes(idx_bytes)
        else:
            cb = (self.R.M + 1) * idx_bytes + int(nnz_c) * (idx_bytes + 8)
        return self.R.nbytes(idx_bytes) + self.A.nbytes(idx_bytes) + self.P.nbytes(idx_bytes) + cb


def stencil_problem(dim: int, side, block: int = 2, omega: float = 2.0 / 3.0) -> Problem:
    """Poisson (5-pt in 2D, 7-pt in 3D) + block aggregation + Jacobi smoothing."""
    if isinstance(side, int):
        dims = (side,) * dim
    else:
        dims = tuple(side)
    A = poisson2d(*dims) if dim == 2 else poisson3d(*dims)
    P0 = block_aggregation(dims, block)
    P = jacobi_smooth(A, P0, omega)
    R = P.transpose()
    name = f"poisson{dim}d_{'x'.join(str(d) for d in dims)}_agg{block}"
    return Problem(name, R, A, P)


def config0() -> Problem:
    """2D 5-point Poisson on 64x64, 2x2 aggregation, one Jacobi step (n=4096)."""
    return stencil_problem(2, 64)


def config1() -> Problem:
    """3D 7-point Poisson on 128^3, 2x2x2 aggregation, one Jacobi step."""
    return stencil_problem(3, 128)


def random_sparse(m: int, n: int, density: float, seed: int, empty_rows: float = 0.0) -> CSR:
    """Seeded random ordered CSR with optional empty rows (edge-case inputs)."""
    rng = np.random.default_rng(seed)
    mat = sp.random(m, n, density=density, format="csr", random_state=rng,
                    data_rvs=lambda k: rng.uniform(-1.0, 1.0, k))
    if empty_rows > 0 and m > 0:
        kill = rng.random(m) < empty_rows
        mat = sp.diags((~kill).astype(np.float64)) @ mat
        mat = sp.csr_matrix(mat)
        mat.eliminate_zeros()
    return CSR.from_scipy(mat)


def log_uniform_sides(rng, count: int, nmin: float = 1e3, nmax: float = 2e5):
    """(dim, side) pairs with n = side^dim log-uniform in [nmin, nmax]."""
    out = []
    for _ in range(count):
        dim = 2 if rng.random() < 0.5 else 3
        n = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        side = max(2, int(round(n ** (1.0 / dim))))
        out.append((dim, side))
    return out


def config3_specs(seed: int = 3, count: int = 256):
    """Grid shapes of the batched workload: a fair coin for 2D / 3D and a
    side drawn log-uniformly so that n runs from 1e3 to 2e5."""
    rng = np.random.default_rng(seed)
    return [(s,) * d for d, s in log_uniform_sides(rng, count)]


def config4_specs(seed: int = 4, count: int = 200, large_fraction: float = 0.1):
    """Grid shapes of the served workload: 90% drawn as config3_specs, 10%
    7-point problems with side 64..128."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        if rng.random() < large_fraction:
            out.append((int(rng.integers(64, 129)),) * 3)
        else:
            d, s = log_uniform_sides(rng, 1)[0]
            out.append((s,) * d)
    return out


def poisson_arrivals(rate: float, count: int, seed: int = 5) -> np.ndarray:
    """Arrival times (seconds from 0) of a Poisson process of `rate`/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, count))


def stencil_operator(dims) -> CSR:
    """The 5-point (2D) or 7-point (3D) Poisson operator on a box grid."""
    return poisson3d(*dims) if len(dims) == 3 else poisson2d(*dims)


def knn_laplacian(npoints: int, k: int = 16, seed: int = 2):
    """Symmetric graph Laplacian of `npoints` seeded uniform points in the
    unit cube joined to their k nearest neighbours (pattern symmetrised):
    off-diagonal weights -U(0.5, 1.5) (one draw per undirected edge), the
    diagonal the sum of |off-diagonals| plus 1e-3.  Returns (A, points)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    pts = rng.random((npoints, 3))
    _, nb = cKDTree(pts).query(pts, k=k + 1)
    rows = np.repeat(np.arange(npoints, dtype=np.int64), k)
    cols = nb[:, 1:].reshape(-1).astype(np.int64)
    lo, hi = np.minimum(rows, cols), np.maximum(rows, cols)
    key = np.unique(lo * npoints + hi)          # undirected edges, sorted
    ei, ej = key // npoints, key % npoints
    w = -rng.uniform(0.5, 1.5, key.size)
    off = sp.coo_matrix((np.concatenate([w, w]), (np.concatenate([ei, ej]),
                                                  np.concatenate([ej, ei]))),
                        shape=(npoints, npoints)).tocsr()
    diag = np.asarray(abs(off).sum(axis=1)).ravel() + 1e-3
    A = (off + sp.diags(diag)).tocsr()
    return CSR.from_scipy(A), pts


def greedy_aggregation(A: CSR, seed: int = 2, max_size: int = 8,
                       min_free: int = 5) -> np.ndarray:
    """Aggregate labels by seeded parallel greedy aggregation: in rounds,
    every unaggregated vertex with at least `min_free` unaggregated
    neighbours whose random priority is the smallest among them becomes a
    root and claims up to max_size-1 of its unaggregated neighbours
    (strongest |a_ij| first; a neighbour adjacent to several roots goes to
    the one with the smallest priority), so every aggregate has diameter
    <= 2.  The vertices left over join the aggregate of their strongest
    aggregated neighbour (in rounds, as aggregates reach them)."""
    n = A.M
    rng = np.random.default_rng(seed)
    prio = np.empty(n, np.int64)
    prio[rng.permutation(n)] = np.arange(n)
    rp, ci = A.indptr.astype(np.int64), A.indices.astype(np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    offd = ci != rows
    er, ec, ew = rows[offd], ci[offd], np.abs(A.data[offd])
    agg = np.full(n, -1, np.int64)
    nagg = 0
    big = np.iinfo(np.int64).max
    while True:
        free = agg < 0
        live = free[er] & free[ec]
        # smallest priority among each free vertex and its free neighbours
        m = np.where(free, prio, big)
        np.minimum.at(m, er[live], prio[ec[live]])
        fdeg = np.bincount(er[live], minlength=n)
        cand = free & (fdeg >= min_free)
        # candidates: the local minimum among candidate neighbours
        mc = np.where(cand, prio, big)
        lc = live & cand[er] & cand[ec]
        np.minimum.at(mc, er[lc], prio[ec[lc]])
        roots = np.flatnonzero(cand & (mc == prio))
        if roots.size == 0:
            break
        is_root = np.zeros(n, bool)
        is_root[roots] = True
        # candidate claims: free non-root neighbour u of a root r
        c = live & is_root[er] & ~is_root[ec]
        cr, cu, cw = er[c], ec[c], ew[c]
        # each u keeps the root of smallest priority
        best = np.full(n, big)
        np.minimum.at(best, cu, prio[cr])
        keep = prio[cr] == best[cu]
        cr, cu, cw = cr[keep], cu[keep], cw[keep]
        # each root keeps its max_size-1 strongest claims
        order = np.lexsort((-cw, prio[cr]))
        cr, cu = cr[order], cu[order]
        first = np.ones(cr.size, bool)
        first[1:] = cr[1:] != cr[:-1]
        start = np.maximum.accumulate(np.where(first, np.arange(cr.size), 0))
        take = (np.arange(cr.size) - start) < max_size - 1
        ids = nagg + np.arange(roots.size)
        label = np.full(n, -1, np.int64)
        label[roots] = ids
        agg[roots] = ids
        agg[cu[take]] = label[cr[take]]
        nagg += roots.size
    while True:
        # leftovers join the aggregate of their strongest aggregated neighbour
        left = agg < 0
        sel = left[er] & ~left[ec]
        if not sel.any():
            break
        r, cc, w = er[sel], ec[sel], ew[sel]
        order = np.lexsort((-w, r))
        r, cc = r[order], cc[order]
        first = np.ones(r.size, bool)
        first[1:] = r[1:] != r[:-1]
        agg[r[first]] = agg[cc[first]]
    still = np.flatnonzero(agg < 0)          # no aggregated neighbour at all
    agg[still] = nagg + np.arange(still.size)
    return agg


def knn_problem(npoints: int = 1_000_000, k: int = 16, seed: int = 2,
                omega: float = 2.0 / 3.0) -> Problem:
    """The irregular workload: kNN Laplacian, greedy aggregation, one
    damped-Jacobi smoothing step, R = P^T."""
    A, _ = knn_laplacian(npoints, k, seed)
    P0 = aggregates_from_labels(greedy_aggregation(A, seed))
    P = jacobi_smooth(A, P0, omega)
    return Problem(f"knn{k}_{npoints}_seed{seed}", P.transpose(), A, P)
