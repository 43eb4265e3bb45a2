// kernels.cu -- sm_100a kernels of the Sp3MM triple product.
//
// Gustavson row-by-row products on ordered CSR, re-designed for the GPU:
//
//  * Row binning by upper-bound size.  A bounds kernel computes, per output
//    row, the number of multiply-adds (the reference's upper bound,
//    code/src/include/SpMMUtilsGeneric.h:112-139, extended to R*A*P for the
//    direct product) and the number of table slots the row can need.  Rows
//    are binned into table-size levels (32 .. 4096 slots in shared memory,
//    larger in global memory) by a count / scatter pair of kernels.  This
//    replaces the reference's OpenMP 1D / 2D row and column partitions
//    (code/src/Sp3MM_CSR_OMP_UB_Generic.c:85-105, :153-182, :216-302).
//
//  * Per-row accumulators: a group of G lanes (G = 4..32, picked from the
//    right operand's mean row length) owns one row and one open-addressing
//    hash table.  This replaces the dense accumulator + index bitmap
//    (code/src/include/sparseMatrix.h:60-110) and the RB-tree
//    (code/src/Sp3MM_CSR_OMP_SymbStep_Generic.c:84-161).
//
//  * Reference summation order without value atomics: the lanes walk the
//    left row's entries one step at a time, and within a step they cover the
//    selected right row, whose column indices are distinct, so no two lanes
//    touch the same slot.  Each output entry therefore receives its
//    contributions in ascending left-row position, as in the reference's
//    scSparseVectMul_ loop (code/src/include/SpMMUtilsGeneric.h:39-55), and
//    the values are bit-identical to the reference's.
//
//  * First-touch order for the direct product: new keys of a step are
//    ranked by ballot + popc in lane order, which is the order in which the
//    reference's bitmap appends them to nnzIdx; the R*A row is then forwarded
//    into P in that order (code/src/Sp3MM_CSR_OMP_UB_Generic.c:542-545).
//
//  * Sorted write-out: the row's keys are compacted and sorted (rank sort
//    for short rows, bitonic sort for long rows), replacing the per-row
//    qsort of sparsifyDirect (code/src/include/SpMMUtilsGeneric.h:230-241).
#include <cub/device/device_scan.cuh>

#include <atomic>
#include <climits>

#include "kernels.cuh"
#include "sp3mm_internal.cuh"

namespace sp3mm {

static std::atomic<uint64_t> g_launches{0};
uint64_t launch_count() { return g_launches.load(); }
static inline void counted() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ---------------------------------------------------------------------------
// Value access in either storage type (uniform branch per launch).
__device__ __forceinline__ double load_val(const void* p, int vt, long long i) {
    if (vt == SP3MM_F32) return static_cast<double>(__ldg(static_cast<const float*>(p) + i));
    return __ldg(static_cast<const double*>(p) + i);
}
__device__ __forceinline__ void store_val(void* p, int vt, long long i, double v) {
    if (vt == SP3MM_F32) static_cast<float*>(p)[i] = __double2float_rn(v);
    else static_cast<double*>(p)[i] = v;
}

// ---------------------------------------------------------------------------
// Bounds.

// need[i] = slots bound of row i of A*B (distinct keys <= min(flops, N)),
// total_flops += flops.
template <int G>
__global__ void __launch_bounds__(256) k_pair_bounds(CsrView A, CsrView B, int* need,
                                                      unsigned long long* total) {
    const Group<G> g;
    const int groups = (gridDim.x * blockDim.x) / G;
    unsigned long long mine = 0;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < A.M; row += groups) {
        const int ab = __ldg(A.rp + row), ae = __ldg(A.rp + row + 1);
        long long f = 0;
        for (int t = ab + g.gl; t < ae; t += G) {
            const int k = __ldg(A.ci + t);
            f += __ldg(B.rp + k + 1) - __ldg(B.rp + k);
        }
        f = g.sum64(f);
        if (g.gl == 0) {
            const long long d = f < B.N ? f : B.N;
            need[row] = static_cast<int>(d < INT_MAX ? d : INT_MAX);
            mine += static_cast<unsigned long long>(f);
        }
    }
    // Every lane reaches this point: one atomic per warp.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(total, mine);
}

// Direct R*A*P: need[i] = max(distinct bound of the R*A row, of the C row);
// total_flops += sum_{k in R(i)} sum_{c in A(k)} len(P(c)).
template <int G>
__global__ void __launch_bounds__(256) k_direct_bounds(CsrView R, CsrView A, CsrView P,
                                                        int* need, unsigned long long* total) {
    const Group<G> g;
    const int groups = (gridDim.x * blockDim.x) / G;
    unsigned long long mine = 0;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < R.M; row += groups) {
        const int rb = __ldg(R.rp + row), re = __ldg(R.rp + row + 1);
        long long u1 = 0, u2 = 0;
        for (int t = rb + g.gl; t < re; t += G) {
            const int k = __ldg(R.ci + t);
            const int ab = __ldg(A.rp + k), ae = __ldg(A.rp + k + 1);
            u1 += ae - ab;
            for (int i = ab; i < ae; ++i) {
                const int c = __ldg(A.ci + i);
                u2 += __ldg(P.rp + c + 1) - __ldg(P.rp + c);
            }
        }
        u1 = g.sum64(u1);
        u2 = g.sum64(u2);
        if (g.gl == 0) {
            const long long d1 = u1 < A.N ? u1 : A.N;
            const long long d2 = u2 < P.N ? u2 : P.N;
            const long long d = d1 > d2 ? d1 : d2;
            // A row that forwards nothing needs no table.
            need[row] = u2 == 0 ? 0 : static_cast<int>(d < INT_MAX ? d : INT_MAX);
            mine += static_cast<unsigned long long>(u2);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(total, mine);
}

__global__ void k_need_from_counts(int M, const int* cnt, const int* cnt1, int* need) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    int n = cnt[i];
    if (cnt1 && n > 0) n = max(n, cnt1[i]);
    need[i] = n;
}

// ---------------------------------------------------------------------------
// Binning by table-size level.

__host__ __device__ __forceinline__ int level_of(int need) {
    if (need <= 0) return -1;   // empty output row
    long long want = static_cast<long long>(need) + need / 4 + 1;
    int lg = kMinLogSlots;
    while ((1ll << lg) < want) ++lg;
    const int L = lg - kMinLogSlots;
    return L < kSharedLevels ? L : kGlobalLevel;
}

__global__ void __launch_bounds__(256) k_bin_levels(int M, const int* need, signed char* level,
                                                     int* counts, int* gmax, int* row_cnt_zero) {
    __shared__ int sc[kLevels + 1];
    __shared__ int smax;
    if (threadIdx.x <= kLevels) sc[threadIdx.x] = 0;
    if (threadIdx.x == 0) smax = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
        const int n = need[i];
        const int L = level_of(n);
        level[i] = static_cast<signed char>(L);
        if (L < 0) {
            atomicAdd(&sc[kLevels], 1);
            if (row_cnt_zero) row_cnt_zero[i] = 0;
        } else {
            atomicAdd(&sc[L], 1);
            if (L == kGlobalLevel) atomicMax(&smax, n);
        }
    }
    __syncthreads();
    if (threadIdx.x <= kLevels && sc[threadIdx.x]) atomicAdd(counts + threadIdx.x, sc[threadIdx.x]);
    if (threadIdx.x == 0 && smax) atomicMax(gmax, smax);
}

// Append every row to its level's list (cursors hold each list's start).
__global__ void __launch_bounds__(256) k_bin_scatter(int M, const signed char* level,
                                                      int* cursors, int* lists) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < M;
    const int L = in ? level[i] : -1;
    // Warp-aggregated append keeps rows of a warp contiguous and ascending.
    const unsigned act = __ballot_sync(0xffffffffu, in && L >= 0);
    if (!(in && L >= 0)) return;
    const unsigned peers = __match_any_sync(act, L);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cursors + L, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    lists[base + __popc(peers & ((1u << lane) - 1u))] = i;
}

// ---------------------------------------------------------------------------
// Row accumulation.

// Left row read from a global CSR (entries [b, e) of ci / v).
struct LeftGlobal {
    const int* ci;
    const void* v;
    int vt;
    int b, e;
    __device__ __forceinline__ int key(int t) const { return __ldg(ci + t); }
    __device__ __forceinline__ double val(int t) const { return load_val(v, vt, t); }
};
// Left row held in shared memory (the forwarded R*A row of the direct
// product, in first-touch order).
struct LeftShared {
    const int* lc;
    const double* lv;
    int b, e;
    __device__ __forceinline__ int key(int t) const { return lc[t]; }
    __device__ __forceinline__ double val(int t) const { return lv[t]; }
};

// Accumulate sum_t left.val(t) * B(left.key(t), :) into the table, in
// ascending t.  ord[n..] receives the slots of new keys in first-touch order.
// Returns the number of distinct keys; `fail` is set (group-uniformly) when
// the table ran out of slots.
template <int G, bool NUM, class Left>
__device__ __forceinline__ int accumulate(const Group<G>& g, const Left& L, const int* b_rp,
                                          const int* b_ci, const void* b_v, int b_vt,
                                          int* keys, double* vals, int* ord, unsigned smask,
                                          int shift, bool& fail) {
    int n = 0;
    for (int t0 = L.b; t0 < L.e; t0 += G) {
        // Prefetch G steps: lane j holds step t0+j's scalar and B row bounds.
        const int t = t0 + g.gl;
        int bb = 0, be = 0;
        double av = 0.0;
        if (t < L.e) {
            const int k = L.key(t);
            if (NUM) av = L.val(t);
            bb = __ldg(b_rp + k);
            be = __ldg(b_rp + k + 1);
        }
        const int cnt = min(G, L.e - t0);
        for (int j = 0; j < cnt; ++j) {
            const int jb = g.bcast(bb, j), je = g.bcast(be, j);
            const double jav = NUM ? g.bcast(av, j) : 0.0;
            for (int e0 = jb; e0 < je; e0 += G) {
                const int e = e0 + g.gl;
                bool is_new = false, bad = false;
                int s = 0;
                if (e < je) {
                    const int c = __ldg(b_ci + e);
                    s = table_insert(keys, smask, shift, c, is_new);
                    if (s < 0) {
                        bad = true;
                    } else if (NUM) {
                        const double bv = load_val(b_v, b_vt, e);
                        vals[s] = __dadd_rn(vals[s], __dmul_rn(bv, jav));
                    }
                }
                const unsigned nb = g.ballot(is_new);
                if (is_new) ord[n + __popc(nb & g.below)] = s;
                n += __popc(nb);
                if (g.ballot(bad)) { fail = true; return n; }
            }
            g.sync();
        }
    }
    return n;
}

// Clear the slots listed in ord[0..n) (and their values).
template <int G, bool NUM>
__device__ __forceinline__ void table_clear(const Group<G>& g, int* keys, double* vals,
                                            const int* ord, int n) {
    for (int i = g.gl; i < n; i += G) {
        const int s = ord[i];
        keys[s] = kEmpty;
        if (NUM) vals[s] = 0.0;
    }
    g.sync();
}

// Clear a whole table (after a failed row, whose ord may be incomplete).
template <int G, bool NUM>
__device__ __forceinline__ void table_clear_all(const Group<G>& g, int* keys, double* vals,
                                                int slots) {
    for (int s = g.gl; s < slots; s += G) {
        keys[s] = kEmpty;
        if (NUM) vals[s] = 0.0;
    }
    g.sync();
}

// Move the row's n entries out of the table into (ck, cv) [ck may alias
// ord: entry i is read then written by the same lane], clearing the slots.
template <int G>
__device__ __forceinline__ void table_extract(const Group<G>& g, int* keys, double* vals,
                                              int* ord, int* ck, double* cv, int n) {
    for (int i = g.gl; i < n; i += G) {
        const int s = ord[i];
        const int k = keys[s];
        const double v = vals[s];
        keys[s] = kEmpty;
        vals[s] = 0.0;
        ck[i] = k;
        cv[i] = v;
    }
    g.sync();
}

constexpr int kRankSortMax = 96;

// Write the n (key, value) pairs in ascending key order to out[base ..].
// Short rows: rank by counting smaller keys.  Long rows: in-place bitonic
// sort over next_pow2(n) entries (capacity >= that), then a coalesced copy.
template <int G>
__device__ __forceinline__ void sorted_write(const Group<G>& g, int* ck, double* cv, int n,
                                             int* out_ci, void* out_v, int out_vt,
                                             long long base) {
    if (n <= kRankSortMax) {
        for (int i = g.gl; i < n; i += G) {
            const int k = ck[i];
            int r = 0;
            for (int j = 0; j < n; ++j) r += ck[j] < k;
            out_ci[base + r] = k;
            store_val(out_v, out_vt, base + r, cv[i]);
        }
        g.sync();
        return;
    }
    const int P2 = static_cast<int>(next_pow2(static_cast<unsigned>(n)));
    for (int i = n + g.gl; i < P2; i += G) ck[i] = INT_MAX;
    g.sync();
    for (int k = 2; k <= P2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = g.gl; i < P2; i += G) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int a = ck[i], b = ck[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        ck[i] = b;
                        ck[ixj] = a;
                        const double t = cv[i];
                        cv[i] = cv[ixj];
                        cv[ixj] = t;
                    }
                }
            }
            g.sync();
        }
    }
    for (int i = g.gl; i < n; i += G) {
        out_ci[base + i] = ck[i];
        store_val(out_v, out_vt, base + i, cv[i]);
    }
    g.sync();
}

// Symbolic write-out of row sizes.
template <int G>
__device__ __forceinline__ void record_count(const Group<G>& g, int* row_cnt, int row, int n) {
    if (g.gl == 0) row_cnt[row] = n;
}

// Output base of a numeric row: the exact row pointer, or a booking in the
// upper-bound space.  Returns -1 when the row cannot be written.
template <int G, int MODE>
__device__ __forceinline__ long long output_base(const Group<G>& g, int row, int n,
                                                 const int* c_rp, unsigned long long* cursor,
                                                 unsigned long long cap, long long* row_off,
                                                 int* row_cnt, unsigned* err) {
    if (MODE == kNumExact) {
        const int b = c_rp[row];
        if (c_rp[row + 1] - b != n) {
            if (g.gl == 0) atomicOr(err, kErrCount);
            return -1;
        }
        return b;
    }
    unsigned long long off = 0;
    if (g.gl == 0) off = atomicAdd(cursor, static_cast<unsigned long long>(n));
    off = g.bcast(off, 0);
    if (off + n > cap) {
        if (g.gl == 0) {
            atomicOr(err, kErrBook);
            row_off[row] = 0;
            row_cnt[row] = 0;
        }
        return -1;
    }
    if (g.gl == 0) {
        row_off[row] = static_cast<long long>(off);
        row_cnt[row] = n;
    }
    return static_cast<long long>(off);
}

// Per-group table region.  Numeric: vals[S] cv[S] keys[S] ord[S] (24 B per
// slot); symbolic: keys[S] ord[S] (8 B per slot).
template <int G, int MODE>
__global__ void __launch_bounds__(256) k_pair_rows(PairArgs p, RowSet rs) {
    constexpr bool NUM = MODE != kSymb;
    extern __shared__ __align__(16) unsigned char smem[];
    const Group<G> g;
    const int gpc = blockDim.x / G;
    const int gid = threadIdx.x / G;
    const int S = rs.slots;
    const unsigned smask = static_cast<unsigned>(S - 1);
    unsigned char* region = rs.gtab
        ? rs.gtab + static_cast<long long>(blockIdx.x * gpc + gid) * rs.gtab_stride
        : smem + static_cast<size_t>(gid) * (NUM ? 24 : 8) * S;
    double* vals = reinterpret_cast<double*>(region);
    double* cv = vals + S;
    int* keys = NUM ? reinterpret_cast<int*>(cv + S) : reinterpret_cast<int*>(region);
    int* ord = keys + S;
    table_clear_all<G, NUM>(g, keys, vals, S);

    for (int it = blockIdx.x * gpc + gid; it < rs.nrows; it += gridDim.x * gpc) {
        const int row = rs.rows[it];
        LeftGlobal L{p.A.ci, p.A.v, p.A.vtype, __ldg(p.A.rp + row), __ldg(p.A.rp + row + 1)};
        bool fail = false;
        const int n = accumulate<G, NUM>(g, L, p.B.rp, p.B.ci, p.B.v, p.B.vtype, keys, vals,
                                         ord, smask, rs.shift, fail);
        if (fail) {
            if (g.gl == 0) atomicOr(p.err, kErrTable);
            table_clear_all<G, NUM>(g, keys, vals, S);
            continue;
        }
        if (!NUM) {
            record_count(g, p.row_cnt, row, n);
            table_clear<G, false>(g, keys, vals, ord, n);
            continue;
        }
        table_extract(g, keys, vals, ord, ord, cv, n);
        const long long base = output_base<G, MODE>(g, row, n, p.c_rp, p.book_cursor,
                                                    p.book_cap, p.row_off, p.row_cnt, p.err);
        if (base < 0) continue;
        if (MODE == kNumExact) sorted_write(g, ord, cv, n, p.c_ci, p.c_v, p.c_vtype, base);
        else sorted_write(g, ord, cv, n, p.ub_ci, p.ub_v, p.c_vtype, base);
    }
}

// Direct R*A*P rows.  Numeric region: vals[S] lv[S] keys[S] ord[S] lc[S]
// (28 B per slot); symbolic: keys[S] ord[S] lc[S] (12 B per slot).
template <int G, int MODE>
__global__ void __launch_bounds__(256) k_direct_rows(DirectArgs p, RowSet rs) {
    constexpr bool NUM = MODE != kSymb;
    extern __shared__ __align__(16) unsigned char smem[];
    const Group<G> g;
    const int gpc = blockDim.x / G;
    const int gid = threadIdx.x / G;
    const int S = rs.slots;
    const unsigned smask = static_cast<unsigned>(S - 1);
    unsigned char* region = rs.gtab
        ? rs.gtab + static_cast<long long>(blockIdx.x * gpc + gid) * rs.gtab_stride
        : smem + static_cast<size_t>(gid) * (NUM ? 28 : 12) * S;
    double* vals = reinterpret_cast<double*>(region);
    double* lv = vals + S;
    int* keys = NUM ? reinterpret_cast<int*>(lv + S) : reinterpret_cast<int*>(region);
    int* ord = keys + S;
    int* lc = ord + S;
    table_clear_all<G, NUM>(g, keys, vals, S);

    for (int it = blockIdx.x * gpc + gid; it < rs.nrows; it += gridDim.x * gpc) {
        const int row = rs.rows[it];
        // Phase 1: the R*A row, first-touch order in ord.
        LeftGlobal L1{p.R.ci, p.R.v, p.R.vtype, __ldg(p.R.rp + row), __ldg(p.R.rp + row + 1)};
        bool fail = false;
        const int n1 = accumulate<G, NUM>(g, L1, p.A.rp, p.A.ci, p.A.v, p.A.vtype, keys, vals,
                                          ord, smask, rs.shift, fail);
        if (fail) {
            if (g.gl == 0) atomicOr(p.err, kErrTable);
            table_clear_all<G, NUM>(g, keys, vals, S);
            continue;
        }
        // Move the R*A row to (lc, lv) in first-touch order; free the table.
        if (NUM) {
            table_extract(g, keys, vals, ord, lc, lv, n1);
        } else {
            for (int i = g.gl; i < n1; i += G) {
                const int s = ord[i];
                lc[i] = keys[s];
                keys[s] = kEmpty;
            }
            g.sync();
        }
        // Phase 2: forward into P.
        LeftShared L2{lc, lv, 0, n1};
        const int n2 = accumulate<G, NUM>(g, L2, p.P.rp, p.P.ci, p.P.v, p.P.vtype, keys, vals,
                                          ord, smask, rs.shift, fail);
        if (fail) {
            if (g.gl == 0) atomicOr(p.err, kErrTable);
            table_clear_all<G, NUM>(g, keys, vals, S);
            continue;
        }
        if (!NUM) {
            record_count(g, p.row_cnt, row, n2);
            if (p.row_cnt1 && g.gl == 0) p.row_cnt1[row] = n1;
            table_clear<G, false>(g, keys, vals, ord, n2);
            continue;
        }
        table_extract(g, keys, vals, ord, ord, lv, n2);
        const long long base = output_base<G, MODE>(g, row, n2, p.c_rp, p.book_cursor,
                                                    p.book_cap, p.row_off, p.row_cnt, p.err);
        if (base < 0) continue;
        if (MODE == kNumExact) sorted_write(g, ord, lv, n2, p.c_ci, p.c_v, p.c_vtype, base);
        else sorted_write(g, ord, lv, n2, p.ub_ci, p.ub_v, p.c_vtype, base);
    }
}

// ---------------------------------------------------------------------------
// Upper-bound flavour: compaction of booked rows into exact CSR
// (replaces mergeRows, code/src/include/SpMMUtilsGeneric.h:364-403).
__global__ void __launch_bounds__(256) k_compact(int M, const int* row_cnt,
                                                  const long long* row_off, const int* ub_ci,
                                                  const void* ub_v, const int* c_rp, int* c_ci,
                                                  void* c_v, int vt) {
    const Group<32> g;
    const int warps = (gridDim.x * blockDim.x) / 32;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < M; row += warps) {
        const int n = row_cnt[row];
        if (!n) continue;
        const long long src = row_off[row];
        const long long dst = c_rp[row];
        for (int i = g.gl; i < n; i += 32) {
            c_ci[dst + i] = ub_ci[src + i];
            if (vt == SP3MM_F32)
                static_cast<float*>(c_v)[dst + i] = static_cast<const float*>(ub_v)[src + i];
            else
                static_cast<double*>(c_v)[dst + i] = static_cast<const double*>(ub_v)[src + i];
        }
    }
}

// ---------------------------------------------------------------------------
// Conversions between the host ABI (64-bit, OFF_F based) and device CSR.

__global__ void k_narrow_rowptr(long long M, long long nnz, const unsigned long long* src,
                                int off, int* dst, unsigned* err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= M;
         i += (long long)gridDim.x * blockDim.x) {
        const long long v = static_cast<long long>(src[i]) - off;
        bool bad = v < 0 || v > nnz;
        if (i == 0) bad |= v != 0;
        if (i == M) bad |= v != nnz;
        if (i > 0) bad |= static_cast<long long>(src[i - 1]) - off > v;
        if (bad) atomicOr(err, kErrInput);
        dst[i] = static_cast<int>(bad ? 0 : v);
    }
}

// Warp per row: narrow columns, check range and strict ascending order.
__global__ void __launch_bounds__(256) k_narrow_cols(long long M, long long N, const int* rp,
                                                      const unsigned long long* src, int off,
                                                      int* dst, int* max_row, unsigned* err) {
    const int lane = threadIdx.x & 31;
    const long long warps = (gridDim.x * (long long)blockDim.x) / 32;
    int my_max = 0;
    for (long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32; row < M;
         row += warps) {
        const int b = rp[row], e = rp[row + 1];
        my_max = max(my_max, e - b);
        for (int j = b + lane; j < e; j += 32) {
            const long long c = static_cast<long long>(src[j]) - off;
            bool bad = c < 0 || c >= N;
            if (j > b) bad |= static_cast<long long>(src[j - 1]) - off >= c;
            if (bad) atomicOr(err, kErrInput);
            dst[j] = static_cast<int>(bad ? 0 : c);
        }
    }
    if (lane == 0 && my_max) atomicMax(max_row, my_max);
}

__global__ void k_widen(long long n, const int* src, int off, unsigned long long* dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = static_cast<unsigned long long>(static_cast<long long>(src[i]) + off);
}

__global__ void k_convert_values(long long n, const void* src, int st_, void* dst, int dt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        store_val(dst, dt, i, load_val(src, st_, i));
}

// Validate a device-side int32 CSR: row_ptr monotone from 0, columns in
// range and strictly ascending within rows.
__global__ void __launch_bounds__(256) k_validate_i32(int M, int N, const int* rp,
                                                       const int* ci, int* max_row,
                                                       unsigned* err) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) / 32;
    int my_max = 0;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < M; row += warps) {
        const int b = rp[row], e = rp[row + 1];
        if (e < b || (row == 0 && b != 0)) {
            if (lane == 0) atomicOr(err, kErrInput);
            continue;
        }
        my_max = max(my_max, e - b);
        for (int j = b + lane; j < e; j += 32) {
            const int c = ci[j];
            bool bad = c < 0 || c >= N;
            if (j > b) bad |= ci[j - 1] >= c;
            if (bad) atomicOr(err, kErrInput);
        }
    }
    if (lane == 0 && my_max) atomicMax(max_row, my_max);
}

// ---------------------------------------------------------------------------
// Transpose.

__global__ void k_col_counts(long long nnz, const int* ci, int* counts) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnz;
         i += (long long)gridDim.x * blockDim.x)
        atomicAdd(counts + ci[i], 1);
}

__global__ void __launch_bounds__(256) k_transpose_scatter(CsrView A, const int* t_rp,
                                                            int* cursor, int* t_ci, void* t_v) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) / 32;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < A.M; row += warps) {
        const int b = A.rp[row], e = A.rp[row + 1];
        for (int j = b + lane; j < e; j += 32) {
            const int c = A.ci[j];
            const int pos = t_rp[c] + atomicAdd(cursor + c, 1);
            t_ci[pos] = row;
            if (A.vtype == SP3MM_F32)
                static_cast<float*>(t_v)[pos] = static_cast<const float*>(A.v)[j];
            else
                static_cast<double*>(t_v)[pos] = static_cast<const double*>(A.v)[j];
        }
    }
}

// Sort each row's (col, val) by col.  Warp per row; short rows by rank in
// registers, long rows by an odd-even transposition over global memory.
__global__ void __launch_bounds__(256) k_sort_rows(int M, const int* rp, int* ci, void* v,
                                                    int vt) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) / 32;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < M; row += warps) {
        const int b = rp[row], e = rp[row + 1];
        const int n = e - b;
        if (n <= 1) continue;
        if (n <= 32) {
            const bool in = lane < n;
            const int k = in ? ci[b + lane] : INT_MAX;
            const double x = in ? load_val(v, vt, b + lane) : 0.0;
            int r = 0;
            for (int j = 0; j < n; ++j) r += __shfl_sync(0xffffffffu, k, j) < k;
            __syncwarp();
            if (in) {
                ci[b + r] = k;
                store_val(v, vt, b + r, x);
            }
            __syncwarp();
            continue;
        }
        for (int phase = 0; phase < n; ++phase) {
            for (int i = b + (phase & 1) + 2 * lane; i + 1 < e; i += 64) {
                const int a0 = ci[i], a1 = ci[i + 1];
                if (a0 > a1) {
                    ci[i] = a1;
                    ci[i + 1] = a0;
                    const double x0 = load_val(v, vt, i), x1 = load_val(v, vt, i + 1);
                    store_val(v, vt, i, x1);
                    store_val(v, vt, i + 1, x0);
                }
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// 2D column-partition upper bounds (code/src/include/SpMMUtilsGeneric.h:146-174).
__global__ void k_colparts_ub(CsrView A, int gridCols, const long long* off, long long* out,
                              unsigned long long* total) {
    unsigned long long mine = 0;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         x < static_cast<long long>(A.M) * gridCols; x += (long long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(x / gridCols);
        const int gc = static_cast<int>(x % gridCols);
        long long s = 0;
        for (int jj = A.rp[r]; jj < A.rp[r + 1]; ++jj) {
            const long long id = static_cast<long long>(A.ci[jj]) * gridCols + gc;
            s += off[id + 1] - off[id];
        }
        out[x] = s;
        mine += static_cast<unsigned long long>(s);
    }
    if (mine) atomicAdd(total, mine);
}

// ---------------------------------------------------------------------------
// Host launchers.

static inline int grid_for(long long work, int block, int cap = 148 * 16) {
    long long g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<int>(g);
}

int choose_group(double mean) {
    if (mean <= 4.0) return 4;
    if (mean <= 8.0) return 8;
    if (mean <= 16.0) return 16;
    return 32;
}

LevelPlan plan_level(int level, bool direct, int mode, int G, size_t budget) {
    LevelPlan pl{};
    pl.slots = 32 << level;
    const size_t per_group = static_cast<size_t>(bytes_per_slot(direct, mode)) * pl.slots;
    if (level >= kSharedLevels || per_group > budget) {
        pl.global = true;
        pl.G = 32;
        pl.groups_per_cta = 8;
        pl.smem_bytes = 0;
        return pl;
    }
    // Large tables use a whole warp per row.
    int g = G;
    if (pl.slots >= 1024 && g < 32) g = 32;
    if (pl.slots >= 512 && g < 16) g = 16;
    const int per_warp = 32 / g;
    int warps = static_cast<int>(budget / (per_group * per_warp));
    if (warps < 1) {
        // Fewer groups than a warp holds: go to one full-warp group.
        g = 32;
        warps = static_cast<int>(budget / per_group);
        if (warps < 1) {
            pl.global = true;
            pl.G = 32;
            pl.groups_per_cta = 8;
            pl.smem_bytes = 0;
            return pl;
        }
    }
    if (warps > 8) warps = 8;
    pl.G = g;
    pl.groups_per_cta = warps * (32 / g);
    pl.smem_bytes = per_group * pl.groups_per_cta;
    pl.global = false;
    return pl;
}

void launch_pair_bounds(const CsrView& A, const CsrView& B, int* need,
                        unsigned long long* total, cudaStream_t st) {
    if (A.M == 0) return;
    const int grid = grid_for(static_cast<long long>(A.M) * 8, 256);
    k_pair_bounds<8><<<grid, 256, 0, st>>>(A, B, need, total);
    counted();
}

void launch_direct_bounds(const CsrView& R, const CsrView& A, const CsrView& P, int* need,
                          unsigned long long* total, cudaStream_t st) {
    if (R.M == 0) return;
    const int grid = grid_for(static_cast<long long>(R.M) * 8, 256);
    k_direct_bounds<8><<<grid, 256, 0, st>>>(R, A, P, need, total);
    counted();
}

void launch_need_from_counts(int M, const int* cnt, const int* cnt1, int* need,
                             cudaStream_t st) {
    if (M == 0) return;
    k_need_from_counts<<<(M + 255) / 256, 256, 0, st>>>(M, cnt, cnt1, need);
    counted();
}

void launch_bin_levels(int M, const int* need, signed char* level, int* counts, int* gmax,
                       int* row_cnt_zero, cudaStream_t st) {
    if (M == 0) return;
    k_bin_levels<<<grid_for(M, 256), 256, 0, st>>>(M, need, level, counts, gmax,
                                                    row_cnt_zero);
    counted();
}

void launch_bin_scatter(int M, const signed char* level, int* cursors, int* lists,
                        cudaStream_t st) {
    if (M == 0) return;
    k_bin_scatter<<<(M + 255) / 256, 256, 0, st>>>(M, level, cursors, lists);
    counted();
}

template <template <int, int> class K>
struct Dummy {};

#define SP3MM_DISPATCH_G(G, BODY) \
    switch (G) {                 \
        case 4: { constexpr int GG = 4; BODY; } break;   \
        case 8: { constexpr int GG = 8; BODY; } break;   \
        case 16: { constexpr int GG = 16; BODY; } break; \
        default: { constexpr int GG = 32; BODY; } break; \
    }

template <int G, int MODE>
static void pair_rows_g(const PairArgs& a, const LevelPlan& pl, const RowSet& rs, int grid,
                        cudaStream_t st) {
    auto k = k_pair_rows<G, MODE>;
    if (pl.smem_bytes > 48 * 1024)
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(pl.smem_bytes));
    k<<<grid, pl.groups_per_cta * G, pl.smem_bytes, st>>>(a, rs);
    counted();
}

template <int G, int MODE>
static void direct_rows_g(const DirectArgs& a, const LevelPlan& pl, const RowSet& rs, int grid,
                          cudaStream_t st) {
    auto k = k_direct_rows<G, MODE>;
    if (pl.smem_bytes > 48 * 1024)
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(pl.smem_bytes));
    k<<<grid, pl.groups_per_cta * G, pl.smem_bytes, st>>>(a, rs);
    counted();
}

void launch_pair_rows(const PairArgs& a, int mode, const LevelPlan& pl, const RowSet& rs,
                      int grid, cudaStream_t st) {
    if (rs.nrows == 0) return;
    switch (mode) {
        case kSymb: SP3MM_DISPATCH_G(pl.G, (pair_rows_g<GG, kSymb>(a, pl, rs, grid, st))); break;
        case kNumExact:
            SP3MM_DISPATCH_G(pl.G, (pair_rows_g<GG, kNumExact>(a, pl, rs, grid, st)));
            break;
        default: SP3MM_DISPATCH_G(pl.G, (pair_rows_g<GG, kNumBook>(a, pl, rs, grid, st))); break;
    }
}

void launch_direct_rows(const DirectArgs& a, int mode, const LevelPlan& pl, const RowSet& rs,
                        int grid, cudaStream_t st) {
    if (rs.nrows == 0) return;
    switch (mode) {
        case kSymb:
            SP3MM_DISPATCH_G(pl.G, (direct_rows_g<GG, kSymb>(a, pl, rs, grid, st)));
            break;
        case kNumExact:
            SP3MM_DISPATCH_G(pl.G, (direct_rows_g<GG, kNumExact>(a, pl, rs, grid, st)));
            break;
        default:
            SP3MM_DISPATCH_G(pl.G, (direct_rows_g<GG, kNumBook>(a, pl, rs, grid, st)));
            break;
    }
}

size_t row_kernel_max_smem() { return 110 * 1024; }

void launch_compact(int M, const int* row_cnt, const long long* row_off, const int* ub_ci,
                    const void* ub_v, const int* c_rp, int* c_ci, void* c_v, int vt,
                    cudaStream_t st) {
    if (M == 0) return;
    k_compact<<<grid_for(static_cast<long long>(M) * 32, 256), 256, 0, st>>>(
        M, row_cnt, row_off, ub_ci, ub_v, c_rp, c_ci, c_v, vt);
    counted();
}

size_t scan_temp_bytes(int M) {
    size_t bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, bytes, static_cast<const int*>(nullptr),
                                  static_cast<int*>(nullptr), M > 0 ? M : 1);
    return bytes;
}

void launch_scan(int M, const int* cnt, int* row_ptr, void* temp, size_t temp_bytes,
                 cudaStream_t st) {
    cudaMemsetAsync(row_ptr, 0, sizeof(int), st);
    if (M == 0) return;
    cub::DeviceScan::InclusiveSum(temp, temp_bytes, cnt, row_ptr + 1, M, st);
    counted();
}

void launch_narrow_rowptr(long long M, long long nnz, const unsigned long long* src, int off,
                          int* dst, unsigned* err, cudaStream_t st) {
    k_narrow_rowptr<<<grid_for(M + 1, 256), 256, 0, st>>>(M, nnz, src, off, dst, err);
    counted();
}

void launch_narrow_cols(long long M, long long N, const int* rp, const unsigned long long* src,
                        int off, int* dst, int* max_row, unsigned* err, cudaStream_t st) {
    if (M == 0) return;
    k_narrow_cols<<<grid_for(M * 32, 256), 256, 0, st>>>(M, N, rp, src, off, dst, max_row,
                                                         err);
    counted();
}

void launch_widen(long long n, const int* src, int off, unsigned long long* dst,
                  cudaStream_t st) {
    if (n == 0) return;
    k_widen<<<grid_for(n, 256), 256, 0, st>>>(n, src, off, dst);
    counted();
}

void launch_convert_values(long long n, const void* src, int src_type, void* dst, int dst_type,
                           cudaStream_t st) {
    if (n == 0) return;
    k_convert_values<<<grid_for(n, 256), 256, 0, st>>>(n, src, src_type, dst, dst_type);
    counted();
}

void launch_validate_i32(int M, int N, const int* rp, const int* ci, int* max_row,
                         unsigned* err, cudaStream_t st) {
    if (M == 0) return;
    k_validate_i32<<<grid_for(static_cast<long long>(M) * 32, 256), 256, 0, st>>>(
        M, N, rp, ci, max_row, err);
    counted();
}

void launch_col_counts(long long nnz, const int* ci, int* counts, cudaStream_t st) {
    if (nnz == 0) return;
    k_col_counts<<<grid_for(nnz, 256), 256, 0, st>>>(nnz, ci, counts);
    counted();
}

void launch_transpose_scatter(const CsrView& A, const int* t_rp, int* cursor, int* t_ci,
                              void* t_v, cudaStream_t st) {
    if (A.M == 0) return;
    k_transpose_scatter<<<grid_for(static_cast<long long>(A.M) * 32, 256), 256, 0, st>>>(
        A, t_rp, cursor, t_ci, t_v);
    counted();
}

void launch_sort_rows(int M, const int* rp, int* ci, void* v, int vt, int max_row,
                      cudaStream_t st) {
    if (M == 0 || max_row <= 1) return;
    k_sort_rows<<<grid_for(static_cast<long long>(M) * 32, 256), 256, 0, st>>>(M, rp, ci, v,
                                                                              vt);
    counted();
}

void launch_colparts_ub(const CsrView& A, const CsrView& B, int gridCols,
                        const long long* bColOffsets, int off, long long* out,
                        unsigned long long* total, cudaStream_t st) {
    (void)B;
    (void)off;
    const long long work = static_cast<long long>(A.M) * gridCols;
    if (work == 0) return;
    k_colparts_ub<<<grid_for(work, 256), 256, 0, st>>>(A, gridCols, bColOffsets, out, total);
    counted();
}

}  // namespace sp3mm
