// rows.cuh -- per-row accumulation kernels of the Sp3MM products (sm_100a).
//
// One group of G lanes owns one output row and its hash tables; a warp holds
// 32/G groups.  The lanes walk the left row one step at a time; within a step
// they cover the selected right row, whose columns are distinct, so every
// output entry receives its contributions in ascending left-row position --
// the order of the reference's scSparseVectMul_ loop
// (code/src/include/SpMMUtilsGeneric.h:39-55) -- with no value atomics, and
// the values are bit-identical to the reference's.  New keys of a step are
// ranked by ballot + popc in lane order, which reproduces the first-touch
// order in which the reference's index map appends them
// (code/src/include/sparseMatrix.h:85-104); the direct product forwards the
// R*A row into P in that order (code/src/Sp3MM_CSR_OMP_UB_Generic.c:542-545).
//
// Warp-synchronous execution: every loop that contains a warp collective runs
// to a warp-uniform bound (the maximum over the warp's groups) with per-group
// predicates, and every vote / shuffle / barrier names the full warp, so the
// groups of a warp issue together.
//
// Latency: the row pointers of the right operand are loaded two chunks of G
// steps ahead and the right-row entries one chunk ahead, into two register
// buffers used in turn.
//
// Value types are template parameters (TV: storage type of every input, TO:
// of the output; accumulation is always FP64), and the tables live in shared
// memory except in the GT (global-table) instantiation used for very long
// rows, so the compiler emits 32-bit shared addressing in the common case.
//
// Table sizes are runtime powers of two.  A row whose distinct-key count
// passes the table's load limit stops inserting, clears its slots and is
// appended to a retry list, which a second launch processes with tables
// sized from a proven bound; results do not depend on the table size.
#pragma once

#include <climits>

#include "kernels.cuh"
#include "sp3mm_internal.cuh"

namespace sp3mm {

constexpr unsigned kFull = 0xffffffffu;

template <typename T> __device__ __forceinline__ double ldv(const T* p, long long i) {
    return static_cast<double>(__ldg(p + i));
}
template <typename T> __device__ __forceinline__ void stv(T* p, long long i, double v) {
    p[i] = static_cast<T>(v);
}

template <int G> __device__ __forceinline__ int wshfl(int v, int j) {
    return __shfl_sync(kFull, v, j, G);
}
template <int G> __device__ __forceinline__ double wshfl(double v, int j) {
    return __shfl_sync(kFull, v, j, G);
}

// Left row in global memory: entries [b, b+n) of (ci, v).
template <typename TV>
struct LeftG {
    const int* ci;
    const TV* v;
    int b;
    __device__ __forceinline__ int key(int t) const { return __ldg(ci + b + t); }
    __device__ __forceinline__ double val(int t) const { return ldv(v, b + t); }
};
// Left row held in a table, read in the order of `ord` (first touch).
struct LeftT {
    const int* keys;
    const double* vals;
    const int* ord;
    __device__ __forceinline__ int key(int t) const { return keys[ord[t]]; }
    __device__ __forceinline__ double val(int t) const { return vals[ord[t]]; }
};

// Distinct keys a table of S slots accepts before the row is retried: at
// most G keys arrive per sub-step and a group stops inserting once it passed
// the limit, so the table never fills; the load factor stays <= 7/8.
__host__ __device__ __forceinline__ int table_limit(int S, int G) {
    const int a = S - G - 1, b = (7 * S) / 8;
    return a < b ? a : b;
}

template <bool NUM>
struct Acc {
    int* keys;
    double* vals;
    int* ord;
    unsigned smask;
    int shift;
    int limit;
};

// One sub-step for the whole warp: lanes with `act` add bv*s into key c.
// `live` (group-uniform) turns false once the group passed its table limit.
template <int G, bool NUM>
__device__ __forceinline__ void sub_step(const Group<G>& g, const Acc<NUM>& T, bool act, int c,
                                         double bv, double s, int& nk, bool& live) {
    act = act && live;
    unsigned slot = hash_slot(c, T.shift);
    const int k0 = act ? T.keys[slot] : c;   // idle lanes count as hits
    bool is_new = false;
    if (k0 != c) {
        // Miss: probe until the key or an empty slot (one always exists:
        // the table never passes its limit).  Bounded by the table size.
        int k = k0;
        for (unsigned probe = 0; probe <= T.smask; ++probe) {
            if (k == kEmpty) {
                const int old = atomicCAS(T.keys + slot, kEmpty, c);
                if (old == kEmpty) {
                    is_new = true;
                    break;
                }
                k = old;
                if (k == c) break;
            }
            slot = (slot + 1) & T.smask;
            k = T.keys[slot];
            if (k == c) break;
        }
    }
    if (NUM && act) T.vals[slot] = __dadd_rn(T.vals[slot], __dmul_rn(bv, s));
    const unsigned nb = __ballot_sync(kFull, is_new);
    if (is_new) T.ord[nk + __popc(nb & g.below)] = static_cast<int>(slot);
    nk += __popc(nb & g.mask);
    live = nk <= T.limit;
}

// Accumulate sum_{t<n} L.val(t) * B(L.key(t), :) in ascending t; n is this
// group's left-row length (0 for an idle group).  Every lane of the warp
// must call it.  Returns the distinct-key count; `fail` when the group
// passed its table limit.  b_long: some right row is longer than EP*G.
template <int G, int EP, bool NUM, typename TB, class Left>
__device__ __forceinline__ int accumulate(const Group<G>& g, const Left& L, int n,
                                          const int* __restrict__ b_rp,
                                          const int* __restrict__ b_ci, const TB* __restrict__ b_v,
                                          bool b_long, const Acc<NUM>& T, bool& fail) {
    int nk = 0;
    bool live = n > 0;
    const int nmax = __reduce_max_sync(kFull, n);
    if (nmax == 0) return 0;

    // Row pointers and scalar of step t0 + gl (lane j <-> step t0 + j).
    auto load_ptrs = [&](int t0, int& pb, int& pe, double& ps) {
        const int t = t0 + g.gl;
        pb = 0;
        pe = 0;
        ps = 0.0;
        if (t < n) {
            const int k = L.key(t);
            if (NUM) ps = L.val(t);
            pb = __ldg(b_rp + k);
            pe = __ldg(b_rp + k + 1);
        }
    };
    constexpr int EPA = EP > 0 ? EP : 1;   // array extent (EP == 0: no prefetch)
    // Entries of a chunk: [j][m] = entry gl + m*G of step j.
    auto load_entries = [&](int pb, int pe, int (&ec)[G][EPA], double (&ev)[G][EPA]) {
        if constexpr (EP > 0) {
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const int jb = wshfl<G>(pb, j), je = wshfl<G>(pe, j);
#pragma unroll
                for (int m = 0; m < EP; ++m) {
                    const int e = jb + m * G + g.gl;
                    ec[j][m] = -1;
                    ev[j][m] = 0.0;
                    if (e < je) {
                        ec[j][m] = __ldg(b_ci + e);
                        if (NUM) ev[j][m] = ldv(b_v, e);
                    }
                }
            }
        }
    };
    // Steps [base, base+G) from the chunk's pointers (pb, pe, ps) and
    // prefetched entries (ec, ev).
    auto run_chunk = [&](int base, int pb, int pe, double ps, const int (&ec)[G][EPA],
                         const double (&ev)[G][EPA]) {
#pragma unroll
        for (int j = 0; j < G; ++j) {
            if (base + j < nmax) {
                const int jb = wshfl<G>(pb, j), je = wshfl<G>(pe, j);
                const double js = NUM ? wshfl<G>(ps, j) : 0.0;
                if constexpr (EP > 0) {
#pragma unroll
                    for (int m = 0; m < EP; ++m) {
                        if (m == 0 || __any_sync(kFull, jb + m * G < je)) {
                            const bool act = jb + m * G + g.gl < je;
                            sub_step<G, NUM>(g, T, act, ec[j][m], ev[j][m], js, nk, live);
                        }
                    }
                }
                if (EP == 0 || b_long) {
                    // Entries not prefetched are loaded in place.
                    for (int e0 = jb + EP * G; __any_sync(kFull, e0 < je); e0 += G) {
                        const int e = e0 + g.gl;
                        const bool act = e < je;
                        int c = -1;
                        double bv = 0.0;
                        if (act) {
                            c = __ldg(b_ci + e);
                            if (NUM) bv = ldv(b_v, e);
                        }
                        sub_step<G, NUM>(g, T, act, c, bv, js, nk, live);
                    }
                }
                __syncwarp();
            }
        }
    };

    int ecA[G][EPA], ecB[G][EPA];
    double evA[G][EPA], evB[G][EPA];
    int pbA, peA, pbB, peB, pbC, peC;
    double psA, psB, psC;
    load_ptrs(0, pbA, peA, psA);
    load_ptrs(G, pbB, peB, psB);
    load_entries(pbA, peA, ecA, evA);
    // Two chunks per iteration: buffers A and B alternate without copies.
    for (int base = 0; base < nmax; base += 2 * G) {
        load_entries(pbB, peB, ecB, evB);
        load_ptrs(base + 2 * G, pbC, peC, psC);
        run_chunk(base, pbA, peA, psA, ecA, evA);
        if (base + G >= nmax) break;
        load_entries(pbC, peC, ecA, evA);
        load_ptrs(base + 3 * G, pbA, peA, psA);
        run_chunk(base + G, pbB, peB, psB, ecB, evB);
        pbB = pbA;
        peB = peA;
        psB = psA;
        pbA = pbC;
        peA = peC;
        psA = psC;
    }
    fail = n > 0 && !live;
    return nk;
}

// Clear the slots listed in ord[0..n).
template <int G, bool NUM>
__device__ __forceinline__ void clear_listed(const Group<G>& g, const Acc<NUM>& T, int n) {
    for (int i = g.gl; i < n; i += G) {
        const int s = T.ord[i];
        T.keys[s] = kEmpty;
        if (NUM) T.vals[s] = 0.0;
    }
}

template <int G, bool NUM>
__device__ __forceinline__ void clear_all(const Group<G>& g, int* keys, double* vals, int S) {
    for (int s = g.gl; s < S; s += G) {
        keys[s] = kEmpty;
        if (NUM) vals[s] = 0.0;
    }
}

// Move the n listed entries of T into (ck, cv)[0..n), clearing T.
template <int G>
__device__ __forceinline__ void extract(const Group<G>& g, const Acc<true>& T, int n, int* ck,
                                        double* cv) {
    for (int i = g.gl; i < n; i += G) {
        const int s = T.ord[i];
        ck[i] = T.keys[s];
        cv[i] = T.vals[s];
        T.keys[s] = kEmpty;
        T.vals[s] = 0.0;
    }
}

// Write (ck, cv)[0..n) in ascending key order to out[base..] for every group
// with base >= 0 (n = 0 for idle groups).  Every lane of the warp must call
// it.  Rows up to 64 entries: rank sort with each lane's keys cached in
// registers.  Longer rows: bitonic sort in place (ck/cv hold
// next_pow2(max n) slots), then a linear copy.  On return ck / cv are reset
// to kEmpty / 0 where they were used.
template <int G, typename TO>
__device__ __forceinline__ void sorted_write(const Group<G>& g, int* ck, double* cv, int n,
                                             int* out_ci, TO* out_v, long long base) {
    const bool writes = base >= 0;
    const int nmax = __reduce_max_sync(kFull, n);
    if (nmax == 0) return;
    constexpr int RM = 64 / G;
    if (nmax <= 64) {
        int mk[RM], rk[RM];
#pragma unroll
        for (int m = 0; m < RM; ++m) {
            const int i = g.gl + m * G;
            mk[m] = i < n ? ck[i] : INT_MAX;
            rk[m] = 0;
        }
        for (int j = 0; j < nmax; ++j) {
            const int kj = j < n ? ck[j] : INT_MAX;
#pragma unroll
            for (int m = 0; m < RM; ++m) rk[m] += kj < mk[m];
        }
#pragma unroll
        for (int m = 0; m < RM; ++m) {
            const int i = g.gl + m * G;
            if (i < n) {
                if (writes) {
                    out_ci[base + rk[m]] = mk[m];
                    stv(out_v, base + rk[m], cv[i]);
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < RM; ++m) {
            const int i = g.gl + m * G;
            if (i < n) {
                ck[i] = kEmpty;
                cv[i] = 0.0;
            }
        }
        __syncwarp();
        return;
    }
    const int P2 = static_cast<int>(next_pow2(static_cast<unsigned>(nmax)));
    for (int i = n + g.gl; i < P2; i += G) ck[i] = INT_MAX;
    __syncwarp();
    for (int k = 2; k <= P2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = g.gl; i < P2; i += G) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int a = ck[i], b = ck[ixj];
                    if ((a > b) == ((i & k) == 0)) {
                        ck[i] = b;
                        ck[ixj] = a;
                        const double t = cv[i];
                        cv[i] = cv[ixj];
                        cv[ixj] = t;
                    }
                }
            }
            __syncwarp();
        }
    }
    if (writes) {
        for (int i = g.gl; i < n; i += G) {
            out_ci[base + i] = ck[i];
            stv(out_v, base + i, cv[i]);
        }
    }
    __syncwarp();
    for (int i = g.gl; i < P2; i += G) {
        ck[i] = kEmpty;
        cv[i] = 0.0;
    }
    __syncwarp();
}

// Warp-aggregated booking of n (group leaders contribute) in the upper-bound
// space: one atomic per warp.  Returns the group's offset, or -1 when the
// space is exhausted or the group does not contribute.  Every lane of the
// warp must call it.
template <int G>
__device__ __forceinline__ long long book_warp(const Group<G>& g, bool contributes, int n,
                                               unsigned long long* cursor,
                                               unsigned long long cap, unsigned* err) {
    const int lane = threadIdx.x & 31;
    const unsigned long long mine = (contributes && g.gl == 0) ? static_cast<unsigned long long>(n) : 0ull;
    unsigned long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += v;
    }
    const unsigned long long total = __shfl_sync(kFull, incl, 31);
    unsigned long long wbase = 0;
    if (lane == 0 && total) wbase = atomicAdd(cursor, total);
    wbase = __shfl_sync(kFull, wbase, 0);
    if (wbase + total > cap) {
        if (lane == 0 && total) atomicOr(err, kErrBook);
        return -1;
    }
    const unsigned long long off = __shfl_sync(kFull, wbase + incl - mine, 0, G);
    return contributes ? static_cast<long long>(off) : -1;
}

template <int G>
__device__ __forceinline__ void retry_row(const Group<G>& g, const RowParams& p, int row) {
    if (g.gl != 0) return;
    if (p.retry_rows) {
        const int pos = atomicAdd(p.retry_count, 1);
        p.retry_rows[pos] = row;
    } else {
        atomicOr(p.err, kErrTable);
    }
}

// Output offset of an accumulated row (all lanes of the warp call it):
// booking in the upper-bound space, or the exact row pointer.
template <int G, int MODE>
__device__ __forceinline__ long long out_base(const Group<G>& g, const RowParams& p, bool ok,
                                              int row, int n) {
    if (MODE == kNumBook) {
        const long long b = book_warp(g, ok, n, p.cursor, p.cap, p.err);
        if (ok && b >= 0 && g.gl == 0) {
            p.row_off[row] = b;
            p.row_cnt[row] = n;
        }
        return b;
    }
    if (!ok) return -1;
    const long long b = p.c_rp[row];
    if (p.c_rp[row + 1] - b != n) {
        if (g.gl == 0) atomicOr(p.err, kErrCount);
        return -1;
    }
    return b;
}

// Per-group table region: shared memory, or the group's slice of gtab.
template <bool GT>
__device__ __forceinline__ unsigned char* group_region(unsigned char* smem, const RowParams& p,
                                                       int gid, int gpc, long long bytes) {
    if constexpr (GT) {
        return p.gtab + (static_cast<long long>(blockIdx.x) * gpc + gid) * p.gstride;
    } else {
        (void)p;
        return smem + static_cast<long long>(gid) * bytes;
    }
}

template <int G> constexpr int prefetch_depth() { return G <= 4 ? 2 : (G <= 8 ? 1 : 0); }

// Direct R*A*P.  Per-group region (numeric): vals1[S1] vals2[S2] keys1[S1]
// keys2[S2] ord1[S1] ord2[S2]; symbolic: keys1 keys2 ord1 ord2.
template <int G, int MODE, typename TV, typename TO, bool GT>
__global__ void __launch_bounds__(256) k_direct_rows(DirectRowArgs a, RowParams p) {
    constexpr bool NUM = MODE != kSymb;
    constexpr int EP = prefetch_depth<G>();
    extern __shared__ __align__(16) unsigned char smem[];
    const Group<G> g;
    const int gpc = blockDim.x / G;
    const int gid = threadIdx.x / G;
    const int S1 = p.S1, S2 = p.S2;
    const long long bytes = static_cast<long long>(NUM ? 16 : 8) * (S1 + S2);
    unsigned char* region = group_region<GT>(smem, p, gid, gpc, bytes);
    double* vals1 = reinterpret_cast<double*>(region);
    double* vals2 = vals1 + S1;
    int* keys1 = NUM ? reinterpret_cast<int*>(vals2 + S2) : reinterpret_cast<int*>(region);
    int* keys2 = keys1 + S1;
    int* ord1 = keys2 + S2;
    int* ord2 = ord1 + S1;
    const Acc<NUM> T1{keys1, vals1, ord1, static_cast<unsigned>(S1 - 1),
                      32 - ilog2_pow2(static_cast<unsigned>(S1)), table_limit(S1, G)};
    const Acc<NUM> T2{keys2, vals2, ord2, static_cast<unsigned>(S2 - 1),
                      32 - ilog2_pow2(static_cast<unsigned>(S2)), table_limit(S2, G)};
    clear_all<G, NUM>(g, keys1, vals1, S1);
    clear_all<G, NUM>(g, keys2, vals2, S2);
    __syncwarp();
    const TV* rv = static_cast<const TV*>(a.R.v);
    const TV* av = static_cast<const TV*>(a.A.v);
    const TV* pv = static_cast<const TV*>(a.P.v);
    const bool a_long = p.a_long, p_long = p.b_long;

    const int gpw = 32 / G;
    const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
    const long long wid = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (long long wbase = wid * gpw; wbase < p.nrows; wbase += warps * gpw) {
        const long long it = wbase + ((threadIdx.x & 31) / G);
        const bool has = it < p.nrows;
        const int row = has ? p.rows[it] : 0;
        int rb = 0, rlen = 0;
        if (has) {
            rb = __ldg(a.R.rp + row);
            rlen = __ldg(a.R.rp + row + 1) - rb;
        }
        // Phase 1: the R*A row, first-touch order in ord1.
        bool fail1 = false, fail2 = false;
        const LeftG<TV> L1{a.R.ci, rv, rb};
        const int n1 = accumulate<G, EP, NUM>(g, L1, rlen, a.A.rp, a.A.ci, av, a_long, T1, fail1);
        __syncwarp();
        // Phase 2: forward the R*A row into P in first-touch order.
        const LeftT L2{keys1, vals1, ord1};
        const int n2 = accumulate<G, EP, NUM>(g, L2, fail1 ? 0 : n1, a.P.rp, a.P.ci, pv, p_long,
                                              T2, fail2);
        __syncwarp();
        clear_listed<G, NUM>(g, T1, n1);
        __syncwarp();
        const bool fail = fail1 || fail2;
        const bool ok = has && !fail;
        if (fail) {
            clear_listed<G, NUM>(g, T2, n2);
            retry_row(g, p, row);
        } else if (ok) {
            if constexpr (NUM) {
                extract(g, T2, n2, keys1, vals1);   // H1 is free: sort scratch
            } else {
                if (g.gl == 0) {
                    p.row_cnt[row] = n2;
                    if (p.row_cnt1) p.row_cnt1[row] = n1;
                }
                clear_listed<G, NUM>(g, T2, n2);
            }
        }
        __syncwarp();
        if constexpr (NUM) {
            const long long base = out_base<G, MODE>(g, p, ok, row, n2);
            int* oc = MODE == kNumBook ? p.ub_ci : p.c_ci;
            TO* ov = static_cast<TO*>(MODE == kNumBook ? p.ub_v : p.c_v);
            sorted_write<G, TO>(g, keys1, vals1, ok ? n2 : 0, oc, ov, base);
        }
    }
}

// Pair-wise A*B.  Region (numeric): vals[S] cv[S] keys[S] ck[S] ord[S];
// symbolic: keys[S] ord[S].
template <int G, int MODE, typename TV, typename TO, bool GT>
__global__ void __launch_bounds__(256) k_pair_rows(PairRowArgs a, RowParams p) {
    constexpr bool NUM = MODE != kSymb;
    constexpr int EP = prefetch_depth<G>();
    extern __shared__ __align__(16) unsigned char smem[];
    const Group<G> g;
    const int gpc = blockDim.x / G;
    const int gid = threadIdx.x / G;
    const int S = p.S1;
    const long long bytes = static_cast<long long>(NUM ? 28 : 8) * S;
    unsigned char* region = group_region<GT>(smem, p, gid, gpc, bytes);
    double* vals = reinterpret_cast<double*>(region);
    double* cv = vals + S;
    int* keys = NUM ? reinterpret_cast<int*>(cv + S) : reinterpret_cast<int*>(region);
    int* ck = NUM ? keys + S : nullptr;
    int* ord = NUM ? ck + S : keys + S;
    const Acc<NUM> T{keys, vals, ord, static_cast<unsigned>(S - 1),
                     32 - ilog2_pow2(static_cast<unsigned>(S)), table_limit(S, G)};
    clear_all<G, NUM>(g, keys, vals, S);
    if (NUM) clear_all<G, NUM>(g, ck, cv, S);
    __syncwarp();
    const TV* avals = static_cast<const TV*>(a.A.v);
    const TV* bvals = static_cast<const TV*>(a.B.v);
    const bool b_long = p.b_long;

    const int gpw = 32 / G;
    const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
    const long long wid = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (long long wbase = wid * gpw; wbase < p.nrows; wbase += warps * gpw) {
        const long long it = wbase + ((threadIdx.x & 31) / G);
        const bool has = it < p.nrows;
        const int row = has ? p.rows[it] : 0;
        int ab = 0, alen = 0;
        if (has) {
            ab = __ldg(a.A.rp + row);
            alen = __ldg(a.A.rp + row + 1) - ab;
        }
        bool fail = false;
        const LeftG<TV> L{a.A.ci, avals, ab};
        const int n = accumulate<G, EP, NUM>(g, L, alen, a.B.rp, a.B.ci, bvals, b_long, T, fail);
        __syncwarp();
        const bool ok = has && !fail;
        if (fail) {
            clear_listed<G, NUM>(g, T, n);
            retry_row(g, p, row);
        } else if (ok) {
            if constexpr (NUM) {
                extract(g, T, n, ck, cv);
            } else {
                if (g.gl == 0) p.row_cnt[row] = n;
                clear_listed<G, NUM>(g, T, n);
            }
        }
        __syncwarp();
        if constexpr (NUM) {
            const long long base = out_base<G, MODE>(g, p, ok, row, n);
            int* oc = MODE == kNumBook ? p.ub_ci : p.c_ci;
            TO* ov = static_cast<TO*>(MODE == kNumBook ? p.ub_v : p.c_v);
            sorted_write<G, TO>(g, ck, cv, ok ? n : 0, oc, ov, base);
        }
    }
}

// Launch one instantiation (sets the dynamic shared-memory limit first).
template <typename K, typename Args>
cudaError_t launch_row_kernel(K k, const Args& a, const RowParams& p, const RowGeom& geo,
                              cudaStream_t st) {
    if (geo.smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(geo.smem));
        if (e != cudaSuccess) return e;
    }
    k<<<geo.grid, geo.block, geo.smem, st>>>(a, p);
    return cudaGetLastError();
}

}  // namespace sp3mm
