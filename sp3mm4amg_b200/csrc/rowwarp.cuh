// rowwarp.cuh -- warp-per-row accumulation kernels (sm_100a).
//
// One warp owns one output row.  The row's products are generated in the
// reference's order -- left-row position t ascending, then the selected
// right row's entries ascending -- and staged in shared memory as
// (column, rounded FP64 product) pairs, kStage at a time.  Each batch of 32
// staged products is resolved with one __match_any_sync: the lowest lane of
// every group of equal columns (the group's leader) finds or inserts the
// column in the row's hash table once and adds the group's products to the
// accumulator one after another in lane order.  Contributions to a column
// therefore arrive in the reference's order (code/src/include/
// SpMMUtilsGeneric.h:39-55: v[j] += b*s, the product rounded before the
// add), so values are bit-identical, with no value atomics and one table
// probe per distinct column per batch instead of one per product.
//
// First touch: new columns are inserted only by leaders, ranked by ballot in
// lane order, which is product order; across batches the order is the batch
// order.  This reproduces the order in which the reference's index map
// appends columns (code/src/include/sparseMatrix.h:85-104), the order in
// which the direct product forwards the R*A row into P
// (code/src/Sp3MM_CSR_OMP_UB_Generic.c:542-545).
//
// Staging: for a chunk of up to 32 left-row steps, lane j loads step j's
// scalar and right-row bounds, a warp scan turns the right-row lengths into
// offsets in the flattened product sequence, and every lane copies its
// step's entries of the current window.  Windows cut the sequence anywhere,
// since products are consumed in order.
//
// Tables are shared memory, or global memory in the GT instantiation used
// for rows too long for shared tables.  A row whose distinct-column count
// passes its table's load limit is cleared and appended to a retry list.
#pragma once

#include "rows.cuh"

namespace sp3mm {

constexpr int kStage = 128;   // staged products per window

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned r;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
    return r;
}

struct WTab {
    int* keys;
    double* vals;
    int* ord;
    unsigned smask;
    int shift;
    int limit;
};

__device__ __forceinline__ WTab make_wtab(int* keys, double* vals, int* ord, int S) {
    return WTab{keys, vals, ord, static_cast<unsigned>(S - 1),
                32 - ilog2_pow2(static_cast<unsigned>(S)), table_limit(S, 32)};
}

// Find `key` or claim an empty slot.  Only group leaders call it, so the
// keys of concurrent callers are distinct.  The table never fills (the row
// stops at the load limit), so the probe ends; it is bounded by the size.
// Probing visits aligned buckets of four slots, read with one 16-byte load
// (tables hold a power of two >= 32 slots at a 16-byte aligned base), which
// cuts the divergent probe iterations of a warp's leaders about fourfold.
// Where a key lands does not matter: insertion order is kept in T.ord.
__device__ __forceinline__ int winsert(const WTab& T, int key, bool& is_new) {
    unsigned s = hash_slot(key, T.shift) & ~3u;
    for (unsigned probe = 0; probe <= T.smask; probe += 4) {
        const int4 q = *reinterpret_cast<const int4*>(T.keys + s);
        const int k[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (k[j] == key) return static_cast<int>(s) + j;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (k[j] == kEmpty) {
                const int old = atomicCAS(T.keys + s + j, kEmpty, key);
                if (old == kEmpty) {
                    is_new = true;
                    return static_cast<int>(s) + j;
                }
                if (old == key) return static_cast<int>(s) + j;
            }
        }
        s = (s + 4) & T.smask;
    }
    return -1;
}

// Find `key` or claim an empty slot probing one slot at a time (linear
// probing from the key's hash).  Same contract as winsert; the batch kernels
// use it for small tables (measured faster there than bucketed probing,
// slower on long rows and the single-product kNN rows).
__device__ __forceinline__ int winsert1(const WTab& T, int key, bool& is_new) {
    unsigned s = hash_slot(key, T.shift);
    for (unsigned probe = 0; probe <= T.smask; ++probe) {
        const int k = T.keys[s];
        if (k == key) return static_cast<int>(s);
        if (k == kEmpty) {
            const int old = atomicCAS(T.keys + s, kEmpty, key);
            if (old == kEmpty) {
                is_new = true;
                return static_cast<int>(s);
            }
            if (old == key) return static_cast<int>(s);
        }
        s = (s + 1) & T.smask;
    }
    return -1;
}

// Probing of wbatch: bucketed (winsert), linear (winsert1), or chosen per
// table -- linear below kBucketMinSlots, where tables are lightly loaded
// and short, bucketed above, where a warp's 32 leaders otherwise wait on
// the longest of their linear probe runs.
enum { kProbeBucket = 0, kProbeLinear = 1, kProbeBySize = 2 };
constexpr unsigned kBucketMinSlots = 256;

// One batch: lane i holds staged product i (key sk[i], value sv[i]) when
// `valid`.  Updates nk, the table's distinct count.
template <bool NUM, int PROBE = kProbeBucket>
__device__ __forceinline__ void wbatch(const WTab& T, const int* sk, const double* sv, int i,
                                       bool valid, int& nk) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const int key = valid ? sk[i] : -2 - lane;   // idle lanes: unique keys
    const unsigned peers = __match_any_sync(kFull, key);
    bool is_new = false;
    int slot = 0;
    if (valid && (peers & lt) == 0) {
        const bool bucket =
            PROBE == kProbeBucket || (PROBE == kProbeBySize && T.smask + 1 >= kBucketMinSlots);
        slot = bucket ? winsert(T, key, is_new) : winsert1(T, key, is_new);
        if (NUM && slot >= 0) {
            double acc = T.vals[slot];
            const int i0 = i - lane;
            unsigned m = peers;
            do {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                acc = __dadd_rn(acc, sv[i0 + l]);
            } while (m);
            T.vals[slot] = acc;
        }
    }
    const unsigned nb = __ballot_sync(kFull, is_new);
    if (is_new) T.ord[nk + __popc(nb & lt)] = slot;
    nk += __popc(nb);
}

__device__ __forceinline__ int wscan_excl(int v, int& total) {
    const int lane = threadIdx.x & 31;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(kFull, x, 31);
    return x - v;
}

// Accumulate sum_{t<n} L.val(t) * B(L.key(t), :) into T in the reference
// order (the warp owns the row; n is warp-uniform).  Returns false when the
// table passed its load limit; nk = distinct columns inserted (listed in
// T.ord either way).
template <bool NUM, int PROBE = kProbeBucket, typename TB, class Left>
__device__ __forceinline__ bool waccumulate(const Left& L, int n, const int* __restrict__ b_rp,
                                            const int* __restrict__ b_ci,
                                            const TB* __restrict__ b_v, const WTab& T, int* sk,
                                            double* sv, int& nk) {
    const int lane = threadIdx.x & 31;
    nk = 0;
    for (int t0 = 0; t0 < n; t0 += 32) {
        const int t = t0 + lane;
        int rb = 0, len = 0;
        double s = 0.0;
        if (t < n) {
            const int k = L.key(t);
            if (NUM) s = L.val(t);
            rb = __ldg(b_rp + k);
            len = __ldg(b_rp + k + 1) - rb;
        }
        int total;
        const int off = wscan_excl(len, total);
        // Short right rows: each lane copies its own run.  Long rows: every
        // lane fills window slots, finding the slot's step by a binary
        // search over the lanes' offsets (the last lane whose offset is at
        // most the slot's position, which has a non-empty run).
        const bool spread = __reduce_max_sync(kFull, static_cast<unsigned>(len)) > 16u;
        for (int w0 = 0; w0 < total; w0 += kStage) {
            if (spread) {
                const int wl = min(kStage, total - w0);
#pragma unroll
                for (int r = 0; r < kStage / 32; ++r) {
                    const int i = lane + 32 * r;
                    const int pidx = w0 + i;
                    int j = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        const int oc = __shfl_sync(kFull, off, j + step);
                        if (oc <= pidx) j += step;
                    }
                    const int rbj = __shfl_sync(kFull, rb, j);
                    const int ofj = __shfl_sync(kFull, off, j);
                    double sj = 0.0;
                    if (NUM) sj = __shfl_sync(kFull, s, j);
                    if (i < wl) {
                        const int e = rbj + pidx - ofj;
                        sk[i] = __ldg(b_ci + e);
                        if (NUM) sv[i] = __dmul_rn(ldv(b_v, e), sj);
                    }
                }
            } else {
                // Stage this lane's entries of window [w0, w0 + kStage).
                const int e_end = min(len, w0 + kStage - off);
                int e = max(0, w0 - off);
#pragma unroll 4
                for (; e < e_end; ++e) {
                    const int pos = off + e - w0;
                    sk[pos] = __ldg(b_ci + rb + e);
                    if (NUM) sv[pos] = __dmul_rn(ldv(b_v, rb + e), s);
                }
            }
            __syncwarp();
            const int wl = min(kStage, total - w0);
            for (int i0 = 0; i0 < wl; i0 += 32) {
                wbatch<NUM, PROBE>(T, sk, sv, i0 + lane, i0 + lane < wl, nk);
                if (nk > T.limit) {
                    __syncwarp();
                    return false;
                }
            }
            __syncwarp();
        }
    }
    return true;
}

__device__ __forceinline__ void wclear(const WTab& T, int n, bool num) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < n; i += 32) {
        const int s = T.ord[i];
        T.keys[s] = kEmpty;
        if (num) T.vals[s] = 0.0;
    }
}

// Move T's n entries (listed in ord) into (ck, cv)[0..n), clearing T.
__device__ __forceinline__ void wextract(const WTab& T, int n, int* ck, double* cv) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < n; i += 32) {
        const int s = T.ord[i];
        ck[i] = T.keys[s];
        cv[i] = T.vals[s];
        T.keys[s] = kEmpty;
        T.vals[s] = 0.0;
    }
}

// Write (ck, cv)[0..n) sorted by key to out[base..]; ck / cv hold
// next_pow2(n) slots and are reset to kEmpty / 0.
template <typename TO>
__device__ __forceinline__ void wsorted_write(int* ck, double* cv, int n, int* out_ci, TO* out_v,
                                              long long base) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    if (n <= 64) {
        const int k0 = lane < n ? ck[lane] : INT_MAX;
        const int k1 = lane + 32 < n ? ck[lane + 32] : INT_MAX;
        int r0 = 0, r1 = 0;
        for (int j = 0; j < n; ++j) {
            const int kj = ck[j];
            r0 += kj < k0;
            r1 += kj < k1;
        }
        if (base >= 0) {
            if (lane < n) {
                out_ci[base + r0] = k0;
                stv(out_v, base + r0, cv[lane]);
            }
            if (lane + 32 < n) {
                out_ci[base + r1] = k1;
                stv(out_v, base + r1, cv[lane + 32]);
            }
        }
        __syncwarp();
        if (lane < n) {
            ck[lane] = kEmpty;
            cv[lane] = 0.0;
        }
        if (lane + 32 < n) {
            ck[lane + 32] = kEmpty;
            cv[lane + 32] = 0.0;
        }
        __syncwarp();
        return;
    }
    const int P2 = static_cast<int>(next_pow2(static_cast<unsigned>(n)));
    for (int i = n + lane; i < P2; i += 32) ck[i] = INT_MAX;
    __syncwarp();
    for (int k = 2; k <= P2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P2; i += 32) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const int a = ck[i], b = ck[ixj];
                    if ((a > b) == ((i & k) == 0)) {
                        ck[i] = b;
                        ck[ixj] = a;
                        const double tv = cv[i];
                        cv[i] = cv[ixj];
                        cv[ixj] = tv;
                    }
                }
            }
            __syncwarp();
        }
    }
    if (base >= 0)
        for (int i = lane; i < n; i += 32) {
            out_ci[base + i] = ck[i];
            stv(out_v, base + i, cv[i]);
        }
    __syncwarp();
    for (int i = lane; i < P2; i += 32) {
        ck[i] = kEmpty;
        cv[i] = 0.0;
    }
    __syncwarp();
}

// Output offset of a finished row: booking (one atomic per row) or the
// exact row pointer; -1 when the row cannot be written.
template <int MODE>
__device__ __forceinline__ long long wout_base(const RowParams& p, int row, int n) {
    const int lane = threadIdx.x & 31;
    if (MODE == kNumBook) {
        unsigned long long off = 0;
        if (lane == 0 && n > 0) off = atomicAdd(p.cursor, static_cast<unsigned long long>(n));
        off = __shfl_sync(kFull, off, 0);
        if (off + n > p.cap) {
            if (lane == 0) atomicOr(p.err, kErrBook);
            return -1;
        }
        if (lane == 0) {
            p.row_off[row] = static_cast<long long>(off);
            p.row_cnt[row] = n;
        }
        return static_cast<long long>(off);
    }
    const long long b = p.c_rp[row];
    if (p.c_rp[row + 1] - b != n) {
        if (lane == 0) atomicOr(p.err, kErrCount);
        return -1;
    }
    return b;
}

__device__ __forceinline__ void wretry(const RowParams& p, int row) {
    if ((threadIdx.x & 31) != 0) return;
    if (p.retry_rows) {
        const int pos = atomicAdd(p.retry_count, 1);
        p.retry_rows[pos] = row;
    } else {
        atomicOr(p.err, kErrTable);
    }
}

// Per-warp region (numeric): sv[kStage] vals1[S1] vals2[S2] sk[kStage]
// keys1[S1] keys2[S2] ord1[S1] ord2[S2]; symbolic: sk keys1 keys2 ord1 ord2.
__host__ __device__ __forceinline__ size_t wdirect_bytes(bool num, int S1, int S2) {
    return num ? static_cast<size_t>(kStage) * 12 + static_cast<size_t>(S1 + S2) * 16
               : static_cast<size_t>(kStage) * 4 + static_cast<size_t>(S1 + S2) * 8;
}
// Pair (numeric): sv[kStage] vals[S] cv[S] sk[kStage] keys[S] ck[S] ord[S];
// symbolic: sk keys ord.
__host__ __device__ __forceinline__ size_t wpair_bytes(bool num, int S) {
    return num ? static_cast<size_t>(kStage) * 12 + static_cast<size_t>(S) * 28
               : static_cast<size_t>(kStage) * 4 + static_cast<size_t>(S) * 8;
}

template <int MODE, typename TV, typename TO, bool GT>
__global__ void __launch_bounds__(256, 4) k_direct_warp(DirectRowArgs a, RowParams p) {
    constexpr bool NUM = MODE != kSymb;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int S1 = p.S1, S2 = p.S2;
    const long long bytes = static_cast<long long>(wdirect_bytes(NUM, S1, S2));
    unsigned char* region = group_region<GT>(smem, p, wib, blockDim.x >> 5, bytes);
    double* sv = reinterpret_cast<double*>(region);
    double* vals1 = sv + kStage;
    double* vals2 = vals1 + S1;
    int* sk = NUM ? reinterpret_cast<int*>(vals2 + S2) : reinterpret_cast<int*>(region);
    int* keys1 = sk + kStage;
    int* keys2 = keys1 + S1;
    int* ord1 = keys2 + S2;
    int* ord2 = ord1 + S1;
    const WTab T1 = make_wtab(keys1, vals1, ord1, S1);
    const WTab T2 = make_wtab(keys2, vals2, ord2, S2);
    for (int s = lane; s < S1; s += 32) {
        keys1[s] = kEmpty;
        if (NUM) vals1[s] = 0.0;
    }
    for (int s = lane; s < S2; s += 32) {
        keys2[s] = kEmpty;
        if (NUM) vals2[s] = 0.0;
    }
    __syncwarp();
    const TV* rv = static_cast<const TV*>(a.R.v);
    const TV* av = static_cast<const TV*>(a.A.v);
    const TV* pv = static_cast<const TV*>(a.P.v);

    const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
    for (long long it = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + wib;
         it < p.nrows; it += warps) {
        const int row = p.rows[it];
        const int rb = __ldg(a.R.rp + row);
        const int rlen = __ldg(a.R.rp + row + 1) - rb;
        int n1 = 0, n2 = 0;
        const LeftG<TV> L1{a.R.ci, rv, rb};
        bool ok = waccumulate<NUM>(L1, rlen, a.A.rp, a.A.ci, av, T1, sk, sv, n1);
        if (ok) {
            const LeftT L2{keys1, vals1, ord1};
            ok = waccumulate<NUM>(L2, n1, a.P.rp, a.P.ci, pv, T2, sk, sv, n2);
        }
        wclear(T1, n1, NUM);
        __syncwarp();
        if (!ok) {
            wclear(T2, n2, NUM);
            wretry(p, row);
            __syncwarp();
            continue;
        }
        if constexpr (!NUM) {
            if (lane == 0) {
                p.row_cnt[row] = n2;
                if (p.row_cnt1) p.row_cnt1[row] = n1;
            }
            wclear(T2, n2, NUM);
            __syncwarp();
        } else {
            wextract(T2, n2, keys1, vals1);   // T1 is free: sort scratch
            const long long base = wout_base<MODE>(p, row, n2);
            int* oc = MODE == kNumBook ? p.ub_ci : p.c_ci;
            TO* ov = static_cast<TO*>(MODE == kNumBook ? p.ub_v : p.c_v);
            wsorted_write<TO>(keys1, vals1, n2, oc, ov, base);
        }
    }
}

template <int MODE, typename TV, typename TO, bool GT>
__global__ void __launch_bounds__(256, 4) k_pair_warp(PairRowArgs a, RowParams p) {
    constexpr bool NUM = MODE != kSymb;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int S = p.S1;
    const long long bytes = static_cast<long long>(wpair_bytes(NUM, S));
    unsigned char* region = group_region<GT>(smem, p, wib, blockDim.x >> 5, bytes);
    double* sv = reinterpret_cast<double*>(region);
    double* vals = sv + kStage;
    double* cv = vals + S;
    int* sk = NUM ? reinterpret_cast<int*>(cv + S) : reinterpret_cast<int*>(region);
    int* keys = sk + kStage;
    int* ck = NUM ? keys + S : keys;
    int* ord = NUM ? ck + S : keys + S;
    const WTab T = make_wtab(keys, vals, ord, S);
    for (int s = lane; s < S; s += 32) {
        keys[s] = kEmpty;
        if (NUM) {
            vals[s] = 0.0;
            ck[s] = kEmpty;
            cv[s] = 0.0;
        }
    }
    __syncwarp();
    const TV* avals = static_cast<const TV*>(a.A.v);
    const TV* bvals = static_cast<const TV*>(a.B.v);

    const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
    for (long long it = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + wib;
         it < p.nrows; it += warps) {
        const int row = p.rows[it];
        const int ab = __ldg(a.A.rp + row);
        const int alen = __ldg(a.A.rp + row + 1) - ab;
        int n = 0;
        const LeftG<TV> L{a.A.ci, avals, ab};
        const bool ok = waccumulate<NUM>(L, alen, a.B.rp, a.B.ci, bvals, T, sk, sv, n);
        if (!ok) {
            wclear(T, n, NUM);
            wretry(p, row);
            __syncwarp();
            continue;
        }
        if constexpr (!NUM) {
            if (lane == 0) p.row_cnt[row] = n;
            wclear(T, n, NUM);
            __syncwarp();
        } else {
            wextract(T, n, ck, cv);
            const long long base = wout_base<MODE>(p, row, n);
            int* oc = MODE == kNumBook ? p.ub_ci : p.c_ci;
            TO* ov = static_cast<TO*>(MODE == kNumBook ? p.ub_v : p.c_v);
            wsorted_write<TO>(ck, cv, n, oc, ov, base);
        }
    }
}

}  // namespace sp3mm
