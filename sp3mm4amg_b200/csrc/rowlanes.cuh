// rowlanes.cuh -- direct R*A*P rows with the products formed in registers
// (sm_100a).
//
// One warp owns one output row and forms its products 32 per batch, one per
// lane, loaded straight from the right operand (no staging buffer).  Batch
// order then lane order is exactly the reference's product order -- left
// position t ascending, then the right row's entries ascending
// (code/src/include/SpMMUtilsGeneric.h:39-55).  Two layouts deal the
// products out: 2^lg lanes per left step when the right rows nearly fill
// them (the stencil rows of fine AMG levels), else packed, 32 consecutive
// products per batch found by a search over the steps' offsets (longer and
// uneven right rows: coarser levels, kNN graphs).
//
// Accumulation of one batch: one __match_any_sync groups equal columns; the
// lowest lane of each group (its leader) finds or inserts the column in the
// row's hash table; new columns are ranked by ballot in lane order, which is
// the reference's first-touch order (code/src/include/sparseMatrix.h:85-104);
// then each leader adds its group's products to the column's value one after
// another in lane order (the reference's order, each product rounded before
// the add), while the leaders of distinct columns work at once.
//
// The direct product (code/src/Sp3MM_CSR_OMP_UB_Generic.c:533-550):
// stage 1 forms the R*A row in table 1; stage 2 walks that row in
// first-touch order (its ord list) as the left row of a product with P into
// table 2, the C row, which is then sorted and written.  A row whose
// distinct-column count passes its table's load limit is cleared and put on
// the retry list, which the warp-per-row kernels redo with proven tables.
#pragma once

#include "rowwarp.cuh"

namespace sp3mm {

constexpr int kLanesPrefetch = 4;   // batches whose products are loaded ahead

// One batch: lane l holds product (key, v) when `valid`.  Updates nk, the
// table's distinct count.
//
// Probing: the leader of each group loads the 4-slot bucket of its key's
// hash with one 16-byte load; the key is there, or the first empty slot of
// the bucket is claimed with one CAS.  Only a full bucket or a lost CAS
// (rare at the tables' load) takes the general bucketed probe.
//
// Values: the leader adds its own product to the table value, then its
// group's other products in lane order, fetched by shuffles in rounds (one
// round per extra member of the largest group), and stores the sum once.
template <bool NUM>
__device__ __forceinline__ void lanes_batch(const WTab& T, int key, double v, bool valid,
                                            int& nk) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const int k = valid ? key : -2 - lane;   // idle lanes: unique keys
    const unsigned peers = __match_any_sync(kFull, k);
    const bool lead = valid && (peers & lt) == 0;
    bool is_new = false;
    int slot = -1;
    if (lead) {
        const unsigned b = hash_slot(k, T.shift) & ~3u;
        const int4 q = *reinterpret_cast<const int4*>(T.keys + b);
        if (q.x == k) slot = static_cast<int>(b);
        else if (q.y == k) slot = static_cast<int>(b) + 1;
        else if (q.z == k) slot = static_cast<int>(b) + 2;
        else if (q.w == k) slot = static_cast<int>(b) + 3;
        else {
            const int e = q.x == kEmpty ? 0 : q.y == kEmpty ? 1 : q.z == kEmpty ? 2
                        : q.w == kEmpty ? 3 : -1;
            if (e >= 0 && atomicCAS(T.keys + b + e, kEmpty, k) == kEmpty) {
                slot = static_cast<int>(b) + e;
                is_new = true;
            }
        }
    }
    if (__any_sync(kFull, lead && slot < 0)) {
        if (lead && slot < 0) slot = winsert(T, k, is_new);
    }
    const unsigned nb = __ballot_sync(kFull, is_new);
    if (is_new) T.ord[nk + __popc(nb & lt)] = slot;
    nk += __popc(nb);
    if constexpr (NUM) {
        double acc = 0.0;
        if (lead) acc = __dadd_rn(T.vals[slot], v);
        unsigned m = lead ? peers & (peers - 1) : 0u;   // members after the leader
        while (__any_sync(kFull, m != 0)) {
            const int src = m ? __ffs(m) - 1 : lane;
            const double x = __shfl_sync(kFull, v, src);
            if (m) {
                acc = __dadd_rn(acc, x);
                m &= m - 1;
            }
        }
        if (lead) T.vals[slot] = acc;
    }
    __syncwarp();
}

// Accumulate sum_{t<n} L.val(t) * B(L.key(t), :) into T in the reference
// order.  Steps are taken 32 at a time (lane j holds step t0 + j), and
// their products, in the reference's order (step, then right-row entry),
// are dealt out 32 per batch in one of two layouts:
//
// * !PACK (every right row has at most 2^lg entries; a longer one flags
//   kErrInput, since its entries past 2^lg would be missed): 2^lg lanes per
//   step, lane l of a batch holding entry (l mod 2^lg) of the batch's step
//   l >> lg.  Lanes past a row's end idle, so this layout is for right rows
//   that nearly fill their 2^lg lanes.
// * PACK: lane l of batch q holds product 32 q + l, whatever the rows'
//   lengths; the lane finds its step by a search over the steps' product
//   offsets (shuffles), so only the last batch of a chunk idles lanes.
//
// n is warp-uniform.  Returns false when the table passed its load limit;
// nk = distinct columns inserted (listed in T.ord either way).
template <bool NUM, bool PACK, typename TB, class Left>
__device__ __forceinline__ bool lanes_accumulate(const Left& L, int n, int lg,
                                                 const int* __restrict__ b_rp,
                                                 const int* __restrict__ b_ci,
                                                 const TB* __restrict__ b_v, const WTab& T,
                                                 unsigned* err, int& nk) {
    const int lane = threadIdx.x & 31;
    const int lgf = PACK ? 0 : lg;
    const int spb = 32 >> lgf;                  // fixed layout: steps per batch
    const int sub = lane >> lgf;                // this lane's step in a batch
    const int e = lane & ((1 << lgf) - 1);      // and its entry in that step
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
            if (!PACK && len > (1 << lgf)) atomicOr(err, kErrInput);
        }
        int off = 0, total = 0, nbat;
        if constexpr (PACK) {
            off = wscan_excl(len, total);
            nbat = (total + 31) >> 5;
        } else {
            const int cn = n - t0 < 32 ? n - t0 : 32;
            nbat = (cn + spb - 1) / spb;
        }
        const int base = rb - off;   // packed: product p of this step is entry base + p
        for (int q0 = 0; q0 < nbat; q0 += kLanesPrefetch) {
            int ck[kLanesPrefetch];
            double cv[kLanesPrefetch];
            bool ok[kLanesPrefetch];
#pragma unroll
            for (int q = 0; q < kLanesPrefetch; ++q) {
                int ei;
                double js;
                if constexpr (PACK) {
                    const int pidx = ((q0 + q) << 5) + lane;
                    // The last step whose first product is at or before
                    // pidx (an empty step shares its offset with the next).
                    int j = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        const int o = __shfl_sync(kFull, off, j + step);
                        if (o <= pidx) j += step;
                    }
                    ei = __shfl_sync(kFull, base, j) + pidx;
                    js = NUM ? __shfl_sync(kFull, s, j) : 0.0;
                    ok[q] = pidx < total;
                } else {
                    // src < 32 always: batches start at multiples of spb.
                    const int src = ((q0 + q) * spb + sub) & 31;
                    const int jl = __shfl_sync(kFull, len, src);
                    ei = __shfl_sync(kFull, rb, src) + e;
                    js = NUM ? __shfl_sync(kFull, s, src) : 0.0;
                    ok[q] = q0 + q < nbat && e < jl;
                }
                ck[q] = 0;
                cv[q] = 0.0;
                if (ok[q]) {
                    ck[q] = __ldg(b_ci + ei);
                    if (NUM) cv[q] = __dmul_rn(ldv(b_v, ei), js);
                }
            }
#pragma unroll
            for (int q = 0; q < kLanesPrefetch; ++q) {
                if (q0 + q < nbat) {
                    lanes_batch<NUM>(T, ck[q], cv[q], ok[q], nk);
                    if (nk > T.limit) return false;
                }
            }
        }
    }
    return true;
}

// Per-warp region (numeric): vals1[S1] vals2[S2] keys1[S1] keys2[S2]
// ord1[S1] ord2[S2]; symbolic: keys1 keys2 ord1 ord2.  S2 <= S1 (the C row
// is sorted in table 1's storage).
__host__ __device__ __forceinline__ size_t wlanes_bytes(bool num, int S1, int S2) {
    return static_cast<size_t>(S1 + S2) * (num ? 16 : 8);
}

template <int MODE, typename TV, typename TO, bool PACK>
__global__ void __launch_bounds__(256, 4) k_direct_lanes(DirectRowArgs a, RowParams p) {
    constexpr bool NUM = MODE != kSymb;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int S1 = p.S1, S2 = p.S2;
    unsigned char* region = smem + static_cast<size_t>(wib) * wlanes_bytes(NUM, S1, S2);
    double* vals1 = reinterpret_cast<double*>(region);
    double* vals2 = vals1 + S1;
    int* keys1 = NUM ? reinterpret_cast<int*>(vals2 + S2) : reinterpret_cast<int*>(region);
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
        bool ok = lanes_accumulate<NUM, PACK>(L1, rlen, p.lg1, a.A.rp, a.A.ci, av, T1, p.err,
                                              n1);
        if (ok) {
            const LeftT L2{keys1, vals1, ord1};
            ok = lanes_accumulate<NUM, PACK>(L2, n1, p.lg2, a.P.rp, a.P.ci, pv, T2, p.err, n2);
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

}  // namespace sp3mm
