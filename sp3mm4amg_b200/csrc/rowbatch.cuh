// rowbatch.cuh -- persistent warp-per-row kernels over the rows of many
// products (a batch).
//
// The rows of every product of a batch form one global row space (product
// b owns rows [row_base_b, row_base_b + M_b)); `row_item[g]` names the
// product of global row g and `items[b]` its operands.  A launch walks a
// list of global rows -- one or more table-size levels of the batch's
// binning -- with a grid-stride loop over persistent warps, so products of
// any size share one launch and the whole GPU.
//
// Each warp owns a fixed region of `scap` slots per table.  A row sizes its
// tables from its own bound (symbolic pass) or exact counts (numeric pass)
// and uses the first S <= scap slots: keys stay kEmpty and values 0 outside
// what a row touches (every row clears what it inserted, through the
// insertion-order list), so any prefix of the region is an empty table.
//
// Rows are accumulated as in the single-product register-product kernel
// (rowlanes.cuh, packed batches: right rows of any length): products formed
// in the reference's order, rounded products added in that order,
// first-touch forwarding of the R*A row into P
// (code/src/Sp3MM_CSR_OMP_UB_Generic.c:498-573), rows written sorted.
// Results are therefore bit-identical to the single-product path.
#pragma once

#include "batch.cuh"
#include "rowlanes.cuh"

namespace sp3mm {

// Bytes of one warp's region: numeric vals1[scap] vals2[scap] keys1[scap]
// keys2[scap] ord1[scap] ord2[scap]; symbolic keys1 keys2 ord1 ord2.
__host__ __device__ __forceinline__ size_t batch_region_bytes(bool num, int scap) {
    return static_cast<size_t>(scap) * (num ? 32 : 16);
}

// Smallest table (power of two >= 32 slots) whose load limit for a warp
// admits `need` distinct keys; the device twin of slots_for_need(need, 32).
__host__ __device__ __forceinline__ int batch_slots(long long need) {
    int S = 32;
    while (S < (1 << 30) && table_limit(S, 32) < need) S <<= 1;
    return S;
}

// Sum of the right-operand row lengths selected by the n keys of T (in
// insertion order): the product count of the next stage.
__device__ __forceinline__ long long batch_next_products(const WTab& T, int n, const int* rp) {
    const int lane = threadIdx.x & 31;
    long long s = 0;
    for (int t = lane; t < n; t += 32) {
        const int k = T.keys[T.ord[t]];
        s += __ldg(rp + k + 1) - __ldg(rp + k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    return s;
}

__device__ __forceinline__ void batch_retry(const BatchRowParams& p, int g, long long need) {
    if ((threadIdx.x & 31) != 0) return;
    if (p.retry_rows) {
        const int pos = atomicAdd(p.retry_count, 1);
        p.retry_rows[pos] = g;
        atomicMax(p.retry_need, static_cast<int>(need < INT_MAX ? need : INT_MAX));
    } else {
        atomicOr(p.err, kErrTable);
    }
}

// Book n entries for row g; -1 when the capacity is exhausted (flagged).
__device__ __forceinline__ long long batch_book(const BatchRowParams& p, int g, int n) {
    const int lane = threadIdx.x & 31;
    unsigned long long off = 0;
    if (lane == 0 && n > 0) off = atomicAdd(p.cursor, static_cast<unsigned long long>(n));
    off = __shfl_sync(kFull, off, 0);
    if (off + n > p.cap) {
        if (lane == 0) atomicOr(p.err, kErrBook);
        return -1;
    }
    if (lane == 0) p.row_off[g] = static_cast<long long>(off);
    return static_cast<long long>(off);
}

// One row's accumulation into T: packed register-product batches.
template <bool NUM, typename TB, class Left>
__device__ __forceinline__ bool batch_acc(const Left& L, int n, const int* b_rp,
                                          const int* b_ci, const TB* b_v, const WTab& T,
                                          unsigned* err, int& nk) {
    return lanes_accumulate<NUM, true>(L, n, -1, b_rp, b_ci, b_v, T, err, nk);
}

// Accumulate with an optimistic table of S slots, then (on overflow) once
// more with the proven size Sp when it fits the region.  Returns the size
// used, or 0 when the row does not fit (the table is left clear).
template <bool NUM, typename TB, class Left>
__device__ __forceinline__ int batch_accumulate(const Left& L, int n, const int* b_rp,
                                                const int* b_ci, const TB* b_v, int* keys,
                                                double* vals, int* ord, int S, int Sp, int scap,
                                                unsigned* err, int& nk) {
    WTab T = make_wtab(keys, vals, ord, S);
    if (batch_acc<NUM>(L, n, b_rp, b_ci, b_v, T, err, nk)) return S;
    wclear(T, nk, NUM);
    __syncwarp();
    if (Sp <= S || Sp > scap) return 0;
    T = make_wtab(keys, vals, ord, Sp);
    if (batch_acc<NUM>(L, n, b_rp, b_ci, b_v, T, err, nk)) return Sp;
    wclear(T, nk, NUM);
    __syncwarp();
    return 0;
}

template <int MODE, typename TV, typename TO, bool GT>
__global__ void __launch_bounds__(256, 4)
    k_batch_rows(const BItem* __restrict__ items, const int* __restrict__ row_item,
                 BatchRowParams p) {
    constexpr bool NUM = MODE != kSymb;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const int scap = p.scap;
    const size_t bytes = batch_region_bytes(NUM, scap);
    unsigned char* region =
        GT ? p.gtab + (static_cast<long long>(blockIdx.x) * nw + wib) * p.gstride
           : smem + static_cast<size_t>(wib) * bytes;
    double* vals1 = reinterpret_cast<double*>(region);
    double* vals2 = vals1 + scap;
    int* keys1 = NUM ? reinterpret_cast<int*>(vals2 + scap) : reinterpret_cast<int*>(region);
    int* keys2 = keys1 + scap;
    int* ord1 = keys2 + scap;
    int* ord2 = ord1 + scap;
    for (int s = lane; s < scap; s += 32) {
        keys1[s] = kEmpty;
        keys2[s] = kEmpty;
        if (NUM) {
            vals1[s] = 0.0;
            vals2[s] = 0.0;
        }
    }
    __syncwarp();

    const int nrows = p.nrows_dev ? *p.nrows_dev : p.nrows;
    const long long warps = static_cast<long long>(gridDim.x) * nw;
    for (long long it = static_cast<long long>(blockIdx.x) * nw + wib; it < nrows; it += warps) {
        const int g = p.rows[p.reverse ? nrows - 1 - it : it];
        const BItem* I = items + __ldg(row_item + g);
        const int kind = I->kind;
        const int i = static_cast<int>(g - I->row_base);
        const CsrView X = I->X;
        const int xb = __ldg(X.rp + i);
        const int xlen = __ldg(X.rp + i + 1) - xb;
        const LeftG<TV> L1{X.ci, static_cast<const TV*>(X.v), xb};
        const CsrView Y = I->Y;
        int n1 = 0, n2 = 0, S1, S2 = 0;
        if (kind == kBatchDirect) {
            const CsrView Z = I->Z;
            long long need2 = 0;
            if constexpr (MODE != kNumExact) {
                const int need1 = __ldg(p.need + g);
                const int opt1 = p.need_opt ? __ldg(p.need_opt + g) : need1 >> p.d1;
                S1 = batch_accumulate<NUM>(L1, xlen, Y.rp, Y.ci, static_cast<const TV*>(Y.v),
                                           keys1, vals1, ord1, batch_slots(opt1),
                                           batch_slots(need1), scap, p.err, n1);
                if (S1 == 0) {
                    batch_retry(p, g, need1);
                    continue;
                }
                const WTab T1 = make_wtab(keys1, vals1, ord1, S1);
                need2 = min(batch_next_products(T1, n1, Z.rp), static_cast<long long>(Z.N));
                const LeftT L2{keys1, vals1, ord1};
                S2 = batch_accumulate<NUM>(L2, n1, Z.rp, Z.ci, static_cast<const TV*>(Z.v),
                                           keys2, vals2, ord2,
                                           min(batch_slots(need2 >> p.d2), scap),
                                           batch_slots(need2), scap, p.err, n2);
                wclear(T1, n1, NUM);
                __syncwarp();
                if (S2 == 0) {
                    batch_retry(p, g, max(static_cast<long long>(need1), need2));
                    continue;
                }
                if (lane == 0) {
                    p.cnt1[g] = n1;
                    p.cnt2[g] = n2;
                }
                if constexpr (MODE == kSymb) {
                    wclear(make_wtab(keys2, vals2, ord2, S2), n2, NUM);
                    __syncwarp();
                } else {
                    wextract(make_wtab(keys2, vals2, ord2, S2), n2, keys1, vals1);
                    const long long base = batch_book(p, g, n2);
                    wsorted_write<TO>(keys1, vals1, n2, p.ub_ci, static_cast<TO*>(p.ub_v), base);
                }
            } else {
                const int e1 = __ldg(p.cnt1 + g), e2 = __ldg(p.cnt2 + g);
                S1 = batch_slots(e1);
                S2 = batch_slots(e2);
                if (S1 <= scap) S1 = min(S1 << p.slack, scap);
                if (S2 <= scap) S2 = min(S2 << p.slack, scap);
                const WTab T1 = make_wtab(keys1, vals1, ord1, S1);
                const WTab T2 = make_wtab(keys2, vals2, ord2, S2);
                bool ok = S1 <= scap && S2 <= scap &&
                          batch_acc<NUM>(L1, xlen, Y.rp, Y.ci, static_cast<const TV*>(Y.v), T1,
                                         p.err, n1);
                if (ok) {
                    const LeftT L2{keys1, vals1, ord1};
                    ok = batch_acc<NUM>(L2, n1, Z.rp, Z.ci, static_cast<const TV*>(Z.v), T2,
                                        p.err, n2);
                }
                if (S1 <= scap) wclear(T1, n1, NUM);
                __syncwarp();
                if (!ok || n2 != e2) {
                    if (S2 <= scap) wclear(T2, n2, NUM);
                    if (lane == 0) atomicOr(p.err, kErrCount);
                    __syncwarp();
                    continue;
                }
                wextract(T2, n2, keys1, vals1);   // T1 is clear: sort scratch
                const long long base = __ldg(p.c_rp + g);
                wsorted_write<TO>(keys1, vals1, n2, p.c_ci, static_cast<TO*>(p.c_v), base);
            }
        } else {
            if constexpr (MODE != kNumExact) {
                const int need1 = __ldg(p.need + g);
                const int opt1 = p.need_opt ? __ldg(p.need_opt + g) : need1 >> p.d1;
                S1 = batch_accumulate<NUM>(L1, xlen, Y.rp, Y.ci, static_cast<const TV*>(Y.v),
                                           keys1, vals1, ord1, batch_slots(opt1),
                                           batch_slots(need1), scap, p.err, n1);
                if (S1 == 0) {
                    batch_retry(p, g, need1);
                    continue;
                }
                if (lane == 0) p.cnt2[g] = n1;
                if constexpr (MODE == kSymb) {
                    wclear(make_wtab(keys1, vals1, ord1, S1), n1, NUM);
                    __syncwarp();
                } else {
                    wextract(make_wtab(keys1, vals1, ord1, S1), n1, keys2, vals2);
                    const long long base = batch_book(p, g, n1);
                    wsorted_write<TO>(keys2, vals2, n1, p.ub_ci, static_cast<TO*>(p.ub_v), base);
                }
            } else {
                const int e = __ldg(p.cnt2 + g);
                S1 = batch_slots(e);
                if (S1 <= scap) S1 = min(S1 << p.slack, scap);
                const WTab T = make_wtab(keys1, vals1, ord1, S1);
                const bool ok = S1 <= scap && batch_acc<NUM>(L1, xlen, Y.rp, Y.ci,
                                                             static_cast<const TV*>(Y.v), T,
                                                             p.err, n1);
                if (!ok || n1 != e) {
                    if (S1 <= scap) wclear(T, n1, NUM);
                    if (lane == 0) atomicOr(p.err, kErrCount);
                    __syncwarp();
                    continue;
                }
                wextract(T, n1, keys2, vals2);   // second table: sort scratch
                const long long base = __ldg(p.c_rp + g);
                wsorted_write<TO>(keys2, vals2, n1, p.c_ci, static_cast<TO*>(p.c_v), base);
            }
        }
    }
}

}  // namespace sp3mm
