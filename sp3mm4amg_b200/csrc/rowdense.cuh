// rowdense.cuh -- direct R*A*P rows with heavy work (coarse AMG levels): one
// CTA per output row, dense accumulators in shared memory (sm_100a).
//
// On the coarse levels of a hierarchy the rows are few and long: an R row
// reaches hundreds of A rows of hundreds of entries, the R*A row has
// thousands of columns, and one warp per row with a hash table large enough
// for it leaves a handful of warps per SM.  Here a CTA of kDWarps warps owns
// one row, accumulating into a dense slice of shared memory indexed by
// column (no hashing).  Every column must receive its contributions in the
// reference's order (left position ascending, then the right row's entries;
// code/src/include/SpMMUtilsGeneric.h:39-55); the two stages keep it in two
// ways.
//
// Stage 1 (the R*A row) steps through the left entries: the CTA takes one
// right row per step (a right row's columns are distinct, so a step has no
// conflicts) and synchronises between steps (dstage1).  It walks the row's
// column span in chunks of kDSpan columns.  Each column's first touch is
// recorded as the flat position of the product that made it (left
// position, then right-row entry), and after each chunk the touched columns
// are listed with their position and value.  Sorting that list by position
// gives the order in which the reference's index map appends the columns
// (code/src/include/sparseMatrix.h:85-104), the order in which the direct
// product forwards the R*A row into P (code/src/Sp3MM_CSR_OMP_UB_Generic.c:
// 542-545).
//
// Stage 2 forwards the list into P over the span of the P columns it
// reaches (one chunk), with the warps splitting the COLUMNS, not the
// products: warp w owns a contiguous column range, finds in every right row
// the segment that falls in its range (right rows are ordered), and
// processes exactly its products in order.  Within a batch of 32 staged
// products, the products of one right row's segment have distinct columns
// and are added at once, segment after segment (batches spread over many
// short segments group equal columns with a match).  The C row is written
// in column order straight from the dense slice (no sort).
//
// A row whose R*A row has more than kDList columns, or whose C row spans more
// than kDSpan columns, is appended to the retry list (processed by the
// retry launch with tables sized from a proven bound).
//
// The file is compiled in two configurations, each in a namespace of its
// own (SP3MM_DENSE_NS): `dbig` (the default: an 8,192-column slice, lists of
// 4,096 columns, one CTA per SM) and `dsmall` (rows_dense_small.cu: half the
// slice and list in half the shared memory, two CTAs per SM, for rows whose
// tables are at most kDenseSmallSlots).
#pragma once

#include "rowwarp.cuh"

#ifndef SP3MM_DENSE_NS
#define SP3MM_DENSE_NS dbig
#define SP3MM_DENSE_SPAN 8192
#define SP3MM_DENSE_LIST 4096
#define SP3MM_DENSE_STAGE 128
#define SP3MM_DENSE_MINB 1
#endif

namespace sp3mm {
namespace SP3MM_DENSE_NS {

constexpr int kDWarps = 16;    // warps per CTA (one output row per CTA)
constexpr int kDSpan = SP3MM_DENSE_SPAN;   // columns of the dense accumulator slice
constexpr int kDList = SP3MM_DENSE_LIST;   // R*A row entries a CTA holds
constexpr int kDStage = SP3MM_DENSE_STAGE;   // stage-2 staged products per warp window
constexpr int kDHist = 1024;   // bins of the column histogram that balances the warps
constexpr int kDSamples = 2048;   // columns sampled per stage for that histogram
constexpr int kDSearch = 4;    // arity of the segment searches
constexpr int kDSteps = kDWarps * 32;   // stage-1 left entries described at a time
constexpr int kDAhead = 4;     // stage-1 steps whose products a thread loads ahead
// The stage-1 step descriptions live over the warps' stage-2 staging.
static_assert(kDSteps * 20 <= kDWarps * kDStage * 16, "step descriptions exceed the staging");

// Dynamic shared memory: acc double[kDSpan] | ftq int[kDSpan] (after stage 1:
// u64 sort keys [kDList]) | lkey int[kDList] | lq int[kDList] |
// lval double[kDList] | touched u8[kDSpan] | per warp: sk int[kDStage],
// sv double[kDStage], sst int[kDStage] | hist int[kDHist] | total int.
__host__ __device__ constexpr size_t dense_smem_bytes() {
    return static_cast<size_t>(kDSpan) * 8 + static_cast<size_t>(kDSpan) * 4 +
           static_cast<size_t>(kDList) * 16 + static_cast<size_t>(kDSpan) +
           static_cast<size_t>(kDWarps) * kDStage * 16 + static_cast<size_t>(kDHist) * 4 + 16;
}

// Pivot step of a K-ary lower bound: the answer (first index whose column
// is >= x) lies in [lo, lo + n]; the K-1 pivots lo + floor(n k / K) were
// loaded into v, and the step keeps the part between the last pivot below x
// and the first at or above it.
template <int K>
__device__ __forceinline__ void kary_step(const int (&m)[K - 1], const int (&v)[K - 1], int x,
                                          int& lo, int& n) {
    int left = lo, right = m[0];
#pragma unroll
    for (int k = 1; k < K; ++k) {
        if (v[k - 1] < x) {
            left = m[k - 1] + 1;
            right = k < K - 1 ? m[k < K - 1 ? k : 0] : lo + n;
        }
    }
    lo = left;
    n = right - left;
}

// The segment [sb, se) of the right row [ab, ae) (columns ascending, first
// and last given) whose columns fall in [wlo, whi); the row reaches the
// range (first < whi, last >= wlo).  Both ends are searched together, K-ary:
// each step loads the K-1 pivots of both searches at once, so the chain of
// dependent loads is log_K of the row's length instead of twice log_2.
template <int K>
__device__ __forceinline__ void segment_bounds(const int* __restrict__ ci, int ab, int ae,
                                               int first, int last, int wlo, int whi, int& sb,
                                               int& se) {
    // The answers lie in [ab + 1, ae - 1] when searched (first < wlo <= last,
    // or first < whi <= last).
    int lo0 = first < wlo ? ab + 1 : ab, n0 = first < wlo ? ae - ab - 2 : 0;
    int lo1 = last >= whi ? ab + 1 : ae, n1 = last >= whi ? ae - ab - 2 : 0;
    while (n0 > 0 || n1 > 0) {
        int m0[K - 1], m1[K - 1], v0[K - 1], v1[K - 1];
#pragma unroll
        for (int k = 1; k < K; ++k) {
            m0[k - 1] = lo0 + static_cast<int>((static_cast<long long>(n0) * k) / K);
            m1[k - 1] = lo1 + static_cast<int>((static_cast<long long>(n1) * k) / K);
        }
#pragma unroll
        for (int k = 0; k < K - 1; ++k) {
            v0[k] = __ldg(ci + (n0 > 0 ? m0[k] : ab));
            v1[k] = __ldg(ci + (n1 > 0 ? m1[k] : ab));
        }
        if (n0 > 0) kary_step<K>(m0, v0, wlo, lo0, n0);
        if (n1 > 0) kary_step<K>(m1, v1, whi, lo1, n1);
    }
    sb = lo0;
    se = lo1;
}

// The stage-1 list in first-touch order: entry t is list index sorted[t]
// (low 32 bits of the sorted (position, index) key).
struct LeftSorted {
    const unsigned long long* sorted;
    const int* keys;
    const double* vals;
    __device__ __forceinline__ int key(int t) const {
        return keys[static_cast<unsigned>(sorted[t])];
    }
    __device__ __forceinline__ double val(int t) const {
        return vals[static_cast<unsigned>(sorted[t])];
    }
};

// Batches whose products come from at most this many right-row segments
// are added in rounds by segment; others group equal columns with a match.
constexpr int kDSegRounds = 3;

// One batch of staged products into the dense slice (slot = column - base),
// marking the columns touched.  sst[i] is the left
// position (step) a staged product comes from; steps never decrease along
// the staging, and one step's columns are distinct (a right row's columns
// are), so the products of one segment of equal steps are added all at
// once, segment after segment: every column receives its products in the
// reference's order without grouping equal columns.  Batches spread over
// many short segments group equal columns with __match_any_sync instead
// (the lowest lane of a group adds the group's products in lane order).
template <bool NUM>
__device__ __forceinline__ void dbatch(double* acc, unsigned char* touched, int base,
                                       const int* sk, const double* sv, const int* sst, int i,
                                       bool valid) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const int st = valid ? sst[i] : -1;
    const int prev = __shfl_up_sync(kFull, st, 1);
    const unsigned starts = __ballot_sync(kFull, valid && (lane == 0 || prev != st));
    const int nseg = __popc(starts);
    if (nseg <= kDSegRounds) {
        const int seg = __popc(starts & (lt | (1u << lane))) - 1;
        const int slot = valid ? sk[i] - base : 0;
        const double v = (NUM && valid) ? sv[i] : 0.0;
        for (int r = 0; r < nseg; ++r) {
            if (valid && seg == r) {
                touched[slot] = 1;
                if (NUM) acc[slot] = __dadd_rn(acc[slot], v);
            }
            __syncwarp();
        }
        return;
    }
    const int key = valid ? sk[i] : -2 - lane;
    const unsigned peers = __match_any_sync(kFull, key);
    if (valid && (peers & lt) == 0) {
        const int slot = key - base;
        touched[slot] = 1;
        if (NUM) {
            double v = acc[slot];
            const int i0 = i - lane;
            unsigned m = peers;
            do {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                v = __dadd_rn(v, sv[i0 + l]);
            } while (m);
            acc[slot] = v;
        }
    }
}

// sum_{t<n} L.val(t) * B(L.key(t), :) restricted to the columns [wlo, whi)
// (inside the slice starting at `base`), in the reference's order (stage 2).
template <bool NUM, typename TB, class Left>
__device__ __forceinline__ void daccumulate(const Left& L, int n, const int* __restrict__ b_rp,
                                            const int* __restrict__ b_ci,
                                            const TB* __restrict__ b_v, int wlo, int whi,
                                            int base, double* acc, unsigned char* touched,
                                            int* sk, double* sv, int* sst) {
    if (wlo >= whi) return;
    const int lane = threadIdx.x & 31;
    for (int t0 = 0; t0 < n; t0 += 32) {
        const int t = t0 + lane;
        int ab = 0, ae = 0, sb = 0, se = 0;
        double s = 0.0;
        if (t < n) {
            const int k = L.key(t);
            if (NUM) s = L.val(t);
            ab = __ldg(b_rp + k);
            ae = __ldg(b_rp + k + 1);
            // Rows wholly on one side of the range need no search.
            sb = se = ae;
            if (ab < ae) {
                const int first = __ldg(b_ci + ab), last = __ldg(b_ci + ae - 1);
                if (last < wlo) {
                    sb = se = ae;
                } else if (first >= whi) {
                    sb = se = ab;
                } else {
                    segment_bounds<kDSearch>(b_ci, ab, ae, first, last, wlo, whi, sb, se);
                }
            }
        }
        const int len = se - sb;
        int total;
        const int off = wscan_excl(len, total);
        if (total == 0) continue;
        // Staged in product order, lane i of a window holding product
        // w0 + i: consecutive lanes read consecutive entries of a segment
        // (the loads coalesce), each lane finding its step by a search over
        // the steps' offsets.
        const int sbase = sb - off;   // product p of this step is entry sbase + p
        for (int w0 = 0; w0 < total; w0 += kDStage) {
            const int wl = min(kDStage, total - w0);
#pragma unroll
            for (int r = 0; r < kDStage / 32; ++r) {
                const int i = lane + 32 * r;
                const int pidx = w0 + i;
                int j = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int oc = __shfl_sync(kFull, off, j + step);
                    if (oc <= pidx) j += step;
                }
                const int e = __shfl_sync(kFull, sbase, j) + pidx;
                double sj = 0.0;
                if (NUM) sj = __shfl_sync(kFull, s, j);
                if (i < wl) {
                    sk[i] = __ldg(b_ci + e);
                    if (NUM) sv[i] = __dmul_rn(ldv(b_v, e), sj);
                    sst[i] = j;
                }
            }
            __syncwarp();
            for (int i0 = 0; i0 < wl; i0 += 32)
                dbatch<NUM>(acc, touched, base, sk, sv, sst, i0 + lane, i0 + lane < wl);
            __syncwarp();
        }
    }
}

// Block-wide sum of `v` into *stot (zeroed by the caller before the barrier
// that precedes this call).
__device__ __forceinline__ void block_total(long long v, long long* stot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(stot),
                                           static_cast<unsigned long long>(v));
}

// Block-wide min / max of (lo, hi) into *slo / *shi (initialised by the
// caller before the barrier that precedes this call).
__device__ __forceinline__ void block_span(int lo, int hi, int* slo, int* shi) {
    lo = __reduce_min_sync(kFull, lo);
    hi = __reduce_max_sync(kFull, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(slo, lo);
        atomicMax(shi, hi);
    }
}

// Shared state of a dense CTA (the dynamic region carved up, plus the
// block's scalars).
struct DenseSmem {
    double* acc;
    int* ftq;
    unsigned long long* sorted;
    int* lkey;
    int* lq;
    double* lval;
    unsigned char* touched;
    int* sk;
    double* sv;
    int* sst;
    int* step;   // stage-1 step descriptions (over the warps' staging)
    int* hist;
    long long* s_tot;
    int* s_n1;
    int* s_lo;
    int* s_hi;
    int* s_cnt;
    long long* s_base;
};

__device__ __forceinline__ DenseSmem dense_smem(unsigned char* smem, int* s_n1, int* s_lo,
                                                int* s_hi, int* s_cnt, long long* s_base) {
    DenseSmem d;
    d.acc = reinterpret_cast<double*>(smem);
    d.ftq = reinterpret_cast<int*>(d.acc + kDSpan);
    d.sorted = reinterpret_cast<unsigned long long*>(d.ftq);
    d.lkey = d.ftq + kDSpan;
    d.lq = d.lkey + kDList;
    d.lval = reinterpret_cast<double*>(d.lq + kDList);
    d.touched = reinterpret_cast<unsigned char*>(d.lval + kDList);
    unsigned char* wst = d.touched + kDSpan + static_cast<size_t>(threadIdx.x >> 5) * kDStage * 16;
    d.sk = reinterpret_cast<int*>(wst);
    d.sv = reinterpret_cast<double*>(d.sk + kDStage);
    d.sst = reinterpret_cast<int*>(d.sv + kDStage);
    d.step = reinterpret_cast<int*>(d.touched + kDSpan);
    d.hist = reinterpret_cast<int*>(d.touched + kDSpan + static_cast<size_t>(kDWarps) * kDStage * 16);
    d.s_tot = reinterpret_cast<long long*>(d.hist + kDHist);
    d.s_n1 = s_n1;
    d.s_lo = s_lo;
    d.s_hi = s_hi;
    d.s_cnt = s_cnt;
    d.s_base = s_base;
    return d;
}

__device__ __forceinline__ void dense_clear(const DenseSmem& d) {
    for (int s = threadIdx.x; s < kDSpan; s += blockDim.x) {
        d.acc[s] = 0.0;
        d.touched[s] = 0;
    }
}

// Column ranges of the warps over [cb, ce) holding about equal numbers of
// products: about kDSamples columns of the right rows (every st-th entry of
// each from a hashed start, st from the stage's product count `total`) go
// into a histogram of
// kDHist bins, and warp w starts at the bin where the cumulative count
// reaches w/kDWarps of the samples.  Any cover of [cb, ce) by disjoint
// ranges gives the same results; this one gives the warps equal work.
template <class Left>
__device__ __forceinline__ void balanced_range(const DenseSmem& d, const Left& L, int n,
                                               const int* __restrict__ b_rp,
                                               const int* __restrict__ b_ci, int cb, int ce,
                                               long long total, int& wlo, int& whi) {
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    int shift = 0;
    while ((static_cast<long long>(kDHist) << shift) < static_cast<long long>(ce) - cb) ++shift;
    for (int b = threadIdx.x; b < kDHist; b += blockDim.x) d.hist[b] = 0;
    __syncthreads();
    const long long stl = (total + kDSamples - 1) / kDSamples;
    const int st = static_cast<int>(stl < 1 ? 1 : (stl > INT_MAX ? INT_MAX : stl));
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = L.key(t);
        const int ab = __ldg(b_rp + k), ae = __ldg(b_rp + k + 1);
        // A hashed start per row: every entry is sampled with probability
        // 1/st, also in rows shorter than st.
        const unsigned h = static_cast<unsigned>(t) * 2654435761u;
        for (long long e = ab + static_cast<int>(h % static_cast<unsigned>(st)); e < ae; e += st) {
            const int col = __ldg(b_ci + e);
            if (col >= cb && col < ce) atomicAdd(&d.hist[(col - cb) >> shift], 1);
        }
    }
    __syncthreads();
    if (wid == 0) {
        // Inclusive prefix: lane l owns bins [32l, 32l + 32).
        int local = 0;
        for (int j = 0; j < 32; ++j) local += d.hist[lane * 32 + ((j + lane) & 31)];
        int all;
        int run = wscan_excl(local, all);
        for (int j = 0; j < 32; ++j) {
            run += d.hist[lane * 32 + j];
            d.hist[lane * 32 + j] = run;
        }
    }
    __syncthreads();
    const int tot = d.hist[kDHist - 1];
    auto bound = [&](int w) -> int {
        if (w <= 0) return cb;
        if (w >= kDWarps) return ce;
        const int q = static_cast<int>((static_cast<long long>(tot) * w + kDWarps - 1) / kDWarps);
        int a = 0, b = kDHist;
        while (a < b) {
            const int m = (a + b) >> 1;
            if (d.hist[m] < q) a = m + 1;
            else b = m;
        }
        const long long c = static_cast<long long>(cb) + (static_cast<long long>(a + 1) << shift);
        return static_cast<int>(c < ce ? c : ce);
    };
    wlo = bound(wid);
    whi = bound(wid + 1);
    __syncthreads();
}

// Stage 1 (the R*A row) over the columns [cb, ce) of the slice starting at
// cb, one left entry (step) at a time: the whole CTA takes step t's right
// row (thread i its entries i, i + blockDim, ...), adds the rounded products
// to the dense slice and records each new column's first touch (the flat
// position of its product: the full lengths of the right rows before t plus
// its offset), then synchronises before step t + 1.  A right row's columns
// are distinct, so a step has no conflicts, and the barrier between steps
// keeps every column's contributions in the reference's order (left
// position ascending; code/src/include/SpMMUtilsGeneric.h:39-55).  Steps are
// described kDSteps at a time in shared memory (bounds, left value, flat
// position), and every thread loads its products (PER entries of each
// right row: 2 when the longest right row is longer than the CTA) kDAhead
// steps ahead, so a step costs a few shared-memory operations and one
// barrier.  Only the first `nw` warps step (enough for the longest right
// row, at most all):
// they synchronise among themselves with a named barrier, so warps that
// would idle add nothing to a step's cost.
template <bool NUM, int PER, typename TV>
__device__ __forceinline__ void dstage1(const DenseSmem& d, const CsrView& R, const CsrView& A,
                                        int rb, int rlen, int cb, int ce, int nw) {
    const int tid = threadIdx.x;
    const int nt = nw * 32;
    const int lane = tid & 31;
    const int wid = tid >> 5;
    const TV* rv = static_cast<const TV*>(R.v);
    const TV* av = static_cast<const TV*>(A.v);
    int* st_ab = d.step;
    int* st_ae = st_ab + kDSteps;
    int* st_fo = st_ae + kDSteps;
    double* st_s = reinterpret_cast<double*>(st_fo + kDSteps);
    int carry = 0;   // full right-row lengths before this block of steps
    for (int b0 = 0; b0 < rlen; b0 += kDSteps) {
        const int nb = min(kDSteps, rlen - b0);
        int ab = 0, ae = 0;
        double sv = 0.0;
        if (tid < nb) {
            const int k = __ldg(R.ci + rb + b0 + tid);
            if (NUM) sv = ldv(rv, rb + b0 + tid);
            ab = __ldg(A.rp + k);
            ae = __ldg(A.rp + k + 1);
        }
        int wt;
        const int x = wscan_excl(ae - ab, wt);
        if (lane == 0) d.hist[wid] = wt;
        __syncthreads();
        int before = carry, all = 0;
        for (int w = 0; w < kDWarps; ++w) {
            const int v = d.hist[w];
            if (w < wid) before += v;
            all += v;
        }
        carry += all;
        if (tid < nb) {
            st_ab[tid] = ab;
            st_ae[tid] = ae;
            st_fo[tid] = before + x;
            st_s[tid] = sv;
        }
        __syncthreads();
        if (wid >= nw) {
            __syncthreads();
            continue;
        }
        // pc / pvv[q][j]: the product of entry tid + j * nt of the right row
        // of step t0 + q (pc = -1: none).
        int pc[kDAhead][PER];
        double pvv[kDAhead][PER];
#pragma unroll
        for (int q = 0; q < kDAhead; ++q) {
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                pc[q][j] = -1;
                pvv[q][j] = 0.0;
                if (q < nb) {
                    const int e = st_ab[q] + tid + j * nt;
                    if (e < st_ae[q]) {
                        pc[q][j] = __ldg(A.ci + e);
                        if (NUM) pvv[q][j] = ldv(av, e);
                    }
                }
            }
        }
        for (int t0 = 0; t0 < nb; t0 += kDAhead) {
#pragma unroll
            for (int q = 0; q < kDAhead; ++q) {
                const int t = t0 + q;
                if (t < nb) {
                    int col[PER];
                    double v[PER];
                    const int tn = t + kDAhead;
#pragma unroll
                    for (int j = 0; j < PER; ++j) {
                        col[j] = pc[q][j];
                        v[j] = pvv[q][j];
                        pc[q][j] = -1;
                        if (tn < nb) {
                            const int e = st_ab[tn] + tid + j * nt;
                            if (e < st_ae[tn]) {
                                pc[q][j] = __ldg(A.ci + e);
                                if (NUM) pvv[q][j] = ldv(av, e);
                            }
                        }
                    }
                    const int fo = st_fo[t];
                    const double s = NUM ? st_s[t] : 0.0;
#pragma unroll
                    for (int j = 0; j < PER; ++j) {
                        if (col[j] >= cb && col[j] < ce) {
                            const int slot = col[j] - cb;
                            if (!d.touched[slot]) {
                                d.touched[slot] = 1;
                                d.ftq[slot] = fo + tid + j * nt;
                            }
                            if (NUM) d.acc[slot] = __dadd_rn(d.acc[slot], __dmul_rn(v[j], s));
                        }
                    }
                    // Right rows longer than PER entries per thread.
                    const int ab_t = st_ab[t], ae_t = st_ae[t];
                    for (int e = ab_t + tid + PER * nt; e < ae_t; e += nt) {
                        const int c2 = __ldg(A.ci + e);
                        if (c2 >= cb && c2 < ce) {
                            const int slot = c2 - cb;
                            if (!d.touched[slot]) {
                                d.touched[slot] = 1;
                                d.ftq[slot] = fo + (e - ab_t);
                            }
                            if (NUM) d.acc[slot] = __dadd_rn(d.acc[slot], __dmul_rn(ldv(av, e), s));
                        }
                    }
                    // Named barrier 1 over the stepping warps.
                    asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
                }
            }
        }
        __syncthreads();
    }
}

// One output row of C = R*A*P (row `row` of R) by the whole CTA.  `finish`
// runs on thread 0 once the counts are known: finish(n1, n2, fail) returns
// the output offset of the row, or -1 when nothing is to be written (the
// symbolic pass, a failed row, a flagged error).  The exact numeric pass
// writes the row to [ebase, eend) as it goes and calls finish at the end
// to check the count.  Leaves the dense slice clear.
template <int MODE, typename TV, typename TO, class Finish>
__device__ __forceinline__ void dense_row(const DenseSmem& d, const CsrView& R, const CsrView& A,
                                          const CsrView& P, int row, int* oc, TO* ov,
                                          long long ebase, long long eend, Finish&& finish) {
    constexpr bool NUM = MODE != kSymb;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const unsigned lt = lanemask_lt();
    const TV* pv = static_cast<const TV*>(P.v);
    const int rb = __ldg(R.rp + row);
    const int rlen = __ldg(R.rp + row + 1) - rb;
    if (threadIdx.x == 0) {
        *d.s_n1 = 0;
        *d.s_lo = INT_MAX;
        *d.s_hi = -1;
        *d.s_tot = 0;
        *d.s_cnt = 0;
    }
    __syncthreads();
    // Stage-1 span (the A rows' first and last columns) and longest A row.
    int lo = INT_MAX, hi = -1, amax = 0;
    for (int t = threadIdx.x; t < rlen; t += blockDim.x) {
        const int k = __ldg(R.ci + rb + t);
        const int ab = __ldg(A.rp + k), ae = __ldg(A.rp + k + 1);
        amax = max(amax, ae - ab);
        if (ab < ae) {
            lo = min(lo, __ldg(A.ci + ab));
            hi = max(hi, __ldg(A.ci + ae - 1));
        }
    }
    block_span(lo, hi, d.s_lo, d.s_hi);
    amax = static_cast<int>(__reduce_max_sync(kFull, static_cast<unsigned>(amax)));
    if (lane == 0) atomicMax(d.s_cnt, amax);
    __syncthreads();
    const int lo1 = *d.s_lo, hi1 = *d.s_hi;
    const int amax1 = *d.s_cnt;
    const int nw1 = min(kDWarps, max(1, (amax1 + 31) >> 5));
    for (long long c0 = lo1; c0 <= hi1; c0 += kDSpan) {
        const int cb = static_cast<int>(c0);
        const int ce = static_cast<int>(min(static_cast<long long>(hi1) + 1, c0 + kDSpan));
        if (amax1 > 32 * kDWarps)
            dstage1<NUM, 2, TV>(d, R, A, rb, rlen, cb, ce, nw1);
        else
            dstage1<NUM, 1, TV>(d, R, A, rb, rlen, cb, ce, nw1);
        // List the slice's touched columns (value and first touch) and
        // clear them.
        for (int s0 = cb + 32 * wid; s0 < ce; s0 += 32 * kDWarps) {
            const int col = s0 + lane;
            const bool hit = col < ce && d.touched[col - cb];
            const unsigned b = __ballot_sync(kFull, hit);
            int pos0 = 0;
            if (lane == 0 && b) pos0 = atomicAdd(d.s_n1, __popc(b));
            pos0 = __shfl_sync(kFull, pos0, 0);
            if (hit) {
                const int slot = col - cb;
                const int pos = pos0 + __popc(b & lt);
                if (pos < kDList) {
                    d.lkey[pos] = col;
                    d.lq[pos] = d.ftq[slot];
                    if (NUM) d.lval[pos] = d.acc[slot];
                }
                d.touched[slot] = 0;
                if (NUM) d.acc[slot] = 0.0;
            }
        }
        __syncthreads();
    }
    const int n1 = *d.s_n1;
    bool fail = n1 > kDList;
    // First-touch order: sort (position, index) keys.
    if (!fail && n1 > 1) {
        const int P2 = static_cast<int>(next_pow2(static_cast<unsigned>(n1)));
        for (int i = threadIdx.x; i < P2; i += blockDim.x)
            d.sorted[i] = i < n1 ? (static_cast<unsigned long long>(static_cast<unsigned>(d.lq[i]))
                                    << 32) | static_cast<unsigned>(i)
                                 : ~0ULL;
        __syncthreads();
        for (int k = 2; k <= P2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < P2; i += blockDim.x) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const unsigned long long x = d.sorted[i], y = d.sorted[ixj];
                        if ((x > y) == ((i & k) == 0)) {
                            d.sorted[i] = y;
                            d.sorted[ixj] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
    } else if (!fail && n1 == 1 && threadIdx.x == 0) {
        d.sorted[0] = 0;
    }
    if (threadIdx.x == 0) {
        *d.s_lo = INT_MAX;
        *d.s_hi = -1;
        *d.s_tot = 0;
    }
    __syncthreads();
    // Stage-2 span: the P rows' first and last columns.
    lo = INT_MAX;
    hi = -1;
    long long tot = 0;
    if (!fail) {
        for (int t = threadIdx.x; t < n1; t += blockDim.x) {
            const int c = d.lkey[t];
            const int pb = __ldg(P.rp + c), pe = __ldg(P.rp + c + 1);
            tot += pe - pb;
            if (pb < pe) {
                lo = min(lo, __ldg(P.ci + pb));
                hi = max(hi, __ldg(P.ci + pe - 1));
            }
        }
    }
    block_span(lo, hi, d.s_lo, d.s_hi);
    block_total(tot, d.s_tot);
    __syncthreads();
    const int lo2 = *d.s_lo, hi2 = *d.s_hi;
    const long long tot2 = *d.s_tot;
    // The exact pass knows where the row goes: it walks the span in slices
    // and writes each slice's columns in order.  The other passes must know
    // the row's length before booking it: one slice, or the row is retried.
    constexpr bool EXACT = MODE == kNumExact;
    if (!EXACT && hi2 >= lo2 && static_cast<long long>(hi2) - lo2 + 1 > kDSpan) fail = true;
    const bool run2 = !fail && hi2 >= lo2;
    const LeftSorted L2{d.sorted, d.lkey, d.lval};
    long long running = 0;
    for (long long c0 = lo2; run2 ? c0 <= hi2 : c0 == lo2; c0 += kDSpan) {
        const int cb = static_cast<int>(c0);
        const int ce = static_cast<int>(min(static_cast<long long>(hi2) + 1, c0 + kDSpan));
        int wlo2 = 0, whi2 = 0;
        if (run2) {
            balanced_range(d, L2, n1, P.rp, P.ci, cb, ce, tot2, wlo2, whi2);
            daccumulate<NUM>(L2, n1, P.rp, P.ci, pv, wlo2, whi2, cb, d.acc, d.touched, d.sk,
                             d.sv, d.sst);
        }
        __syncthreads();
        int cnt = 0;
        if (run2) {
            for (int s0 = wlo2; s0 < whi2; s0 += 32) {
                const int col = s0 + lane;
                cnt += __popc(__ballot_sync(kFull, col < whi2 && d.touched[col - cb]));
            }
        }
        if (lane == 0) d.s_cnt[wid] = cnt;
        __syncthreads();
        int chunk_n = 0;
        for (int w = 0; w < kDWarps; ++w) chunk_n += d.s_cnt[w];
        if (!EXACT) {
            if (threadIdx.x == 0) *d.s_base = finish(n1, chunk_n, fail);
            __syncthreads();
        }
        if (run2) {
            // Write this warp's columns in order and clear the slice.
            const long long base = EXACT ? ebase + running : *d.s_base;
            long long wpos = base;
            for (int w = 0; w < wid; ++w) wpos += d.s_cnt[w];
            for (int s0 = wlo2; s0 < whi2; s0 += 32) {
                const int col = s0 + lane;
                const bool hit = col < whi2 && d.touched[col - cb];
                const unsigned b = __ballot_sync(kFull, hit);
                if (hit) {
                    const int slot = col - cb;
                    const long long o = wpos + __popc(b & lt);
                    if (NUM && base >= 0 && (!EXACT || o < eend)) {
                        oc[o] = col;
                        stv(ov, o, d.acc[slot]);
                    }
                    d.touched[slot] = 0;
                    if (NUM) d.acc[slot] = 0.0;
                }
                wpos += __popc(b);
            }
        }
        running += chunk_n;
        __syncthreads();
        if (!run2) break;
    }
    if (EXACT && threadIdx.x == 0) finish(n1, static_cast<int>(running), fail);
    __syncthreads();
}

template <int MODE, typename TV, typename TO>
__global__ void __launch_bounds__(kDWarps * 32, SP3MM_DENSE_MINB)
    k_direct_dense(DirectRowArgs a, RowParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_n1, s_lo, s_hi, s_cnt[kDWarps];
    __shared__ long long s_base;
    const DenseSmem d = dense_smem(smem, &s_n1, &s_lo, &s_hi, s_cnt, &s_base);
    dense_clear(d);
    int* oc = MODE == kNumBook ? p.ub_ci : p.c_ci;
    TO* ov = static_cast<TO*>(MODE == kNumBook ? p.ub_v : p.c_v);
    const long long nrows = p.nrows_dev ? *p.nrows_dev : p.nrows;
    for (long long it = blockIdx.x; it < nrows; it += gridDim.x) {
        const int row = p.rows[it];
        const long long eb = MODE == kNumExact ? p.c_rp[row] : 0;
        const long long ee = MODE == kNumExact ? p.c_rp[row + 1] : 0;
        dense_row<MODE, TV, TO>(d, a.R, a.A, a.P, row, oc, ov, eb, ee,
                                [&](int n1, int n2, bool fail) -> long long {
            if (fail) {
                if (p.retry_rows) p.retry_rows[atomicAdd(p.retry_count, 1)] = row;
                else atomicOr(p.err, kErrTable);
                return -1;
            }
            if (MODE == kSymb) {
                p.row_cnt[row] = n2;
                if (p.row_cnt1) p.row_cnt1[row] = n1;
                return -1;
            }
            if (MODE == kNumBook) {
                const unsigned long long off =
                    n2 > 0 ? atomicAdd(p.cursor, static_cast<unsigned long long>(n2)) : 0ULL;
                if (off + n2 > p.cap) {
                    atomicOr(p.err, kErrBook);
                    return -1;
                }
                p.row_off[row] = static_cast<long long>(off);
                p.row_cnt[row] = n2;
                return static_cast<long long>(off);
            }
            if (ee - eb != n2) atomicOr(p.err, kErrCount);
            return -1;
        });
    }
}

}  // namespace SP3MM_DENSE_NS
}  // namespace sp3mm
