// batch.cu -- many independent products in one binned, persistent pass.
//
// The reference computes one product per call, each an OpenMP region over
// that product's rows (code/src/Sp3MM_CSR_OMP_UB_Generic.c:498-573 for the
// direct triple product, :56-124 and code/src/Sp3MM_CSR_OMP_Num_Generic.c:
// 93-146 for SpMM).  An AMG setup over many operators (hierarchy levels,
// independent systems) calls it once per product; on a GPU each small call
// then pays its own launches and host round trips and fills a fraction of
// the 148 SMs.  A batch instead concatenates the rows of all its products
// into one row space and runs the whole set as one product:
//
//   plan     bounds of every row -> binning by table level -> persistent
//            symbolic launches (optimistic tables, in-kernel retry with the
//            proven size, global-memory tables for the rest) -> one scan of
//            the row counts -> exact binning -> output allocation, and the
//            numeric pass captured once as a CUDA graph;
//   execute  one replay of that graph: each tier of table levels is one
//            persistent launch, the tiers run as parallel graph branches.
//
// The plan needs four host round trips per batch, not per product; execute
// needs none and can be replayed whenever the operands' values change but
// their patterns and addresses do not (numeric re-setup).  Results are
// bit-identical to the single-product entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "batch.cuh"
#include "context.cuh"
#include "sp3mm_b200.h"

using namespace sp3mm;

namespace {

// need[g] = distinct-key bound of the first table of global row g (the
// product count of its row of X*Y, at most Y.N); row_item[g] = its product.
// *total += the output-size bound of every row (SpMM: need; direct:
// min(R*A products times Z's longest row, Z.N)).  need_opt[g] = the
// optimistic first-table size: need >> d1 capped at 8 sqrt(products) (long
// rows repeat their columns; the single-product bound kernel uses the same
// guess), or need itself when the row's products reach Y's column count
// (such rows are dense).
__global__ void k_batch_bounds(const BItem* __restrict__ items, const long long* __restrict__ bases,
                               int n, long long rows, int d1, int* need, int* need_opt,
                               int* row_item, unsigned long long* total) {
    unsigned long long ub = 0;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n;   // largest b with bases[b] <= g; bases[n] = rows
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(bases + mid) <= g) lo = mid;
            else hi = mid;
        }
        const BItem* I = items + lo;
        const int i = static_cast<int>(g - I->row_base);
        const int* xrp = I->X.rp;
        const int* xci = I->X.ci;
        const int* yrp = I->Y.rp;
        long long u = 0;
        for (int t = __ldg(xrp + i); t < __ldg(xrp + i + 1); ++t) {
            const int k = __ldg(xci + t);
            u += __ldg(yrp + k + 1) - __ldg(yrp + k);
        }
        const int nd = static_cast<int>(u < I->Y.N ? u : I->Y.N);
        need[g] = nd;
        // (a positive bound stays positive: binning skips rows of need 0)
        long long o = nd >> d1;
        const long long r = static_cast<long long>(ceil(8.0 * sqrt(static_cast<double>(u))));
        if (r < o) o = r;
        need_opt[g] = nd == 0 ? 0 : (u >= I->Y.N ? nd : max(1, static_cast<int>(o)));
        row_item[g] = lo;
        if (I->kind == kBatchDirect) {
            const long long zm = I->zmax >= 0 ? I->zmax : I->Z.N;
            const long long b2 = u * zm;
            ub += static_cast<unsigned long long>(b2 < I->Z.N ? b2 : I->Z.N);
        } else {
            ub += static_cast<unsigned long long>(u < I->Y.N ? u : I->Y.N);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ub += __shfl_xor_sync(0xffffffffu, ub, o);
    if ((threadIdx.x & 31) == 0 && ub) atomicAdd(total, ub);
}

// Per-product output offset and length from the global row pointers.
__global__ void k_batch_item_spans(const BItem* __restrict__ items, int n, const int* crp,
                                   long long* span) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const long long g0 = items[b].row_base, g1 = g0 + items[b].M;
    span[2 * b] = crp[g0];
    span[2 * b + 1] = static_cast<long long>(crp[g1]) - crp[g0];
}

// Longest C row of every product (span[2n + b]), from the row counts.
__global__ void k_batch_item_max(const int* __restrict__ row_item, long long rows,
                                 const int* cnt, long long* span_max) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         g - threadIdx.x % 32 < rows; g += (long long)gridDim.x * blockDim.x) {
        const bool in = g < rows;
        const int b = in ? row_item[g] : -1;
        int m = in ? cnt[g] : 0;
        // Lanes of one product reduce together; one atomic per product.
        const unsigned same = __match_any_sync(0xffffffffu, b);
        m = static_cast<int>(__reduce_max_sync(same, static_cast<unsigned>(m)));
        if (in && (threadIdx.x & 31) == __ffs(same) - 1 && m > 0)
            atomicMax(reinterpret_cast<unsigned long long*>(span_max + b),
                      static_cast<unsigned long long>(m));
    }
}

// Local row pointers of every product: rp_local[rp_off[b] + i] =
// crp[row_base + i] - crp[row_base] for i = 0..M (the arrays of empty
// products are zeroed by the caller).
__global__ void k_batch_local_rp(const BItem* __restrict__ items, const int* __restrict__ row_item,
                                 const long long* __restrict__ rp_off, long long rows,
                                 const int* crp, int* rp_local) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const int b = row_item[g];
        const long long base = items[b].row_base;
        const int i = static_cast<int>(g - base);
        const int c0 = crp[base];
        int* out = rp_local + rp_off[b];
        out[i] = crp[g] - c0;
        if (i == items[b].M - 1) out[i + 1] = crp[g + 1] - c0;
    }
}

int grid_for_rows(long long rows) {
    long long g = (rows + 255) / 256;
    return static_cast<int>(std::max<long long>(1, std::min<long long>(g, 148LL * 32)));
}

}  // namespace

// A tier: a contiguous range of table levels run by one persistent launch.
struct BatchTier {
    int lo = 0, hi = 0;      // levels [lo, hi]
    int first = 0, count = 0;   // rows: lists[first, first + count)
    int scap = 0;
    int slack = 0;           // numeric: tables 2^slack times the exact size
    bool gt = false;
    bool dense = false;      // one CTA per row, dense accumulators (heavy direct rows)
    int block = 0, grid = 0;
    size_t smem = 0;
};

struct sp3mm_batch {
    sp3mm_ctx* ctx = nullptr;
    std::vector<BItem> items;
    std::vector<long long> bases;   // n + 1 row offsets
    long long rows = 0;
    int tv = SP3MM_F64, to = SP3MM_F64;
    // Tuning: symbolic shifts, numeric slack, tier split levels (a new tier
    // starts at each listed level; empty: one tier per non-empty level).
    int d1 = 2, d2 = 1, slack = 0;
    int flavour = SP3MM_UB;        // UB: booked numeric plan; SYMBNUM: symbolic plan
    bool values_ready = false;     // the plan computed the values (UB)
    bool trimmed = false;
    std::vector<int> splits;
    bool auto_split = true;
    std::vector<int> level_slack = std::vector<int>(kLevels, -1);   // per top level; -1: slack
    int warps_cap = 8;
    // Tiers whose per-warp tables exceed this go to global memory, where
    // more warps per SM run (one or two warps per SM hide no latency).
    size_t smem_tier_max = 110 * 1024;
    // Device state.
    DevBuf d_items, d_bases, d_row_item, d_need, d_need_opt, d_cnt1, d_cnt2, d_crp;
    DevBuf d_ci, d_v, d_rp, d_rp_off, d_counters;
    DevBuf num_gtab;
    Bins nbins;
    std::vector<BatchTier> tiers;
    std::vector<long long> rp_off;
    std::vector<sp3mm_dcsr> results;
    long long nnz = 0;
    long long retried = 0;   // rows of the last plan redone with proven tables
    bool planned = false;
    // Numeric graph (tiers as parallel branches).
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> events;
    int graph_kernels = 0;

    ~sp3mm_batch() { drop_graph(); }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        for (auto s : branch) cudaStreamDestroy(s);
        for (auto e : events) cudaEventDestroy(e);
        branch.clear();
        events.clear();
    }
};

namespace {

int batch_fail(sp3mm_batch* b, int code, const char* msg) {
    return set_error(b ? b->ctx : nullptr, code, "batch: %s", msg);
}

}  // namespace

namespace {

// Rows binned to tables of at least this many slots (thousands of distinct
// columns) run on the CTA-per-row kernel in all-direct batches.
constexpr int kBatchDenseMinSlots = 2048;
// Exact pass: table levels up to this size hold at most 3584 distinct R*A
// columns per row, within the CTA's 4096-entry list.
constexpr int kBatchDenseMaxSlots = 4096;

// Tiers over the non-empty levels of `bins`.  A tier's tables hold
// 32 << (its top level + extra) slots per warp (extra: the numeric slack,
// or the symbolic shift d1 so that a proven-size retry still fits).  Tiers
// whose region does not fit one CTA's shared memory merge into one
// global-memory tier.
int make_tiers(sp3mm_batch* b, const Bins& bins, int mode, int extra, int tv, int to,
               std::vector<BatchTier>& out) {
    sp3mm_ctx* ctx = b->ctx;
    out.clear();
    const bool num = mode != kSymb;
    BatchTier gt;
    gt.gt = true;
    gt.lo = kLevels;
    gt.hi = -1;
    // Heavy levels of an all-direct batch run one CTA per row: in the
    // symbolic and booked passes, whose retry rounds take the rows it cannot
    // hold; in the exact numeric pass (no retries), the levels of at most
    // kBatchDenseMaxSlots, whose exact counts fit its R*A list.
    bool all_direct = !b->items.empty();
    for (const BItem& I : b->items) all_direct = all_direct && I.kind == kBatchDirect;
    const bool dense_ok = all_direct && batch_dense_smem() + 1024 <= ctx->smem_optin;
    auto tier_of = [&](int L) {
        if (b->auto_split) return L;
        int t = 0;
        for (int s : b->splits)
            if (L >= s) ++t;
        return t;
    };
    int L = 0;
    while (L < kLevels) {
        if (!bins.counts[L]) {
            ++L;
            continue;
        }
        BatchTier t;
        t.lo = t.hi = L;
        const int id = tier_of(L);
        int M = L + 1;
        while (M < kLevels && tier_of(M) == id) {
            if (bins.counts[M]) t.hi = M;
            ++M;
        }
        t.first = bins.offsets[t.lo];
        t.count = bins.offsets[t.hi] + bins.counts[t.hi] - t.first;
        int ex = extra;
        if (mode == kNumExact) {
            ex = b->level_slack[t.hi] >= 0 ? b->level_slack[t.hi] : b->slack;
            t.slack = ex;
        }
        const int top = std::min(t.hi + ex, 30 - 5);
        t.scap = 32 << top;
        const long long slots = 32LL << std::min(t.hi, 25);
        if (dense_ok && slots >= kBatchDenseMinSlots &&
            (mode != kNumExact || slots <= kBatchDenseMaxSlots)) {
            t.dense = true;
            t.block = 512;
            t.smem = batch_dense_smem();
            t.grid = static_cast<int>(std::min<long long>(t.count, ctx->num_sms));
            out.push_back(t);
            L = M;
            continue;
        }
        const size_t bytes = batch_row_region_bytes(num, t.scap);
        if (bytes > std::min(ctx->smem_optin, b->smem_tier_max)) {
            // Global-memory tier: extend it (levels are visited ascending).
            if (gt.hi < 0) {
                gt.lo = t.lo;
                gt.first = t.first;
            }
            gt.hi = t.hi;
            gt.count = bins.offsets[t.hi] + bins.counts[t.hi] - gt.first;
            gt.scap = t.scap;
            gt.slack = t.slack;
            L = M;
            continue;
        }
        int w = static_cast<int>(std::min<size_t>(b->warps_cap, ctx->smem_optin / bytes));
        w = std::max(1, w);
        t.block = 32 * w;
        t.smem = bytes * w;
        int per_sm = 0;
        CK(ctx, batch_rows_configure(mode, false, tv, to, t.block, t.smem, ctx->smem_optin,
                                     &per_sm));
        per_sm = std::max(1, per_sm);
        const long long need_ctas = (t.count + w - 1) / w;
        t.grid = static_cast<int>(std::min<long long>(need_ctas, 1LL * per_sm * ctx->num_sms));
        out.push_back(t);
        L = M;
    }
    if (gt.hi >= 0) {
        const size_t stride = (batch_row_region_bytes(num, gt.scap) + 255) / 256 * 256;
        long long warps = std::min<long long>(gt.count, 8LL * ctx->num_sms);
        const size_t budget = size_t(2) << 30;
        while (warps > 1 && static_cast<size_t>(warps) * stride > budget) warps >>= 1;
        const int w = static_cast<int>(std::min<long long>(8, warps));
        gt.block = 32 * w;
        gt.grid = static_cast<int>((warps + w - 1) / w);
        gt.smem = stride;   // per-warp stride (the launch uses no shared memory)
        out.push_back(gt);
    }
    return SP3MM_OK;
}

size_t gt_bytes(const BatchTier& t) {
    return static_cast<size_t>(t.grid) * (t.block / 32) * t.smem;
}

// Launch the tiers; with several, tier 0 runs on the context stream and the
// others on branch streams forked from it and joined back (parallel graph
// branches when captured).
int run_tiers(sp3mm_batch* b, int mode, const std::vector<BatchTier>& tiers, const int* lists,
              BatchRowParams base, unsigned char* gtab) {
    sp3mm_ctx* ctx = b->ctx;
    const cudaStream_t st = ctx->stream;
    const int nt = static_cast<int>(tiers.size());
    while (static_cast<int>(b->branch.size()) < nt - 1) {
        cudaStream_t s;
        CK(ctx, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        b->branch.push_back(s);
    }
    while (static_cast<int>(b->events.size()) < nt) {
        cudaEvent_t e;
        CK(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->events.push_back(e);
    }
    if (nt > 1) CK(ctx, cudaEventRecord(b->events[0], st));
    for (int k = 0; k < nt; ++k) {
        const BatchTier& t = tiers[k];
        const cudaStream_t s = k == 0 ? st : b->branch[k - 1];
        if (k > 0) CK(ctx, cudaStreamWaitEvent(s, b->events[0], 0));
        BatchRowParams p = base;
        p.rows = lists + t.first;
        p.nrows = t.count;
        p.scap = t.scap;
        if (mode == kNumExact) p.slack = t.slack;
        p.reverse = t.hi > t.lo ? 1 : 0;
        size_t smem = t.smem;
        if (t.gt) {
            p.gtab = gtab;
            p.gstride = static_cast<long long>(t.smem);
            smem = 0;
        }
        if (t.dense)
            CK(ctx, launch_batch_dense(mode, b->tv, b->to, t.grid, s, b->d_items.as<BItem>(),
                                       b->d_row_item.as<int>(), p));
        else
            CK(ctx, launch_batch_rows(mode, t.gt, b->tv, b->to, t.grid, t.block, smem, s,
                                      b->d_items.as<BItem>(), b->d_row_item.as<int>(), p));
        if (k > 0) {
            CK(ctx, cudaEventRecord(b->events[k], s));
            CK(ctx, cudaStreamWaitEvent(st, b->events[k], 0));
        }
    }
    return SP3MM_OK;
}

// Numeric tiers, their global-memory tables and the captured graph.
int build_numeric(sp3mm_batch* b) {
    sp3mm_ctx* ctx = b->ctx;
    const cudaStream_t st = ctx->stream;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    TRY(make_tiers(b, b->nbins, kNumExact, b->slack, b->tv, b->to, b->tiers));
    size_t need_gt = 0;
    for (const auto& t : b->tiers)
        if (t.gt) need_gt = gt_bytes(t);
    b->num_gtab.release();
    if (need_gt) TRY(b->num_gtab.alloc(ctx, need_gt));
    BatchRowParams p{};
    p.slack = b->slack;
    p.cnt1 = b->d_cnt1.as<int>();
    p.cnt2 = b->d_cnt2.as<int>();
    p.c_rp = b->d_crp.as<int>();
    p.c_ci = b->d_ci.as<int>();
    p.c_v = b->d_v.p;
    p.err = ctx->d_err;
    // Create branch streams and events before capture begins.
    const int nt = static_cast<int>(b->tiers.size());
    while (static_cast<int>(b->branch.size()) < nt - 1) {
        cudaStream_t s;
        CK(ctx, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        b->branch.push_back(s);
    }
    while (static_cast<int>(b->events.size()) < nt) {
        cudaEvent_t e;
        CK(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->events.push_back(e);
    }
    CK(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = run_tiers(b, kNumExact, b->tiers, b->nbins.lists.as<int>(), p,
                             b->num_gtab.as<unsigned char>());
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != SP3MM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    CK(ctx, e);
    b->graph = g;
    CK(ctx, cudaGraphInstantiate(&b->exec, g, 0));
    b->graph_kernels = nt;
    return SP3MM_OK;
}

}  // namespace

namespace {

// The row pass of a plan -- symbolic (kSymb) or booked numeric (kNumBook):
// tiers of the optimistic levels of `sb`, then rounds for the rows whose
// proven tables exceed their tier, with global-memory tables sized from the
// largest proven bound (a direct row learns its second bound only once its
// first table is complete, hence up to three rounds).
int row_pass(sp3mm_batch* b, int mode, const Bins& sb, BatchRowParams p, int* rinfo,
             const char* label) {
    sp3mm_ctx* ctx = b->ctx;
    const cudaStream_t st = ctx->stream;
    const bool num = mode != kSymb;
    const size_t R1 = static_cast<size_t>(b->rows) + 1;
    std::vector<BatchTier> tiers;
    TRY(make_tiers(b, sb, mode, num ? 0 : b->d1, b->tv, b->to, tiers));
    DevBuf retry_a, retry_b, gtab;
    TRY(retry_a.alloc(ctx, sizeof(int) * R1));
    TRY(retry_b.alloc(ctx, sizeof(int) * R1));
    size_t gb = 0;
    for (const auto& t : tiers)
        if (t.gt) gb = gt_bytes(t);
    if (gb) TRY(gtab.alloc(ctx, gb));
    CK(ctx, cudaMemsetAsync(rinfo, 0, 2 * sizeof(int), st));
    p.retry_rows = retry_a.as<int>();
    p.retry_count = rinfo;
    p.retry_need = rinfo + 1;
    if (!tiers.empty()) {
        int rc = SP3MM_OK;
        prof(ctx, label, [&] {
            rc = run_tiers(b, mode, tiers, sb.lists.as<int>(), p, gtab.as<unsigned char>());
        });
        TRY(rc);
    }
    int* cur = retry_a.as<int>();
    int* nxt = retry_b.as<int>();
    for (int round = 0;; ++round) {
        int h[2] = {0, 0};
        CK(ctx, cudaMemcpyAsync(h, rinfo, sizeof h, cudaMemcpyDeviceToHost, st));
        CK(ctx, cudaStreamSynchronize(st));
        if (h[0] == 0) break;
        if (round == 3) return batch_fail(b, SP3MM_EDEVICE, "row retries did not converge");
        b->retried += h[0];
        CK(ctx, cudaMemsetAsync(rinfo, 0, 2 * sizeof(int), st));
        BatchTier t;
        t.gt = true;
        t.first = 0;
        t.count = h[0];
        t.scap = batch_slots_for(h[1]);
        const size_t stride = (batch_row_region_bytes(num, t.scap) + 255) / 256 * 256;
        long long warps = std::min<long long>(h[0], 8LL * ctx->num_sms);
        while (warps > 1 && static_cast<size_t>(warps) * stride > (size_t(2) << 30)) warps >>= 1;
        const int w = static_cast<int>(std::min<long long>(8, warps));
        t.block = 32 * w;
        t.grid = static_cast<int>((warps + w - 1) / w);
        t.smem = stride;
        DevBuf g;
        TRY(g.alloc(ctx, gt_bytes(t)));
        BatchRowParams q = p;
        q.retry_rows = nxt;
        std::vector<BatchTier> one{t};
        int rc = SP3MM_OK;
        prof(ctx, label, [&] { rc = run_tiers(b, mode, one, cur, q, g.as<unsigned char>()); });
        TRY(rc);
        std::swap(cur, nxt);
    }
    return SP3MM_OK;
}

// Exact binning of the rows by max(R*A, C) row counts and the numeric graph.
int ensure_numeric(sp3mm_batch* b) {
    if (b->exec) return SP3MM_OK;
    sp3mm_ctx* ctx = b->ctx;
    Counters* dc = b->d_counters.as<Counters>() + 1;
    CK(ctx, cudaMemsetAsync(dc, 0, sizeof(Counters), ctx->stream));
    const int M = static_cast<int>(b->rows);
    if (M > 0)
        launch_need_from_counts(M, b->d_cnt2.as<int>(), b->d_cnt1.as<int>(), b->d_need.as<int>(),
                                ctx->stream);
    TRY(bin_rows(ctx, M, b->d_need.as<int>(), 0, 32, dc, nullptr, b->nbins));
    ProfSpan span(ctx, "batch.graph");
    return build_numeric(b);
}

int batch_plan(sp3mm_batch* b) {
    sp3mm_ctx* ctx = b->ctx;
    ProfSpan whole(ctx, "batch.plan");
    const cudaStream_t st = ctx->stream;
    const int n = static_cast<int>(b->items.size());
    const long long rows = b->rows;
    const int M = static_cast<int>(rows);
    const size_t R1 = static_cast<size_t>(rows) + 1;
    b->planned = false;
    b->values_ready = false;
    b->retried = 0;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->results.assign(n, sp3mm_dcsr{});
    TRY(b->d_items.alloc(ctx, sizeof(BItem) * n));
    TRY(b->d_bases.alloc(ctx, sizeof(long long) * (n + 1)));
    CK(ctx, cudaMemcpyAsync(b->d_items.p, b->items.data(), sizeof(BItem) * n,
                            cudaMemcpyHostToDevice, st));
    CK(ctx, cudaMemcpyAsync(b->d_bases.p, b->bases.data(), sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, st));
    TRY(b->d_row_item.alloc(ctx, sizeof(int) * R1));
    TRY(b->d_need.alloc(ctx, sizeof(int) * R1));
    TRY(b->d_need_opt.alloc(ctx, sizeof(int) * R1));
    TRY(b->d_cnt1.alloc(ctx, sizeof(int) * R1));
    TRY(b->d_cnt2.alloc(ctx, sizeof(int) * R1));
    TRY(b->d_crp.alloc(ctx, sizeof(int) * R1));
    const size_t cbytes = sizeof(Counters) * 2 + 4 * sizeof(int);
    TRY(b->d_counters.alloc(ctx, cbytes));
    Counters* dc = b->d_counters.as<Counters>();
    int* rinfo = reinterpret_cast<int*>(dc + 2);   // retry count, retry need
    CK(ctx, cudaMemsetAsync(b->d_cnt1.p, 0, sizeof(int) * R1, st));
    CK(ctx, cudaMemsetAsync(b->d_cnt2.p, 0, sizeof(int) * R1, st));
    CK(ctx, cudaMemsetAsync(b->d_counters.p, 0, cbytes, st));
    if (rows > 0) {
        prof(ctx, "batch.bounds", [&] {
            k_batch_bounds<<<grid_for_rows(rows), 256, 0, st>>>(
                b->d_items.as<BItem>(), b->d_bases.as<long long>(), n, rows, b->d1,
                b->d_need.as<int>(), b->d_need_opt.as<int>(), b->d_row_item.as<int>(),
                &dc->total);
        });
        note_launch();
        CK(ctx, cudaGetLastError());
    }
    Bins sb;
    TRY(bin_rows(ctx, M, b->d_need_opt.as<int>(), 0, 32, dc, nullptr, sb));

    BatchRowParams p{};
    p.d1 = b->d1;
    p.d2 = b->d2;
    p.need = b->d_need.as<int>();
    p.need_opt = b->d_need_opt.as<int>();
    p.cnt1 = b->d_cnt1.as<int>();
    p.cnt2 = b->d_cnt2.as<int>();
    p.err = ctx->d_err;
    bool booked = false;
    DevBuf ub_ci, ub_v, row_off, cursor;
    if (b->flavour == SP3MM_UB && rows > 0) {
        // One numeric pass: every row books its exact length from one
        // cursor, in space bounded by the output bound, by twice the
        // operands' nonzeros and by half the free memory (a batch that
        // overflows it is planned symbolically instead).  Galerkin products
        // and their A*P0 steps write well under their operands' nonzeros;
        // reserving more made the pool map tens of GB for a batch of large
        // hierarchies' first levels.
        const size_t eb = sizeof(int) + vbytes(b->to);
        long long in_nnz = 0;
        for (const BItem& I : b->items)
            in_nnz += I.X.nnz + I.Y.nnz + (I.kind == kBatchDirect ? I.Z.nnz : 0);
        unsigned long long cap = std::min<unsigned long long>(
            sb.total, std::max<unsigned long long>(1ULL << 20, 2ULL * in_nnz));
        if (cap * eb > (size_t(1) << 30) && pool_idle_bytes(ctx) < cap * eb)
            cap = std::min<unsigned long long>(
                cap, std::max<unsigned long long>(1ULL << 20, free_device_bytes(ctx) / 2 / eb));
        TRY(ub_ci.alloc(ctx, sizeof(int) * std::max<unsigned long long>(cap, 1)));
        TRY(ub_v.alloc(ctx, vbytes(b->to) * std::max<unsigned long long>(cap, 1)));
        TRY(row_off.alloc(ctx, sizeof(long long) * R1));
        TRY(cursor.alloc(ctx, sizeof(unsigned long long)));
        CK(ctx, cudaMemsetAsync(cursor.p, 0, sizeof(unsigned long long), st));
        BatchRowParams q = p;
        q.cursor = cursor.as<unsigned long long>();
        q.cap = cap;
        q.row_off = row_off.as<long long>();
        q.ub_ci = ub_ci.as<int>();
        q.ub_v = ub_v.p;
        TRY(row_pass(b, kNumBook, sb, q, rinfo, "batch.book"));
        unsigned e = 0;
        TRY(read_err(ctx, &e));
        if (e != 0 && e != kErrBook) return check_device_err(ctx);
        if (e == kErrBook) {
            // The booking space ran out: plan this batch symbolically.
            CK(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), st));
            CK(ctx, cudaMemsetAsync(b->d_cnt1.p, 0, sizeof(int) * R1, st));
            CK(ctx, cudaMemsetAsync(b->d_cnt2.p, 0, sizeof(int) * R1, st));
        } else {
            booked = true;
        }
    }
    if (!booked && rows > 0) TRY(row_pass(b, kSymb, sb, p, rinfo, "batch.symbolic"));

    // Row pointers of the whole batch, product spans and longest rows.
    DevBuf tmp, span;
    const size_t tb = scan_temp_bytes(M);
    TRY(tmp.alloc(ctx, tb));
    TRY(span.alloc(ctx, sizeof(long long) * 3 * (n + 1)));
    if (rows > 0) {
        prof(ctx, "batch.scan", [&] {
            launch_scan(M, b->d_cnt2.as<int>(), b->d_crp.as<int>(), tmp.p, tb, st);
        });
    } else {
        CK(ctx, cudaMemsetAsync(b->d_crp.p, 0, sizeof(int), st));
    }
    CK(ctx, cudaGetLastError());
    std::vector<long long> hspan(3 * static_cast<size_t>(n) + 3, 0);
    if (n > 0) {
        k_batch_item_spans<<<(n + 255) / 256, 256, 0, st>>>(b->d_items.as<BItem>(), n,
                                                           b->d_crp.as<int>(),
                                                           span.as<long long>());
        CK(ctx, cudaMemsetAsync(span.as<long long>() + 2 * n, 0, sizeof(long long) * n, st));
        if (rows > 0)
            k_batch_item_max<<<grid_for_rows(rows), 256, 0, st>>>(
                b->d_row_item.as<int>(), rows, b->d_cnt2.as<int>(), span.as<long long>() + 2 * n);
        note_launch();
        note_launch();
        CK(ctx, cudaGetLastError());
        CK(ctx, cudaMemcpyAsync(hspan.data(), span.p, sizeof(long long) * 3 * n,
                                cudaMemcpyDeviceToHost, st));
    }
    TRY(check_device_err(ctx));   // synchronises: hspan is complete
    long long nnz = 0;
    for (int i = 0; i < n; ++i) nnz += hspan[2 * i + 1];
    if (nnz >= INT32_MAX) return batch_fail(b, SP3MM_ELIMIT, "the batch has too many nonzeros");
    b->nnz = nnz;

    // Outputs: one array of columns and values for the batch, one array of
    // local row pointers per product.
    TRY(b->d_ci.alloc(ctx, sizeof(int) * static_cast<size_t>(nnz)));
    TRY(b->d_v.alloc(ctx, vbytes(b->to) * static_cast<size_t>(nnz)));
    b->rp_off.assign(n, 0);
    long long rp_total = 0;
    for (int i = 0; i < n; ++i) {
        b->rp_off[i] = rp_total;
        rp_total += b->items[i].M + 1;
    }
    TRY(b->d_rp.alloc(ctx, sizeof(int) * static_cast<size_t>(rp_total)));
    TRY(b->d_rp_off.alloc(ctx, sizeof(long long) * std::max(n, 1)));
    CK(ctx, cudaMemsetAsync(b->d_rp.p, 0, sizeof(int) * static_cast<size_t>(rp_total), st));
    if (n > 0)
        CK(ctx, cudaMemcpyAsync(b->d_rp_off.p, b->rp_off.data(), sizeof(long long) * n,
                                cudaMemcpyHostToDevice, st));
    if (rows > 0) {
        k_batch_local_rp<<<grid_for_rows(rows), 256, 0, st>>>(
            b->d_items.as<BItem>(), b->d_row_item.as<int>(), b->d_rp_off.as<long long>(), rows,
            b->d_crp.as<int>(), b->d_rp.as<int>());
        note_launch();
        CK(ctx, cudaGetLastError());
    }
    if (booked) {
        prof(ctx, "batch.compact", [&] {
            launch_compact(M, b->d_cnt2.as<int>(), row_off.as<long long>(), ub_ci.as<int>(),
                           ub_v.p, b->d_crp.as<int>(), b->d_ci.as<int>(), b->d_v.p, b->to, st);
        });
        CK(ctx, cudaGetLastError());
    }
    for (int i = 0; i < n; ++i) {
        sp3mm_dcsr& C = b->results[i];
        C.M = b->items[i].M;
        C.N = b->items[i].N;
        C.nnz = hspan[2 * i + 1];
        C.row_ptr = b->d_rp.as<int>() + b->rp_off[i];
        C.col = b->d_ci.as<int>() + hspan[2 * i];
        C.val = static_cast<unsigned char*>(b->d_v.p) + vbytes(b->to) * hspan[2 * i];
        C.val_type = b->to;
        C.max_row = static_cast<int>(hspan[2 * static_cast<size_t>(n) + i]);
    }
    b->values_ready = booked || rows == 0;
    if (!booked) TRY(ensure_numeric(b));
    b->planned = true;
    return SP3MM_OK;
}

int check_operand(sp3mm_ctx* ctx, const sp3mm_dcsr& m, int tv, const char* what) {
    TRY(check_dcsr(ctx, &m, what));
    if (m.val_type != tv)
        return set_error(ctx, SP3MM_EINVAL, "batch: %s has another value type", what);
    return SP3MM_OK;
}

}  // namespace

namespace sp3mm {

void batch_trim(sp3mm_batch* b) {
    b->trimmed = true;
    b->drop_graph();
    b->tiers.clear();
    b->d_items.release();
    b->d_bases.release();
    b->d_row_item.release();
    b->d_need.release();
    b->d_need_opt.release();
    b->d_cnt1.release();
    b->d_cnt2.release();
    b->d_crp.release();
    b->d_rp_off.release();
    b->d_counters.release();
    b->num_gtab.release();
    b->nbins.level.release();
    b->nbins.lists.release();
}

}  // namespace sp3mm

extern "C" {

int sp3mm_batch_create(sp3mm_ctx* ctx, int n, const int* kinds, const sp3mm_dcsr* X,
                       const sp3mm_dcsr* Y, const sp3mm_dcsr* Z, int out_val_type,
                       sp3mm_batch** out) {
    if (!ctx || !out || n < 0 || (n > 0 && (!kinds || !X || !Y)))
        return set_error(ctx, SP3MM_EINVAL, "batch: invalid arguments");
    if (out_val_type != SP3MM_F64 && out_val_type != SP3MM_F32)
        return set_error(ctx, SP3MM_EINVAL, "batch: unknown output value type");
    auto* b = new sp3mm_batch();
    b->ctx = ctx;
    b->to = out_val_type;
    b->tv = n > 0 ? X[0].val_type : SP3MM_F64;
    b->items.resize(n);
    b->bases.assign(n + 1, 0);
    long long rows = 0;
    for (int i = 0; i < n; ++i) {
        BItem& I = b->items[i];
        int rc = SP3MM_OK;
        if (kinds[i] != SP3MM_BATCH_SPMM && kinds[i] != SP3MM_BATCH_RAP)
            rc = set_error(ctx, SP3MM_EINVAL, "batch: product %d has an unknown kind", i);
        if (rc == SP3MM_OK) rc = check_operand(ctx, X[i], b->tv, "X");
        if (rc == SP3MM_OK) rc = check_operand(ctx, Y[i], b->tv, "Y");
        if (rc == SP3MM_OK && X[i].N != Y[i].M)
            rc = set_error(ctx, SP3MM_EINVAL, "batch: product %d: X.N != Y.M", i);
        if (rc == SP3MM_OK && kinds[i] == SP3MM_BATCH_RAP) {
            if (!Z) rc = set_error(ctx, SP3MM_EINVAL, "batch: product %d needs Z", i);
            if (rc == SP3MM_OK) rc = check_operand(ctx, Z[i], b->tv, "Z");
            if (rc == SP3MM_OK && Y[i].N != Z[i].M)
                rc = set_error(ctx, SP3MM_EINVAL, "batch: product %d: Y.N != Z.M", i);
        }
        if (rc != SP3MM_OK) {
            delete b;
            return rc;
        }
        I.X = view(X[i]);
        I.Y = view(Y[i]);
        I.kind = kinds[i] == SP3MM_BATCH_RAP ? kBatchDirect : kBatchPair;
        if (I.kind == kBatchDirect) I.Z = view(Z[i]);
        else I.Z = CsrView{};
        I.zmax = I.kind == kBatchDirect ? Z[i].max_row : -1;
        I.M = X[i].M;
        I.N = I.kind == kBatchDirect ? Z[i].N : Y[i].N;
        I.row_base = rows;
        b->bases[i] = rows;
        rows += X[i].M;
    }
    b->bases[n] = rows;
    if (rows >= INT32_MAX) {
        delete b;
        return set_error(ctx, SP3MM_ELIMIT, "batch: too many rows");
    }
    b->rows = rows;
    *out = b;
    return SP3MM_OK;
}

int sp3mm_batch_set_tuning(sp3mm_batch* b, int d1, int d2, int slack, int nsplits,
                           const int32_t* splits) {
    if (!b || d1 < 0 || d1 > 8 || d2 < 0 || d2 > 8 || slack < 0 || slack > 3 ||
        (nsplits > 0 && !splits))
        return batch_fail(b, SP3MM_EINVAL, "invalid tuning");
    b->d1 = d1;
    b->d2 = d2;
    const bool numeric_changed =
        slack != b->slack || (nsplits < 0) != b->auto_split ||
        (nsplits >= 0 && std::vector<int>(splits, splits + nsplits) != b->splits);
    b->slack = slack;
    b->auto_split = nsplits < 0;
    b->splits.assign(splits && nsplits > 0 ? splits : nullptr,
                     splits && nsplits > 0 ? splits + nsplits : nullptr);
    if (b->exec && numeric_changed) return build_numeric(b);
    return SP3MM_OK;
}

int sp3mm_batch_set_flavour(sp3mm_batch* b, int flavour) {
    if (!b || (flavour != SP3MM_UB && flavour != SP3MM_SYMBNUM))
        return batch_fail(b, SP3MM_EINVAL, "unknown flavour");
    b->flavour = flavour;
    return SP3MM_OK;
}

int sp3mm_batch_plan(sp3mm_batch* b) {
    if (!b) return SP3MM_EINVAL;
    return batch_plan(b);
}

int sp3mm_batch_execute(sp3mm_batch* b) {
    if (!b) return SP3MM_EINVAL;
    if (!b->planned) return batch_fail(b, SP3MM_EINVAL, "execute before plan");
    if (b->trimmed) return batch_fail(b, SP3MM_EINVAL, "the batch was trimmed");
    TRY(ensure_numeric(b));
    sp3mm_ctx* ctx = b->ctx;
    cudaError_t e = cudaSuccess;
    prof(ctx, "batch.numeric", [&] { e = cudaGraphLaunch(b->exec, ctx->stream); });
    CK(ctx, e);
    return SP3MM_OK;
}

int sp3mm_batch_run(sp3mm_batch* b) {
    if (!b) return SP3MM_EINVAL;
    if (!b->planned) {
        TRY(batch_plan(b));
        if (b->values_ready) return SP3MM_OK;   // the booked plan computed them
    }
    TRY(sp3mm_batch_execute(b));
    return check_device_err(b->ctx);
}

int sp3mm_batch_result(const sp3mm_batch* b, int i, sp3mm_dcsr* C) {
    if (!b || !C || !b->planned || i < 0 || i >= static_cast<int>(b->results.size()))
        return SP3MM_EINVAL;
    *C = b->results[i];
    return SP3MM_OK;
}

int sp3mm_batch_info(const sp3mm_batch* b, int64_t* rows, int64_t* nnz, int* tiers,
                     int* global_tiers, int64_t* retried) {
    if (!b) return SP3MM_EINVAL;
    if (rows) *rows = b->rows;
    if (nnz) *nnz = b->nnz;
    if (retried) *retried = b->retried;
    int t = 0, g = 0;
    for (const auto& x : b->tiers) (x.gt ? g : t)++;
    if (tiers) *tiers = t + g;
    if (global_tiers) *global_tiers = g;
    return SP3MM_OK;
}

int sp3mm_batch_free(sp3mm_batch* b) {
    if (!b) return SP3MM_EINVAL;
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
    return SP3MM_OK;
}

int sp3mm_batch_autotune(sp3mm_batch* b, int reps, char* report, size_t len) {
    if (!b || reps < 1) return SP3MM_EINVAL;
    sp3mm_ctx* ctx = b->ctx;
    const cudaStream_t st = ctx->stream;
    if (!b->planned) TRY(batch_plan(b));
    if (b->trimmed) return batch_fail(b, SP3MM_EINVAL, "the batch was trimmed");
    TRY(ensure_numeric(b));
    std::string rep;
    // Time `reps` replays of the current numeric graph.
    auto time_graph = [&](float* out) -> int {
        TRY(build_numeric(b));
        CK(ctx, cudaGraphLaunch(b->exec, st));   // warm-up
        CK(ctx, cudaEventRecord(ctx->ev0, st));
        for (int r = 0; r < reps; ++r) CK(ctx, cudaGraphLaunch(b->exec, st));
        CK(ctx, cudaEventRecord(ctx->ev1, st));
        CK(ctx, cudaEventSynchronize(ctx->ev1));
        float ms = 0.f;
        CK(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        *out = ms / reps;
        return SP3MM_OK;
    };
    // 1. Tiering: one tier per level, a single tier, or two tiers split at
    //    one of the first present levels.
    struct Cand {
        bool autos;
        std::vector<int> splits;
        float ms;
    };
    std::vector<int> present;
    for (int L = 0; L < kLevels; ++L)
        if (b->nbins.counts[L]) present.push_back(L);
    std::vector<Cand> cands;
    cands.push_back({true, {}, 0.f});
    cands.push_back({false, {}, 0.f});
    for (size_t k = 1; k < present.size() && k <= 4; ++k) cands.push_back({false, {present[k]}, 0.f});
    std::fill(b->level_slack.begin(), b->level_slack.end(), -1);
    b->slack = 0;
    size_t best = 0;
    for (size_t c = 0; c < cands.size(); ++c) {
        Cand& k = cands[c];
        b->auto_split = k.autos;
        b->splits = k.splits;
        TRY(time_graph(&k.ms));
        char line[160];
        snprintf(line, sizeof line, "%s split=%d tiers=%zu ms=%.4f\n",
                 k.autos ? "per-level" : (k.splits.empty() ? "one-tier" : "two-tier"),
                 k.splits.empty() ? -1 : k.splits[0], b->tiers.size(), k.ms);
        rep += line;
        if (k.ms < cands[best].ms) best = c;
    }
    b->auto_split = cands[best].autos;
    b->splits = cands[best].splits;
    float best_ms = cands[best].ms;
    // 2. Table slack per tier (larger tables shorten probe chains of heavy
    //    rows at the cost of shared memory per warp).
    TRY(build_numeric(b));
    std::vector<int> tops;
    for (const auto& t : b->tiers) tops.push_back(t.hi);
    for (int top : tops) {
        for (int sl = 1; sl <= 2; ++sl) {
            const int keep = b->level_slack[top];
            b->level_slack[top] = sl;
            float ms = 0.f;
            TRY(time_graph(&ms));
            char line[160];
            snprintf(line, sizeof line, "  tier level %d slack=%d ms=%.4f\n", top, sl, ms);
            rep += line;
            if (ms < best_ms) best_ms = ms;
            else b->level_slack[top] = keep;
        }
    }
    TRY(check_device_err(ctx));
    TRY(build_numeric(b));
    char line[96];
    snprintf(line, sizeof line, "best ms=%.4f\n", best_ms);
    rep += line;
    if (report && len) snprintf(report, len, "%s", rep.c_str());
    return SP3MM_OK;
}

}  // extern "C"
