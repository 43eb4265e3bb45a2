// capi.cu -- host runtime and C ABI of libsp3mm_b200.so.
//
// Layer 2 (sp3mm_*): contexts, device-resident CSR, device products.
// Layer 1 (reference names): upload host spmat -> device product -> download
// into malloc'd host spmat, with the reference's ownership and NULL-on-error
// behaviour (code/src/include/Sp3MM_CSR_OMP_Multi.h:50-53,
// code/src/include/sparseMatrix.h:154-168, code/src/include/macros.h:85-86).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <sys/mman.h>

#include "buffer_cache.h"
#include "context.cuh"
#include "host_pool.h"
#include "kernels.cuh"
#include "sp3mm_b200.h"
#include "sp3mm_internal.cuh"

using namespace sp3mm;

double Start = 0.0, End = 0.0, Elapsed = 0.0, ElapsedInternal = 0.0;

namespace sp3mm {

int set_error(sp3mm_ctx* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->last_error = buf;
    fprintf(stderr, "sp3mm_b200: %s\n", buf);
    return code;
}

int check_dcsr(sp3mm_ctx* ctx, const sp3mm_dcsr* m, const char* what) {
    if (!m) return set_error(ctx, SP3MM_EINVAL, "%s is NULL", what);
    if (m->M < 0 || m->N < 0 || m->nnz < 0 || !m->row_ptr || (m->nnz > 0 && (!m->col || !m->val)))
        return set_error(ctx, SP3MM_EINVAL, "%s is not a valid device CSR", what);
    if (m->val_type != SP3MM_F64 && m->val_type != SP3MM_F32)
        return set_error(ctx, SP3MM_EINVAL, "%s has an unknown value type", what);
    return SP3MM_OK;
}

size_t pool_idle_bytes(sp3mm_ctx* ctx) {
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) !=
            cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return reserved > used ? static_cast<size_t>(reserved - used) : 0;
}

void pool_reserve(sp3mm_ctx* ctx, size_t bytes) {
    if (bytes == 0 || pool_idle_bytes(ctx) >= bytes) return;
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes, ctx->stream) != cudaSuccess) {
        cudaGetLastError();   // not fatal: the pool grows on demand instead
        return;
    }
    cudaFreeAsync(p, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) cudaGetLastError();
}

size_t free_device_bytes(sp3mm_ctx* ctx) {
    // The reading is refreshed every 100 ms; in between, the pool's own
    // growth is subtracted from it (other processes' use is seen at the
    // next refresh).
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) !=
            cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        cudaGetLastError();
        reserved = used = 0;
    }
    const double now = std::chrono::duration<double>(
                           std::chrono::steady_clock::now().time_since_epoch())
                           .count();
    if (ctx->free_checked_s < 0 || now - ctx->free_checked_s > 0.1) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        ctx->free_at_check = fr;
        ctx->reserved_at_check = reserved;
        ctx->free_checked_s = now;
    }
    const uint64_t grown = reserved > ctx->reserved_at_check ? reserved - ctx->reserved_at_check : 0;
    size_t fr = ctx->free_at_check > grown ? ctx->free_at_check - grown : 0;
    if (reserved > used) fr += static_cast<size_t>(reserved - used);
    return fr;
}

int read_err(sp3mm_ctx* ctx, unsigned* out) {
    CK(ctx, cudaMemcpyAsync(out, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                            ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return SP3MM_OK;
}

int check_device_err(sp3mm_ctx* ctx) {
    unsigned e = 0;
    TRY(read_err(ctx, &e));
    if (e) {
        CK(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), ctx->stream));
        if (e & kErrInput) return set_error(ctx, SP3MM_EINVAL, "malformed CSR input (flags 0x%x)", e);
        return set_error(ctx, SP3MM_EDEVICE, "device error flags 0x%x", e);
    }
    return SP3MM_OK;
}

int bin_rows(sp3mm_ctx* ctx, int M, const int* need, int shift, int G, Counters* dcnt,
             int* row_cnt, Bins& b, const int* est) {
    TRY(b.level.alloc(ctx, static_cast<size_t>(M) + 1));
    TRY(b.lists.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
    prof(ctx, "bin.levels", [&] {
        launch_bin_levels(M, need, shift, G, b.level.as<signed char>(), dcnt->counts,
                          &dcnt->nmax, row_cnt, ctx->stream, est);
    });
    Counters h{};
    CK(ctx, cudaMemcpyAsync(&h, dcnt, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    int off = 0;
    for (int L = 0; L < kLevels; ++L) {
        b.counts[L] = h.counts[L];
        b.offsets[L] = off;
        h.cursors[L] = off;
        off += h.counts[L];
    }
    b.counts[kLevels] = h.counts[kLevels];
    b.nmax = h.nmax;
    b.total = h.total;
    CK(ctx, cudaMemcpyAsync(dcnt->cursors, h.cursors, sizeof h.cursors, cudaMemcpyHostToDevice,
                            ctx->stream));
    prof(ctx, "bin.scatter", [&] {
        launch_bin_scatter(M, b.level.as<signed char>(), dcnt->cursors, b.lists.as<int>(),
                           ctx->stream);
    });
    return SP3MM_OK;
}

}  // namespace sp3mm

namespace {

void prof_clear(sp3mm_ctx* ctx) {
    for (auto& r : ctx->prof) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    ctx->prof.clear();
}

double wall_seconds() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Lanes per row: the tuning, else a whole warp (the warp kernels); the
// mean row length of the right operand is kept for callers that tune by it.
int pick_group(const sp3mm_ctx* ctx, double mean) {
    (void)mean;
    if (ctx->tune_G && ctx->tune_G != kDenseLanes) return ctx->tune_G;
    return 32;
}

// Whether a launch of the direct product runs the CTA-per-row kernel: every
// row when the tuning asks for it; by default the rows binned to tables of
// kDenseMinSlots or more (thousands of distinct columns: coarse levels),
// where a warp per row with such a table leaves few warps per SM.  Never
// the retry launch, which needs proven-size tables.
constexpr int kDenseMinSlots = 2048;
bool use_dense(const sp3mm_ctx* ctx, const RowParams& p) {
    if (!p.retry_rows) return false;
    if (dense_row_smem() + 1024 > ctx->smem_optin) return false;
    if (ctx->tune_G == kDenseLanes) return true;
    return ctx->tune_G == 0 && p.S1 >= kDenseMinSlots;
}

// One row-kernel family over a set of rows: shared-memory tables when they
// fit the CTA budget, global-memory tables otherwise.
struct RowRunner {
    sp3mm_ctx* ctx;
    bool direct;
    int mode;
    DirectRowArgs da;
    PairRowArgs pa;
    // Longest row of the right operands (first / last; -1: unknown).
    int a_max = -1, b_max = -1;

    // Whether a direct launch runs the register-product kernel (rowlanes.cuh):
    // by default (no lane tuning) when the operands' longest rows are known
    // and the tables fit shared memory; never the retry launch, which the
    // warp kernels run with proven tables.
    static constexpr size_t kLanesMaxWarpBytes = 16 * 1024;
    bool use_lanes(const RowParams& p, int G) const {
        if (ctx->tune_G != 0 || G != 32 || !p.retry_rows) return false;
        if (a_max < 0 || b_max < 0) return false;
        return p.S2 <= p.S1;
    }

    // Batch layout of a lanes stage whose right operand has rows of at most
    // `mx` entries, `avg` on average: 2^lg lanes per step when the rows
    // fill at least 3/4 of them (stencil rows: 1.53 ms at 128^3 against
    // 1.57 packed), else packed (the kNN product's A rows of 16-31 entries:
    // 8.4 ms against 11.3 on the staged kernel).
    static int lanes_layout(int mx, const CsrView& B) {
        if (mx <= 0) return 0;
        if (mx > 32) return -1;
        const int lg = ilog2_pow2(next_pow2(static_cast<unsigned>(mx)));
        const double avg = B.M > 0 ? static_cast<double>(B.nnz) / B.M : 0.0;
        return avg >= 0.75 * (1 << lg) ? lg : -1;
    }

    long long operand_nnz() const {
        return direct ? da.R.nnz + da.A.nnz + da.P.nnz : pa.A.nnz + pa.B.nnz;
    }

    int launch(RowParams p, int G, DevBuf& gtab) {
        if (direct && use_dense(ctx, p)) {
            static const char* const kDense[3] = {"direct.dense.symb", "direct.dense.num",
                                                  "direct.dense.book"};
            static const char* const kDense2[3] = {"direct.dense2.symb", "direct.dense2.num",
                                                   "direct.dense2.book"};
            // Products whose A has many columns run two CTAs per SM first
            // (half the slice and list); the rows that outgrow it run again
            // on the default configuration (its row count stays on the
            // device), and what that cannot hold joins the retry list.
            const int per_sm = da.A.N >= kDenseSmallMinCols ? dense_small_ctas_per_sm() : 0;
            cudaError_t e = cudaSuccess;
            if (per_sm >= 2) {
                DevBuf again;
                TRY(again.alloc(ctx, sizeof(int) * (static_cast<size_t>(p.nrows) + 1)));
                int* n_again = again.as<int>() + p.nrows;
                CK(ctx, cudaMemsetAsync(n_again, 0, sizeof(int), ctx->stream));
                RowParams ps = p;
                ps.retry_rows = again.as<int>();
                ps.retry_count = n_again;
                prof(ctx, kDense2[mode], [&] {
                    e = launch_direct_dense_small(da, ps, mode, per_sm * ctx->num_sms,
                                                  ctx->stream);
                });
                if (e == cudaSuccess) {
                    RowParams pb = p;
                    pb.rows = again.as<int>();
                    pb.nrows_dev = n_again;
                    prof(ctx, kDense[mode], [&] {
                        e = launch_direct_dense(da, pb, mode, ctx->num_sms, ctx->stream);
                    });
                }
            } else {
                prof(ctx, kDense[mode], [&] {
                    e = launch_direct_dense(da, p, mode, ctx->num_sms, ctx->stream);
                });
            }
            if (e != cudaSuccess)
                return set_error(ctx, SP3MM_ECUDA, "dense row kernel launch failed: %s",
                                 cudaGetErrorString(e));
            return SP3MM_OK;
        }
        if (direct && use_lanes(p, G)) {
            // Tables twice the bin's size (the second half the first):
            // fewer probe steps and retried rows; measured 8 % faster at 128^3.
            // Where that does not fit, the second table (the C row, which in
            // a Galerkin product holds fewer columns than the R*A row) is
            // still half the first unless the caller tuned it: more warps
            // fit an SM (128^3 level 1: 4.24 -> 3.32 ms); a row whose C row
            // overflows it is retried with proven tables.
            if (lanes_row_bytes(mode, 2 * p.S1, p.S1) <= kLanesMaxWarpBytes) {
                p.S1 *= 2;
                p.S2 = p.S1 / 2;
            } else if (ctx->tune_d2 < 0 && p.S2 == p.S1 && p.S1 >= 64) {
                p.S2 = p.S1 / 2;
            }
            const size_t per_warp = lanes_row_bytes(mode, p.S1, p.S2);
            int warps = static_cast<int>(ctx->smem_budget / per_warp);
            if (warps > 8) warps = 8;
            if (warps >= 1) {
                RowGeom geo{};
                geo.G = 32;
                geo.block = 32 * warps;
                geo.smem = per_warp * warps;
                const long long grid = (p.nrows + warps - 1) / warps;
                const long long cap = static_cast<long long>(ctx->num_sms) * 16;
                geo.grid = static_cast<int>(grid < cap ? grid : cap);
                p.gtab = nullptr;
                p.lg1 = lanes_layout(a_max, da.A);
                p.lg2 = lanes_layout(b_max, da.P);
                static const char* const kLanes[3] = {"direct.lanes.symb", "direct.lanes.num",
                                                      "direct.lanes.book"};
                cudaError_t e = cudaSuccess;
                prof(ctx, kLanes[mode],
                     [&] { e = launch_direct_lanes(da, p, mode, geo, ctx->stream); });
                if (e != cudaSuccess)
                    return set_error(ctx, SP3MM_ECUDA, "lanes row kernel launch failed: %s",
                                     cudaGetErrorString(e));
                return SP3MM_OK;
            }
        }
        const size_t per_group = row_table_bytes(direct, mode, G, p.S1, p.S2);
        const int gpw = 32 / G;
        int warps = static_cast<int>(ctx->smem_budget / (per_group * gpw));
        if (warps > 8) warps = 8;
        RowGeom geo{};
        geo.G = G;
        if (warps >= 1) {
            geo.block = 32 * warps;
            geo.smem = per_group * gpw * warps;
            const int gpc = gpw * warps;
            long long grid = (p.nrows + gpc - 1) / gpc;
            const long long cap = static_cast<long long>(ctx->num_sms) * 16;
            geo.grid = static_cast<int>(grid < cap ? grid : cap);
            p.gtab = nullptr;
        } else {
            // Tables in global memory, one warp per row; concurrency bounded
            // by a 2 GiB scratch budget.
            geo.G = G = 32;
            const size_t stride = row_table_bytes(direct, mode, 32, p.S1, p.S2);
            size_t groups = static_cast<size_t>(p.nrows);
            const size_t cap = static_cast<size_t>(ctx->num_sms) * 8;
            if (groups > cap) groups = cap;
            const size_t budget = size_t(2) << 30;
            while (groups > 1 && groups * stride > budget) groups >>= 1;
            groups = (groups + 7) / 8 * 8;
            TRY(gtab.alloc(ctx, groups * stride));
            p.gtab = gtab.as<unsigned char>();
            p.gstride = static_cast<long long>(stride);
            geo.block = 256;
            geo.smem = 0;
            geo.grid = static_cast<int>(groups / 8);
        }
        const int cover = row_prefetch_cover(geo.G);
        p.a_long = a_max < 0 || a_max > cover;
        p.b_long = b_max < 0 || b_max > cover;
        static const char* const kLabels[2][3] = {
            {"pair.rows.symb", "pair.rows.num", "pair.rows.book"},
            {"direct.rows.symb", "direct.rows.num", "direct.rows.book"}};
        cudaError_t e = cudaSuccess;
        prof(ctx, kLabels[direct ? 1 : 0][mode], [&] {
            e = direct ? launch_direct_rows(da, p, mode, geo, ctx->stream)
                       : launch_pair_rows(pa, p, mode, geo, ctx->stream);
        });
        if (e != cudaSuccess)
            return set_error(ctx, SP3MM_ECUDA, "row kernel launch failed: %s",
                             cudaGetErrorString(e));
        return SP3MM_OK;
    }

    // Every level of `bins` with optimistic tables (S1 from the level, S2 =
    // S1 >> d2), then one retry launch for rows that overflowed, with tables
    // sized from the bounds s1_max / s2_max.
    int run(const Bins& bins, RowParams base, int G, int d2, long long s1_max, long long s2_max,
            Counters* dcnt) {
        DevBuf retry;
        TRY(run_levels(bins, base, G, d2, dcnt, retry));
        int nretry = 0;
        CK(ctx, cudaMemcpyAsync(&nretry, &dcnt->retry_count, sizeof(int), cudaMemcpyDeviceToHost,
                                ctx->stream));
        CK(ctx, cudaStreamSynchronize(ctx->stream));
        return run_retry(base, nretry, retry, s1_max, s2_max);
    }

    // The level launches alone, with no host round trip; rows that
    // overflowed are listed in `retry` and counted in dcnt->retry_count.
    int run_levels(const Bins& bins, RowParams base, int G, int d2, Counters* dcnt,
                   DevBuf& retry) {
        TRY(retry.alloc(ctx, sizeof(int) * (static_cast<size_t>(base.nrows) + 1)));
        CK(ctx, cudaMemsetAsync(&dcnt->retry_count, 0, sizeof(int), ctx->stream));
        for (int L = 0; L < kLevels; ++L) {
            if (!bins.counts[L]) continue;
            RowParams p = base;
            p.rows = bins.lists.as<int>() + bins.offsets[L];
            p.nrows = bins.counts[L];
            p.S1 = 32 << L;
            p.S2 = direct ? std::max(32, p.S1 >> d2) : 0;
            p.retry_rows = retry.as<int>();
            p.retry_count = &dcnt->retry_count;
            DevBuf gtab;
            TRY(launch(p, G, gtab));
        }
        return SP3MM_OK;
    }

    // The retry launch for `nretry` listed rows, tables sized from the
    // bounds.
    int run_retry(RowParams base, int nretry, DevBuf& retry, long long s1_max, long long s2_max) {
        if (nretry <= 0) return SP3MM_OK;
        RowParams p = base;
        p.rows = retry.as<int>();
        p.nrows = nretry;
        p.S1 = slots_for_need(s1_max, 32);
        p.S2 = direct ? slots_for_need(s2_max, 32) : 0;
        // The direct kernel sorts the C row in the first table's storage.
        if (p.S1 < p.S2) p.S1 = p.S2;
        p.retry_rows = nullptr;
        p.retry_count = nullptr;
        DevBuf gtab;
        TRY(launch(p, 32, gtab));
        return SP3MM_OK;
    }
};

int finish_matrix(sp3mm_dcsr* C, DevBuf& rp, DevBuf& ci, DevBuf& v) {
    C->row_ptr = static_cast<int*>(rp.detach());
    C->col = static_cast<int*>(ci.detach());
    C->val = v.detach();
    return SP3MM_OK;
}

// A result's row_ptr allocation: row_ptr[M+1], the longest row in the slot
// after it, then (8-byte aligned) the 64-bit total of the row counts, which
// tells a total past the int32 range from one the 32-bit scan wrapped.
size_t rp_bytes(int M) { return ((static_cast<size_t>(M) + 2) * 4 + 7) / 8 * 8 + 8; }
unsigned long long* rp_sum(const DevBuf& rp, int M) {
    return reinterpret_cast<unsigned long long*>(rp.as<unsigned char>() + rp_bytes(M) - 8);
}

// Scan row counts into a fresh row_ptr; returns the total (64-bit: a total
// of 2^31 or more is reported as such, not wrapped).
int scan_counts(sp3mm_ctx* ctx, int M, const int* row_cnt, DevBuf& rp, long long* total,
                int* max_row = nullptr) {
    TRY(rp.alloc(ctx, rp_bytes(M)));
    DevBuf tmp;
    const size_t tb = scan_temp_bytes(M);
    TRY(tmp.alloc(ctx, tb));
    prof(ctx, "scan", [&] { launch_scan(M, row_cnt, rp.as<int>(), tmp.p, tb, ctx->stream); });
    CK(ctx, cudaGetLastError());
    int* mr = rp.as<int>() + M + 1;
    unsigned long long* sum = rp_sum(rp, M);
    CK(ctx, cudaMemsetAsync(mr, 0, sizeof(int), ctx->stream));
    CK(ctx, cudaMemsetAsync(sum, 0, sizeof(unsigned long long), ctx->stream));
    launch_count_max(M, row_cnt, nullptr, mr, ctx->stream, sum);
    int t[2] = {0, 0};
    unsigned long long t64 = 0;
    CK(ctx, cudaMemcpyAsync(t, rp.as<int>() + M, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                            ctx->stream));
    CK(ctx, cudaMemcpyAsync(&t64, sum, sizeof t64, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    *total = static_cast<long long>(t64);
    if (max_row) *max_row = t[1];
    return SP3MM_OK;
}

// The words a booked product reads back after its numeric pass.
struct TailReads {
    long long total;   // nnz(C)
    int max_row;       // longest C row
    int retry;         // rows left for the retry launch
    unsigned err;      // device error word
};

// Scan row counts into row_ptr (allocated on first use) and read back, in
// one round trip through the context's pinned words, the total, the longest
// row, the retry count (d_retry, may be null) and the error word.
int scan_read(sp3mm_ctx* ctx, int M, const int* row_cnt, DevBuf& rp, const int* d_retry,
              TailReads* out) {
    const cudaStream_t st = ctx->stream;
    if (!rp.p) TRY(rp.alloc(ctx, rp_bytes(M)));
    DevBuf tmp;
    const size_t tb = scan_temp_bytes(M);
    TRY(tmp.alloc(ctx, tb));
    prof(ctx, "scan", [&] { launch_scan(M, row_cnt, rp.as<int>(), tmp.p, tb, st); });
    CK(ctx, cudaGetLastError());
    int* mr = rp.as<int>() + M + 1;
    unsigned long long* sum = rp_sum(rp, M);
    CK(ctx, cudaMemsetAsync(mr, 0, sizeof(int), st));
    CK(ctx, cudaMemsetAsync(sum, 0, sizeof(unsigned long long), st));
    launch_count_max(M, row_cnt, nullptr, mr, st, sum);
    unsigned* box = ctx->host_box;
    box[2] = 0;
    CK(ctx, cudaMemcpyAsync(box, rp.as<int>() + M, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    if (d_retry)
        CK(ctx, cudaMemcpyAsync(box + 2, d_retry, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(ctx, cudaMemcpyAsync(box + 3, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(ctx, cudaMemcpyAsync(box + 4, sum, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st));
    CK(ctx, cudaStreamSynchronize(st));
    out->total = static_cast<long long>(*reinterpret_cast<unsigned long long*>(box + 4));
    out->max_row = static_cast<int>(box[1]);
    out->retry = static_cast<int>(box[2]);
    out->err = box[3];
    return SP3MM_OK;
}

// Read back the retry count (d_retry, may be null: 0) and the error word in
// one round trip.
int read_retry_err(sp3mm_ctx* ctx, const int* d_retry, TailReads* out) {
    const cudaStream_t st = ctx->stream;
    unsigned* box = ctx->host_box;
    box[2] = 0;
    if (d_retry)
        CK(ctx, cudaMemcpyAsync(box + 2, d_retry, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(ctx, cudaMemcpyAsync(box + 3, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(ctx, cudaStreamSynchronize(st));
    out->retry = static_cast<int>(box[2]);
    out->err = box[3];
    return SP3MM_OK;
}

// Longest row of m, computed on the device when not recorded.
int known_max_row(sp3mm_ctx* ctx, const sp3mm_dcsr& m, int* out) {
    if (m.max_row >= 0) {
        *out = m.max_row;
        return SP3MM_OK;
    }
    DevBuf b;
    TRY(b.alloc(ctx, sizeof(int)));
    CK(ctx, cudaMemsetAsync(b.p, 0, sizeof(int), ctx->stream));
    launch_count_max(m.M, nullptr, m.row_ptr, b.as<int>(), ctx->stream);
    CK(ctx, cudaMemcpyAsync(out, b.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return SP3MM_OK;
}

// The shared tail of every product: symbolic + exact numeric, or booked
// numeric + compaction.  `need` holds the first table's distinct-key bound
// per row; s1_max/s2_max bound the tables of the retry launch.
int product_rows(sp3mm_ctx* ctx, RowRunner& rr, int M, int N, int flavour, int out_vt,
                 DevBuf& need, Counters* dc, int G, int d1, int d2, long long s1_bound,
                 long long s2_bound, double p_max_row, sp3mm_dcsr* C,
                 const int* est = nullptr) {
    const cudaStream_t st = ctx->stream;
    DevBuf row_cnt, row_cnt1, rp, ci, v;
    TRY(row_cnt.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
    Bins bins;
    TRY(bin_rows(ctx, M, need.as<int>(), d1, G, dc, row_cnt.as<int>(), bins, est));
    const long long s1_max = std::min<long long>(bins.nmax, s1_bound);
    const long long s2_max = std::min<long long>(
        static_cast<long long>(static_cast<double>(bins.nmax) * p_max_row), s2_bound);

    RowParams p{};
    p.nrows = M;
    p.row_cnt = row_cnt.as<int>();
    p.err = ctx->d_err;
    p.c_vt = out_vt;
    long long nnz = 0;
    int cmax = -1;
    if (flavour == SP3MM_SYMBNUM) {
        if (rr.direct) {
            TRY(row_cnt1.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
            CK(ctx, cudaMemsetAsync(row_cnt1.p, 0, sizeof(int) * (static_cast<size_t>(M) + 1), st));
            p.row_cnt1 = row_cnt1.as<int>();
        }
        rr.mode = kSymb;
        DevBuf retry;
        TRY(rr.run_levels(bins, p, G, d2, dc, retry));
        TailReads tr{};
        TRY(scan_read(ctx, M, row_cnt.as<int>(), rp, &dc->retry_count, &tr));
        if (tr.err) return check_device_err(ctx);
        if (tr.retry > 0) {
            TRY(rr.run_retry(p, tr.retry, retry, s1_max, s2_max));
            TRY(scan_read(ctx, M, row_cnt.as<int>(), rp, nullptr, &tr));
            if (tr.err) return check_device_err(ctx);
        }
        nnz = tr.total;
        cmax = tr.max_row;
        if (nnz < 0 || nnz >= INT32_MAX)
            return set_error(ctx, SP3MM_ELIMIT, "result has too many nonzeros");
        TRY(ci.alloc(ctx, sizeof(int) * static_cast<size_t>(nnz)));
        TRY(v.alloc(ctx, vbytes(out_vt) * static_cast<size_t>(nnz)));
        // Exact sizes: re-bin by max(C row, R*A row) distinct counts.
        CK(ctx, cudaMemsetAsync(dc, 0, sizeof(Counters), st));
        prof(ctx, "need", [&] {
            launch_need_from_counts(M, row_cnt.as<int>(), rr.direct ? row_cnt1.as<int>() : nullptr,
                                    need.as<int>(), st);
        });
        Bins nb;
        TRY(bin_rows(ctx, M, need.as<int>(), 0, G, dc, nullptr, nb));
        p.row_cnt1 = nullptr;
        p.c_rp = rp.as<int>();
        p.c_ci = ci.as<int>();
        p.c_v = v.p;
        rr.mode = kNumExact;
        TRY(rr.run_levels(nb, p, G, 0, dc, retry));
        TRY(read_retry_err(ctx, &dc->retry_count, &tr));
        if (tr.retry > 0 && !tr.err) {
            TRY(rr.run_retry(p, tr.retry, retry, s1_max, s2_max));
            TRY(read_retry_err(ctx, nullptr, &tr));
        }
        if (tr.err) return check_device_err(ctx);
    } else {
        // Rows book their exact length from one cursor, so the space need
        // only exceed nnz(C): the bound, capped at half the free memory; a
        // product that still overflows it is redone symbolically.
        const size_t eb = sizeof(int) + vbytes(out_vt);
        unsigned long long cap = std::min<unsigned long long>(
            bins.total,
            std::max<unsigned long long>(1ULL << 20,
                                         8ULL * static_cast<unsigned long long>(rr.operand_nnz())));
        // Space the pool already holds idle is used without asking the
        // device for its free memory (a slow query).
        if (cap * eb > (size_t(1) << 30) && pool_idle_bytes(ctx) < cap * eb)
            cap = std::min<unsigned long long>(
                cap, std::max<unsigned long long>(1ULL << 20, free_device_bytes(ctx) / 2 / eb));
        DevBuf ub_ci, ub_v, row_off, retry;
        TRY(ub_ci.alloc(ctx, sizeof(int) * cap));
        TRY(ub_v.alloc(ctx, vbytes(out_vt) * cap));
        TRY(row_off.alloc(ctx, sizeof(long long) * (static_cast<size_t>(M) + 1)));
        CK(ctx, cudaMemsetAsync(&dc->cursor, 0, sizeof(unsigned long long), st));
        p.cursor = &dc->cursor;
        p.cap = cap;
        p.row_off = row_off.as<long long>();
        p.ub_ci = ub_ci.as<int>();
        p.ub_v = ub_v.p;
        rr.mode = kNumBook;
        // The scan, the retry count and the error word come back together;
        // rows that overflowed their tables are redone and rescanned.
        TRY(rr.run_levels(bins, p, G, d2, dc, retry));
        TailReads tr{};
        TRY(scan_read(ctx, M, row_cnt.as<int>(), rp, &dc->retry_count, &tr));
        for (int pass = 0; pass < 2; ++pass) {
            if (tr.err & ~kErrBook) return check_device_err(ctx);
            if (tr.err == kErrBook) {
                // The booking space overflowed (possible only below the
                // bound): redo the product symbolically.
                CK(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), st));
                ub_ci.release();
                ub_v.release();
                CK(ctx, cudaMemsetAsync(dc, 0, sizeof(Counters), st));
                return product_rows(ctx, rr, M, N, SP3MM_SYMBNUM, out_vt, need, dc, G, d1, d2,
                                     s1_bound, s2_bound, p_max_row, C, est);
            }
            if (pass == 1 || tr.retry <= 0) break;
            TRY(rr.run_retry(p, tr.retry, retry, s1_max, s2_max));
            TRY(scan_read(ctx, M, row_cnt.as<int>(), rp, nullptr, &tr));
        }
        nnz = tr.total;
        cmax = tr.max_row;
        if (nnz < 0 || nnz >= INT32_MAX)
            return set_error(ctx, SP3MM_ELIMIT, "result has too many nonzeros");
        TRY(ci.alloc(ctx, sizeof(int) * static_cast<size_t>(nnz)));
        TRY(v.alloc(ctx, vbytes(out_vt) * static_cast<size_t>(nnz)));
        prof(ctx, "compact", [&] {
            launch_compact(M, row_cnt.as<int>(), row_off.as<long long>(), ub_ci.as<int>(), ub_v.p,
                           rp.as<int>(), ci.as<int>(), v.p, out_vt, st);
        });
    }
    // Both tails read the error word after their last flag-setting kernel
    // (the compaction sets none).
    C->M = M;
    C->N = N;
    C->nnz = nnz;
    C->val_type = out_vt;
    C->max_row = cmax;
    return finish_matrix(C, rp, ci, v);
}

// ---------------------------------------------------------------------------
// C = A*B.
int spmm_impl(sp3mm_ctx* ctx, const sp3mm_dcsr& A, const sp3mm_dcsr& B, int flavour, int out_vt,
              sp3mm_dcsr* C) {
    if (A.N != B.M)
        return set_error(ctx, SP3MM_EINVAL, "inner dimensions differ (%d vs %d)", A.N, B.M);
    if (A.val_type != B.val_type)
        return set_error(ctx, SP3MM_EINVAL, "operands must share one value storage type");
    const int M = A.M;
    const cudaStream_t st = ctx->stream;
    int G = pick_group(ctx, B.M ? static_cast<double>(B.nnz) / B.M : 1.0);
    // Rows of a few products (a hierarchy's A*P0: 7 per row) leave most of
    // a warp idle: 4 lanes a row, 8 rows a warp (128^3 A*P0: 1.76 -> 0.85 ms).
    const double products = (A.M ? static_cast<double>(A.nnz) / A.M : 0.0) *
                            (B.M ? static_cast<double>(B.nnz) / B.M : 0.0);
    if (ctx->tune_G == 0 && products <= 8.0) G = 4;
    const int d1 = ctx->tune_d1 >= 0 ? ctx->tune_d1 : 2;
    DevBuf cnt_buf, need;
    TRY(cnt_buf.alloc(ctx, sizeof(Counters)));
    TRY(need.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
    Counters* dc = cnt_buf.as<Counters>();
    CK(ctx, cudaMemsetAsync(dc, 0, sizeof(Counters), st));
    prof(ctx, "pair.bounds", [&] {
        launch_pair_bounds(view(A), view(B), need.as<int>(), &dc->total, st);
    });
    RowRunner rr{ctx, false, kSymb, {}, PairRowArgs{view(A), view(B)}, -1, B.max_row};
    return product_rows(ctx, rr, M, B.N, flavour, out_vt, need, dc, G, d1, 0, B.N, 0, 0.0, C);
}

// C = R*A*P, direct (row forwarding).
int direct_impl(sp3mm_ctx* ctx, const sp3mm_dcsr& R, const sp3mm_dcsr& A, const sp3mm_dcsr& P,
                int flavour, int out_vt, sp3mm_dcsr* C) {
    if (R.N != A.M || A.N != P.M)
        return set_error(ctx, SP3MM_EINVAL, "inner dimensions differ");
    if (R.val_type != A.val_type || A.val_type != P.val_type)
        return set_error(ctx, SP3MM_EINVAL, "operands must share one value storage type");
    const int M = R.M;
    const cudaStream_t st = ctx->stream;
    const double mean = std::max(A.M ? static_cast<double>(A.nnz) / A.M : 1.0,
                                 P.M ? static_cast<double>(P.nnz) / P.M : 1.0);
    const int G = pick_group(ctx, mean);
    const int d1 = ctx->tune_d1 >= 0 ? ctx->tune_d1 : 2;
    const int d2 = ctx->tune_d2 >= 0 ? ctx->tune_d2 : 0;
    int pmax = 0, amax = 0;
    TRY(known_max_row(ctx, P, &pmax));
    TRY(known_max_row(ctx, A, &amax));
    DevBuf cnt_buf, need, need_opt;
    TRY(cnt_buf.alloc(ctx, sizeof(Counters)));
    TRY(need.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
    TRY(need_opt.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
    Counters* dc = cnt_buf.as<Counters>();
    CK(ctx, cudaMemsetAsync(dc, 0, sizeof(Counters), st));
    prof(ctx, "direct.bounds", [&] {
        launch_direct_bounds(view(R), view(A), pmax, need.as<int>(), &dc->total, st,
                             need_opt.as<int>(), d1);
    });
    RowRunner rr{ctx, true, kSymb, DirectRowArgs{view(R), view(A), view(P)}, {}, amax, pmax};
    return product_rows(ctx, rr, M, P.N, flavour, out_vt, need, dc, G, d1, d2, A.N, P.N,
                        static_cast<double>(pmax), C, need_opt.as<int>());
}

void free_dcsr_arrays(sp3mm_ctx* ctx, sp3mm_dcsr* m) {
    if (!m) return;
    if (m->row_ptr) cudaFreeAsync(m->row_ptr, ctx->stream);
    if (m->col) cudaFreeAsync(m->col, ctx->stream);
    if (m->val) cudaFreeAsync(m->val, ctx->stream);
    m->row_ptr = nullptr;
    m->col = nullptr;
    m->val = nullptr;
}

int rap_impl(sp3mm_ctx* ctx, const sp3mm_dcsr& R, const sp3mm_dcsr& A, const sp3mm_dcsr& P,
             int variant, int flavour, int out_vt, sp3mm_dcsr* C) {
    if (variant == SP3MM_DIRECT) return direct_impl(ctx, R, A, P, flavour, out_vt, C);
    sp3mm_dcsr T{};
    int rc;
    // The intermediate is stored in the operands' value type (FP64 operands:
    // an FP64 intermediate, so the pair is bit-identical to the reference).
    if (variant == SP3MM_PAIR) {
        TRY(spmm_impl(ctx, R, A, flavour, R.val_type, &T));
        rc = spmm_impl(ctx, T, P, flavour, out_vt, C);
    } else if (variant == SP3MM_PAIR_RIGHT) {
        TRY(spmm_impl(ctx, A, P, flavour, A.val_type, &T));
        rc = spmm_impl(ctx, R, T, flavour, out_vt, C);
    } else {
        return set_error(ctx, SP3MM_EINVAL, "unknown variant %d", variant);
    }
    free_dcsr_arrays(ctx, &T);
    return rc;
}

// Upload from 64-bit host arrays with index offset `off`.
// Pinned staging of at least `bytes` (at most kHostStageMax) on the context.
constexpr size_t kHostStageMax = size_t(256) << 20;

// Page-locked staging buffers outlive the contexts that used them
// (buffer_cache.h): cudaHostAlloc costs about 0.4 ms per MB (100 ms for
// 256 MB on a B200 host), ten times the copy it stages, and a server
// creates its loader contexts per instance, a caller thread its context per
// thread.  A buffer is given back only after its context's stream has been
// synchronised, so no copy from it is in flight.
struct PinnedAlloc {
    void* operator()(size_t bytes) const {
        void* p = nullptr;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) return nullptr;
        return p;
    }
};
struct PinnedRelease {
    void operator()(void* p) const { cudaFreeHost(p); }
};
using PinnedCache = BufferCache<PinnedAlloc, PinnedRelease>;

// Never destroyed: cached buffers are released with the process.
PinnedCache& pinned_cache() {
    static PinnedCache* c = new PinnedCache(PinnedAlloc{}, PinnedRelease{}, size_t(1) << 30);
    return *c;
}

// Sizes are rounded up to powers of two (1 MB .. kHostStageMax), so a
// context grows its staging a few times at most.
int host_stage(sp3mm_ctx* ctx, size_t bytes, void** out) {
    bytes = std::min(std::max<size_t>(bytes, size_t(1) << 20), kHostStageMax);
    size_t want = size_t(1) << 20;
    while (want < bytes) want <<= 1;
    if (ctx->host_stage_bytes < want) {
        if (ctx->host_stage) {
            CK(ctx, cudaStreamSynchronize(ctx->stream));
            pinned_cache().give(ctx->host_stage, ctx->host_stage_bytes);
        }
        ctx->host_stage = nullptr;
        ctx->host_stage_bytes = 0;
        size_t got = 0;
        void* p = pinned_cache().take(want, &got);
        if (!p) {
            cudaGetLastError();
            return set_error(ctx, SP3MM_ENOMEM, "page-locked staging of %zu bytes", want);
        }
        ctx->host_stage = p;
        ctx->host_stage_bytes = got;
    }
    *out = ctx->host_stage;
    return SP3MM_OK;
}

// Persistent host workers for the transfer loops (host_pool.h).  One
// caller at a time uses the pool; a concurrent caller (e.g. a server's
// second loader thread) spawns its own threads instead.
HostPool& host_pool() {
    static HostPool* pool = [] {
        const unsigned hw = std::thread::hardware_concurrency();
        const int n = static_cast<int>(std::max(1u, std::min(hw ? hw : 1u, 16u)) - 1);
        return new HostPool(n);
    }();
    return *pool;
}

// f(lo, hi) over [0, n) on up to 16 host threads (one for small n).
template <typename F>
void host_parallel(long long n, F&& f) {
    const long long per = 1 << 18;
    const unsigned hw = std::thread::hardware_concurrency();
    int t = static_cast<int>(std::min<long long>((n + per - 1) / per, 16));
    if (hw) t = std::min<int>(t, static_cast<int>(hw));
    if (t <= 1) {
        f(0LL, n);
        return;
    }
    const long long chunk = (n + t - 1) / t;
    HostPool& pool = host_pool();
    std::unique_lock<std::mutex> lk(pool.use, std::try_to_lock);
    if (lk.owns_lock() && pool.size() > 0) {
        const std::function<void(long long, long long)> fn = [&f](long long lo, long long hi) {
            f(lo, hi);
        };
        pool.run(fn, n, chunk, static_cast<int>((n + chunk - 1) / chunk));
        return;
    }
    std::vector<std::thread> th;
    for (int k = 0; k < t; ++k) {
        const long long lo = k * chunk, hi = std::min(n, lo + chunk);
        if (lo < hi) th.emplace_back([&f, lo, hi] { f(lo, hi); });
    }
    for (auto& x : th) x.join();
}

// Pinned host sources: copy the 64-bit arrays as they are into a device
// stage and narrow / validate them there.
int upload_u64_direct(sp3mm_ctx* ctx, long long M, long long N, long long nnz, const uint64_t* irp,
               const uint64_t* ja, const double* as, int off, int vt, sp3mm_dcsr* out) {
    if (M < 0 || N < 0 || nnz < 0) return set_error(ctx, SP3MM_EINVAL, "negative sizes");
    if (M >= INT32_MAX || N >= INT32_MAX || nnz >= INT32_MAX)
        return set_error(ctx, SP3MM_ELIMIT,
                         "matrix %lldx%lld with %lld nonzeros exceeds the 32-bit device limits",
                         M, N, nnz);
    if (!irp || (nnz > 0 && (!ja || !as)))
        return set_error(ctx, SP3MM_EINVAL, "NULL CSR arrays");
    const cudaStream_t st = ctx->stream;
    DevBuf rp, ci, v, stage, maxrow;
    TRY(rp.alloc(ctx, sizeof(int) * (M + 1)));
    TRY(ci.alloc(ctx, sizeof(int) * nnz));
    TRY(v.alloc(ctx, vbytes(vt) * nnz));
    TRY(maxrow.alloc(ctx, sizeof(int)));
    TRY(stage.alloc(ctx, sizeof(uint64_t) * std::max(M + 1, nnz)));
    CK(ctx, cudaMemsetAsync(maxrow.p, 0, sizeof(int), st));
    CK(ctx, cudaMemcpyAsync(stage.p, irp, sizeof(uint64_t) * (M + 1), cudaMemcpyHostToDevice, st));
    // Malformed row pointers are flagged and narrowed to 0, so the column
    // pass below stays in bounds; the error is reported by the final check.
    launch_narrow_rowptr(M, nnz, stage.as<unsigned long long>(), off, rp.as<int>(), ctx->d_err, st);
    CK(ctx, cudaGetLastError());
    if (nnz > 0) {
        CK(ctx, cudaMemcpyAsync(stage.p, ja, sizeof(uint64_t) * nnz, cudaMemcpyHostToDevice, st));
        launch_narrow_cols(M, N, rp.as<int>(), stage.as<unsigned long long>(), off, ci.as<int>(),
                           maxrow.as<int>(), ctx->d_err, st);
        CK(ctx, cudaGetLastError());
        if (vt == SP3MM_F64) {
            CK(ctx, cudaMemcpyAsync(v.p, as, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
        } else {
            CK(ctx, cudaMemcpyAsync(stage.p, as, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
            launch_convert_values(nnz, stage.p, SP3MM_F64, v.p, vt, st);
        }
    }
    int mr = 0;
    CK(ctx, cudaMemcpyAsync(&mr, maxrow.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY(check_device_err(ctx));
    out->M = static_cast<int>(M);
    out->N = static_cast<int>(N);
    out->nnz = nnz;
    out->val_type = vt;
    out->max_row = mr;
    return finish_matrix(out, rp, ci, v);
}

bool host_pinned(const void* p) {
    if (!p) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Pageable host sources: host threads narrow the indices to int32 -- validating the row pointers completely
// (start 0, end nnz, monotone) and the column range -- into pinned staging,
// two halves used in turn so that filling one overlaps the copy of the
// other; the device then checks the columns' order and records the longest
// row.
int upload_u64_staged(sp3mm_ctx* ctx, long long M, long long N, long long nnz,
                      const uint64_t* irp,
               const uint64_t* ja, const double* as, int off, int vt, sp3mm_dcsr* out) {
    if (M < 0 || N < 0 || nnz < 0) return set_error(ctx, SP3MM_EINVAL, "negative sizes");
    if (M >= INT32_MAX || N >= INT32_MAX || nnz >= INT32_MAX)
        return set_error(ctx, SP3MM_ELIMIT,
                         "matrix %lldx%lld with %lld nonzeros exceeds the 32-bit device limits",
                         M, N, nnz);
    if (!irp || (nnz > 0 && (!ja || !as)))
        return set_error(ctx, SP3MM_EINVAL, "NULL CSR arrays");
    const cudaStream_t st = ctx->stream;
    DevBuf rp, ci, v, maxrow;
    TRY(rp.alloc(ctx, sizeof(int) * (M + 1)));
    TRY(ci.alloc(ctx, sizeof(int) * nnz));
    TRY(v.alloc(ctx, vbytes(vt) * nnz));
    TRY(maxrow.alloc(ctx, sizeof(int)));
    CK(ctx, cudaMemsetAsync(maxrow.p, 0, sizeof(int), st));
    const size_t biggest =
        std::max<size_t>(sizeof(int) * (M + 1), std::max<size_t>(sizeof(double), 4) * nnz);
    void* stage = nullptr;
    TRY(host_stage(ctx, 2 * std::min(biggest, kHostStageMax / 2), &stage));
    const size_t half = ctx->host_stage_bytes / 2 / 256 * 256;
    std::atomic<bool> bad(false);
    int h = 0;
    // Fill and copy one array in chunks through the staging halves: half h
    // is filled while the other half's copy is in flight; the stream is
    // synchronised (so that copy, and the other half, are done) before the
    // copy of half h is issued, so a half is never refilled while copied.
    auto push = [&](void* dst, size_t esz, long long n, auto&& fill) -> int {
        const long long per = static_cast<long long>(half / esz);
        for (long long b = 0; b < n; b += per) {
            const long long k = std::min(per, n - b);
            unsigned char* buf = static_cast<unsigned char*>(stage) + h * half;
            host_parallel(k, [&](long long lo, long long hi) { fill(b, lo, hi, buf); });
            CK(ctx, cudaStreamSynchronize(st));
            CK(ctx, cudaMemcpyAsync(static_cast<unsigned char*>(dst) + b * esz, buf, esz * k,
                                    cudaMemcpyHostToDevice, st));
            h ^= 1;
        }
        return SP3MM_OK;
    };
    TRY(push(rp.p, sizeof(int), M + 1, [&](long long b, long long lo, long long hi, void* buf) {
        int* o = static_cast<int*>(buf);
        bool ok = true;
        for (long long i = lo; i < hi; ++i) {
            const long long g = b + i;
            const long long x = static_cast<long long>(irp[g]) - off;
            ok &= x >= 0 && x <= nnz;
            if (g == 0) ok &= x == 0;
            if (g == M) ok &= x == nnz;
            if (g > 0) ok &= static_cast<long long>(irp[g - 1]) - off <= x;
            o[i] = static_cast<int>(x);
        }
        if (!ok) bad = true;
    }));
    if (nnz > 0 && !bad) {
        TRY(push(ci.p, sizeof(int), nnz, [&](long long b, long long lo, long long hi, void* buf) {
            int* o = static_cast<int*>(buf);
            bool ok = true;
            for (long long i = lo; i < hi; ++i) {
                const long long c = static_cast<long long>(ja[b + i]) - off;
                ok &= c >= 0 && c < N;
                o[i] = static_cast<int>(c);
            }
            if (!ok) bad = true;
        }));
        if (vt == SP3MM_F64) {
            TRY(push(v.p, sizeof(double), nnz,
                     [&](long long b, long long lo, long long hi, void* buf) {
                         std::memcpy(static_cast<double*>(buf) + lo, as + b + lo,
                                     sizeof(double) * (hi - lo));
                     }));
        } else {
            TRY(push(v.p, sizeof(float), nnz,
                     [&](long long b, long long lo, long long hi, void* buf) {
                         float* o = static_cast<float*>(buf);
                         for (long long i = lo; i < hi; ++i) o[i] = static_cast<float>(as[b + i]);
                     }));
        }
    }
    if (bad) {
        CK(ctx, cudaStreamSynchronize(st));
        return set_error(ctx, SP3MM_EINVAL,
                         "malformed CSR input (row pointers or column range)");
    }
    launch_validate_i32(static_cast<int>(M), static_cast<int>(N), rp.as<int>(), ci.as<int>(),
                        maxrow.as<int>(), ctx->d_err, st);
    CK(ctx, cudaGetLastError());
    int mr = 0;
    CK(ctx, cudaMemcpyAsync(&mr, maxrow.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY(check_device_err(ctx));
    out->M = static_cast<int>(M);
    out->N = static_cast<int>(N);
    out->nnz = nnz;
    out->val_type = vt;
    out->max_row = mr;
    return finish_matrix(out, rp, ci, v);
}

// Host 64-bit CSR (indices shifted by off) -> device CSR, by the faster route
// for the sources' memory (validated either way).
int upload_u64(sp3mm_ctx* ctx, long long M, long long N, long long nnz, const uint64_t* irp,
               const uint64_t* ja, const double* as, int off, int vt, sp3mm_dcsr* out) {
    if (host_pinned(irp) && host_pinned(ja) && host_pinned(as))
        return upload_u64_direct(ctx, M, N, nnz, irp, ja, as, off, vt, out);
    return upload_u64_staged(ctx, M, N, nnz, irp, ja, as, off, vt, out);
}

// Copy a device CSR into malloc'd host arrays, indices shifted by `off`.
// Device CSR -> host 64-bit arrays (indices shifted by off, values FP64).
// The compact device arrays go through pinned staging (full-speed copies);
// widening and the copy into the caller's (possibly never-touched, pageable)
// arrays run on host threads.
int download_u64(sp3mm_ctx* ctx, const sp3mm_dcsr& m, int off, uint64_t* irp, uint64_t* ja,
                 double* as) {
    const cudaStream_t st = ctx->stream;
    void* stage = nullptr;
    const size_t want = 2 * std::max<size_t>(sizeof(int) * (static_cast<size_t>(m.M) + 1),
                                             sizeof(double) * static_cast<size_t>(m.nnz));
    TRY(host_stage(ctx, std::min(want, kHostStageMax), &stage));
    const size_t half = ctx->host_stage_bytes / 2 / 256 * 256;
    // The three arrays as one sequence of chunks, each copied into one half
    // of the staging while the host threads widen the previous chunk from
    // the other half (an event per half marks its copy done).
    struct Piece {
        const void* src;
        size_t esz;
        long long b, k;
        int what;   // 0 row pointers, 1 columns, 2 values
    };
    std::vector<Piece> pieces;
    auto add = [&](const void* src, size_t esz, long long n, int what) {
        const long long per = static_cast<long long>(half / esz);
        for (long long b = 0; b < n; b += per) pieces.push_back({src, esz, b, std::min(per, n - b), what});
    };
    add(m.row_ptr, sizeof(int), static_cast<long long>(m.M) + 1, 0);
    if (m.nnz > 0) {
        add(m.col, sizeof(int), m.nnz, 1);
        add(m.val, vbytes(m.val_type), m.nnz, 2);
    }
    auto issue = [&](size_t i) -> int {
        const Piece& q = pieces[i];
        void* buf = static_cast<unsigned char*>(stage) + (i & 1) * half;
        CK(ctx, cudaMemcpyAsync(buf, static_cast<const unsigned char*>(q.src) + q.b * q.esz,
                                q.esz * q.k, cudaMemcpyDeviceToHost, st));
        CK(ctx, cudaEventRecord((i & 1) ? ctx->ev1 : ctx->ev0, st));
        return SP3MM_OK;
    };
    if (!pieces.empty()) TRY(issue(0));
    const uint64_t o = static_cast<uint64_t>(off);
    for (size_t i = 0; i < pieces.size(); ++i) {
        if (i + 1 < pieces.size()) TRY(issue(i + 1));
        CK(ctx, cudaEventSynchronize((i & 1) ? ctx->ev1 : ctx->ev0));
        const Piece& q = pieces[i];
        const void* buf = static_cast<unsigned char*>(stage) + (i & 1) * half;
        const long long b = q.b;
        if (q.what == 0 || q.what == 1) {
            const int* src = static_cast<const int*>(buf);
            uint64_t* dst = (q.what == 0 ? irp : ja) + b;
            host_parallel(q.k, [&](long long lo, long long hi) {
                for (long long x = lo; x < hi; ++x) dst[x] = static_cast<uint64_t>(src[x]) + o;
            });
        } else if (m.val_type == SP3MM_F64) {
            const double* src = static_cast<const double*>(buf);
            host_parallel(q.k, [&](long long lo, long long hi) {
                std::memcpy(as + b + lo, src + lo, sizeof(double) * (hi - lo));
            });
        } else {
            const float* src = static_cast<const float*>(buf);
            host_parallel(q.k, [&](long long lo, long long hi) {
                for (long long x = lo; x < hi; ++x) as[b + x] = static_cast<double>(src[x]);
            });
        }
    }
    return SP3MM_OK;
}

int ctx_init(sp3mm_ctx* c, int device) {
    c->device = device;
    CK(c, cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(c, cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return set_error(c, SP3MM_ECUDA, "device %d (sm_%d%d) is not a Blackwell sm_100 GPU",
                         device, prop.major, prop.minor);
    c->num_sms = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    CK(c, cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    CK(c, cudaMalloc(&c->d_err, sizeof(unsigned)));
    CK(c, cudaMemset(c->d_err, 0, sizeof(unsigned)));
    CK(c, cudaEventCreate(&c->ev0));
    CK(c, cudaEventCreate(&c->ev1));
    CK(c, cudaHostAlloc(reinterpret_cast<void**>(&c->host_box), 64, cudaHostAllocDefault));
    // Keep freed pool memory cached between products.
    cudaMemPool_t pool;
    CK(c, cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = UINT64_MAX;
    CK(c, cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    return SP3MM_OK;
}

// Per-thread default context of the reference-named entry points.
thread_local sp3mm_ctx* tl_ctx = nullptr;

sp3mm_ctx* default_ctx() {
    if (tl_ctx) return tl_ctx;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    sp3mm_ctx* c = new sp3mm_ctx();
    if (ctx_init(c, dev) != SP3MM_OK) {
        delete c;
        return nullptr;
    }
    tl_ctx = c;
    return c;
}

// ---- layer 1 helpers ------------------------------------------------------

enum { F_NONE = -1 };

int upload_spmat(sp3mm_ctx* ctx, const spmat* m, int off, sp3mm_dcsr* out) {
    if (!m) return set_error(ctx, SP3MM_EINVAL, "NULL spmat");
    return upload_u64(ctx, static_cast<long long>(m->M), static_cast<long long>(m->N),
                      static_cast<long long>(m->NZ), reinterpret_cast<const uint64_t*>(m->IRP),
                      reinterpret_cast<const uint64_t*>(m->JA), m->AS, off, SP3MM_F64, out);
}

void advise_huge(void* p, size_t bytes) {
#ifdef MADV_HUGEPAGE
    if (!p || bytes < (size_t(8) << 20)) return;
    const uintptr_t pg = 4096;
    const uintptr_t a = (reinterpret_cast<uintptr_t>(p) + pg - 1) & ~(pg - 1);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes) & ~(pg - 1);
    if (e > a) madvise(reinterpret_cast<void*>(a), e - a, MADV_HUGEPAGE);
#else
    (void)p;
    (void)bytes;
#endif
}

spmat* download_spmat(sp3mm_ctx* ctx, const sp3mm_dcsr& m, int off) {
    spmat* out = static_cast<spmat*>(calloc(1, sizeof(spmat)));
    if (!out) {
        fprintf(stderr, "sp3mm_b200: output spmat calloc failed\n");
        return nullptr;
    }
    out->M = static_cast<idx_t>(m.M);
    out->N = static_cast<idx_t>(m.N);
    out->NZ = static_cast<idx_t>(m.nnz);
    out->IRP = static_cast<idx_t*>(calloc(static_cast<size_t>(m.M) + 1, sizeof(idx_t)));
    out->JA = static_cast<idx_t*>(malloc(sizeof(idx_t) * std::max<long long>(m.nnz, 1)));
    out->AS = static_cast<double*>(malloc(sizeof(double) * std::max<long long>(m.nnz, 1)));
    // Large result arrays are written once by the host threads: ask for
    // huge pages so that the first touch takes far fewer page faults.
    advise_huge(out->JA, sizeof(idx_t) * static_cast<size_t>(std::max<long long>(m.nnz, 1)));
    advise_huge(out->AS, sizeof(double) * static_cast<size_t>(std::max<long long>(m.nnz, 1)));
    if (!out->IRP || !out->JA || !out->AS) {
        fprintf(stderr, "sp3mm_b200: output spmat arrays allocation failed\n");
        free(out->IRP);
        free(out->JA);
        free(out->AS);
        free(out);
        return nullptr;
    }
    if (download_u64(ctx, m, off, reinterpret_cast<uint64_t*>(out->IRP),
                     reinterpret_cast<uint64_t*>(out->JA), out->AS) != SP3MM_OK) {
        free(out->IRP);
        free(out->JA);
        free(out->AS);
        free(out);
        return nullptr;
    }
    return out;
}

typedef void (*chunks_fn)(unsigned long, spmat*, CONFIG*);

// Device time of `body` in seconds (events on the context stream).
template <typename F>
int timed(sp3mm_ctx* ctx, double* secs, F&& body) {
    Start = wall_seconds();
    CK(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    const int rc = body();
    CK(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    CK(ctx, cudaEventSynchronize(ctx->ev1));
    End = wall_seconds();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    *secs = ms * 1e-3;
    return rc;
}

struct Uploaded {
    sp3mm_ctx* ctx;
    std::vector<sp3mm_dcsr> mats;
    ~Uploaded() {
        for (auto& m : mats) free_dcsr_arrays(ctx, &m);
    }
};

spmat* host_spmm(spmat* A, spmat* B, CONFIG* cfg, int off, int flavour) {
    sp3mm_ctx* ctx = default_ctx();
    if (!ctx) return nullptr;
    if (!A || !B) {
        set_error(ctx, SP3MM_EINVAL, "NULL matrix");
        return nullptr;
    }
    Uploaded up{ctx, {}};
    up.mats.resize(3);
    if (upload_spmat(ctx, A, off, &up.mats[0]) || upload_spmat(ctx, B, off, &up.mats[1]))
        return nullptr;
    double secs = 0;
    const int rc = timed(ctx, &secs, [&] {
        return spmm_impl(ctx, up.mats[0], up.mats[1], flavour, SP3MM_F64, &up.mats[2]);
    });
    if (rc) return nullptr;
    ElapsedInternal = secs;
    spmat* out = download_spmat(ctx, up.mats[2], off);
    if (out && cfg && cfg->chunkDistrbFunc)
        reinterpret_cast<chunks_fn>(cfg->chunkDistrbFunc)(static_cast<unsigned long>(A->M), out,
                                                          cfg);
    return out;
}

spmat* host_sp3mm(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, int off, int variant,
                  int flavour) {
    sp3mm_ctx* ctx = default_ctx();
    if (!ctx) return nullptr;
    if (!R || !AC || !P) {
        set_error(ctx, SP3MM_EINVAL, "NULL matrix");
        return nullptr;
    }
    Uploaded up{ctx, {}};
    up.mats.resize(4);
    if (upload_spmat(ctx, R, off, &up.mats[0]) || upload_spmat(ctx, AC, off, &up.mats[1]) ||
        upload_spmat(ctx, P, off, &up.mats[2]))
        return nullptr;
    double secs = 0;
    const int rc = timed(ctx, &secs, [&] {
        return rap_impl(ctx, up.mats[0], up.mats[1], up.mats[2], variant, flavour, SP3MM_F64,
                        &up.mats[3]);
    });
    if (rc) return nullptr;
    ElapsedInternal = secs;
    spmat* out = download_spmat(ctx, up.mats[3], off);
    if (out && cfg && cfg->chunkDistrbFunc)
        reinterpret_cast<chunks_fn>(cfg->chunkDistrbFunc)(static_cast<unsigned long>(R->M), out,
                                                          cfg);
    return out;
}

idx_t* host_rowsizes(spmat* A, spmat* B, int off, bool exact) {
    sp3mm_ctx* ctx = default_ctx();
    if (!ctx) return nullptr;
    if (!A || !B) {
        set_error(ctx, SP3MM_EINVAL, "NULL matrix");
        return nullptr;
    }
    Uploaded up{ctx, {}};
    up.mats.resize(2);
    if (upload_spmat(ctx, A, off, &up.mats[0]) || upload_spmat(ctx, B, off, &up.mats[1]))
        return nullptr;
    const int M = up.mats[0].M;
    DevBuf rows;
    if (rows.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1))) return nullptr;
    int64_t total = 0;
    if (sp3mm_spmm_rowsizes(ctx, &up.mats[0], &up.mats[1], exact ? 1 : 0, rows.as<int32_t>(),
                            &total))
        return nullptr;
    std::vector<int> h(static_cast<size_t>(M) + 1);
    if (cudaMemcpyAsync(h.data(), rows.p, sizeof(int) * M, cudaMemcpyDeviceToHost,
                        ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        set_error(ctx, SP3MM_ECUDA, "row sizes readback failed");
        return nullptr;
    }
    idx_t* out = static_cast<idx_t*>(calloc(static_cast<size_t>(M) + 1, sizeof(idx_t)));
    if (!out) {
        fprintf(stderr, "sp3mm_b200: row sizes calloc failed\n");
        return nullptr;
    }
    for (int i = 0; i < M; ++i) out[i] = static_cast<idx_t>(h[i]);
    out[M] = static_cast<idx_t>(total);
    return out;
}

// SpMM entry points of this library and their flavours, to recognise the
// `spmm` argument of the pair drivers.
SPMM* const kUBFuncs[] = {&spmmSerial_0, &spmmRowByRow_0, &spmmRowByRow1DBlocks_0,
                          &spmmRowByRow2DBlocks_0, &spmmRowByRow2DBlocksAllocated_0,
                          &spmmSerial_1, &spmmRowByRow_1, &spmmRowByRow1DBlocks_1,
                          &spmmRowByRow2DBlocks_1, &spmmRowByRow2DBlocksAllocated_1};
SPMM* const kSNFuncs[] = {&spmmRowByRow_SymbNum_0, &spmmRowByRow1DBlocks_SymbNum_0,
                          &spmmRowByRow2DBlocks_SymbNum_0,
                          &spmmRowByRow2DBlocksAllocated_SymbNum_0, &spmmRowByRow_SymbNum_1,
                          &spmmRowByRow1DBlocks_SymbNum_1, &spmmRowByRow2DBlocks_SymbNum_1,
                          &spmmRowByRow2DBlocksAllocated_SymbNum_1};

int flavour_of(SPMM_INTERF f) {
    for (SPMM* g : kUBFuncs)
        if (f == g) return SP3MM_UB;
    for (SPMM* g : kSNFuncs)
        if (f == g) return SP3MM_SYMBNUM;
    return F_NONE;
}

// Pair driver: our SpMMs stay on the device; a foreign spmm is called on the
// host matrices like the reference does (Sp3MM_CSR_OMP_UB_Generic.c:475-491).
spmat* pair_driver(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, SPMM_INTERF spmm, int off,
                   int variant, int default_flavour) {
    int fl = spmm ? flavour_of(spmm) : default_flavour;
    if (fl != F_NONE) return host_sp3mm(R, AC, P, cfg, off, variant, fl);
    const double t0 = wall_seconds();
    spmat* T = variant == SP3MM_PAIR_RIGHT ? spmm(AC, P, cfg) : spmm(R, AC, cfg);
    if (!T) return nullptr;
    spmat* out = variant == SP3MM_PAIR_RIGHT ? spmm(R, T, cfg) : spmm(T, P, cfg);
    free(T->AS);
    free(T->JA);
    free(T->IRP);
    free(T);
    ElapsedInternal = wall_seconds() - t0;
    return out;
}

}  // namespace

namespace sp3mm {
int report_error(sp3mm_ctx* ctx, int code, const char* msg) {
    return set_error(ctx, code, "%s", msg);
}
}  // namespace sp3mm

// ---------------------------------------------------------------------------
// Layer 2 C ABI.
extern "C" {

int sp3mm_ctx_create(int device, sp3mm_ctx** out) {
    if (!out) return SP3MM_EINVAL;
    sp3mm_ctx* c = new sp3mm_ctx();
    const int rc = ctx_init(c, device);
    if (rc) {
        delete c;
        return rc;
    }
    *out = c;
    return SP3MM_OK;
}

int sp3mm_ctx_destroy(sp3mm_ctx* ctx) {
    if (!ctx) return SP3MM_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    pinned_cache().give(ctx->host_stage, ctx->host_stage_bytes);
    if (ctx->host_box) cudaFreeHost(ctx->host_box);
    if (tl_ctx == ctx) tl_ctx = nullptr;
    delete ctx;
    return SP3MM_OK;
}

int sp3mm_ctx_set_stream(sp3mm_ctx* ctx, void* stream) {
    if (!ctx) return SP3MM_EINVAL;
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return SP3MM_OK;
}

void* sp3mm_ctx_stream(sp3mm_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int sp3mm_ctx_set_workspace_limit(sp3mm_ctx* ctx, size_t bytes) {
    if (!ctx) return SP3MM_EINVAL;
    ctx->ws_limit = bytes;
    return SP3MM_OK;
}

int sp3mm_ctx_trim(sp3mm_ctx* ctx) {
    if (!ctx) return SP3MM_EINVAL;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    cudaMemPool_t pool;
    CK(ctx, cudaDeviceGetDefaultMemPool(&pool, ctx->device));
    CK(ctx, cudaMemPoolTrimTo(pool, 0));
    // Page-locked staging: this context's (allocated again on next use) and
    // the process-wide cache of buffers other contexts gave back.
    if (ctx->host_stage) CK(ctx, cudaFreeHost(ctx->host_stage));
    ctx->host_stage = nullptr;
    ctx->host_stage_bytes = 0;
    pinned_cache().drain();
    return SP3MM_OK;
}

const char* sp3mm_ctx_last_error(sp3mm_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

uint64_t sp3mm_ctx_launches(sp3mm_ctx* ctx) {
    (void)ctx;
    return launch_count();
}

int sp3mm_ctx_sync(sp3mm_ctx* ctx) {
    if (!ctx) return SP3MM_EINVAL;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return SP3MM_OK;
}

int sp3mm_ctx_set_tuning(sp3mm_ctx* ctx, int lanes_per_row, int d1, int d2) {
    if (!ctx) return SP3MM_EINVAL;
    if (lanes_per_row != 0 && lanes_per_row != 4 && lanes_per_row != 8 && lanes_per_row != 16 &&
        lanes_per_row != 32 && lanes_per_row != kDenseLanes)
        return set_error(ctx, SP3MM_EINVAL, "lanes per row must be 0, 4, 8, 16, 32 or %d",
                         kDenseLanes);
    if (d1 > 16 || d2 > 16) return set_error(ctx, SP3MM_EINVAL, "table shifts must be <= 16");
    ctx->tune_G = lanes_per_row;
    ctx->tune_d1 = d1;
    ctx->tune_d2 = d2;
    return SP3MM_OK;
}

int sp3mm_ctx_set_profiling(sp3mm_ctx* ctx, int on) {
    if (!ctx) return SP3MM_EINVAL;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    prof_clear(ctx);
    ctx->profiling = on != 0;
    return SP3MM_OK;
}

int sp3mm_ctx_profile_report(sp3mm_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || len == 0) return SP3MM_EINVAL;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    struct Agg {
        std::string label;
        int count;
        double total_ms, max_ms;
    };
    std::vector<Agg> agg;
    for (auto& r : ctx->prof) {
        float ms = 0.f;
        CK(ctx, cudaEventElapsedTime(&ms, r.a, r.b));
        auto it = std::find_if(agg.begin(), agg.end(),
                               [&](const Agg& a) { return a.label == r.label; });
        if (it == agg.end()) {
            agg.push_back({r.label, 1, ms, ms});
        } else {
            it->count++;
            it->total_ms += ms;
            it->max_ms = std::max(it->max_ms, static_cast<double>(ms));
        }
    }
    std::string out;
    char line[160];
    for (auto& a : agg) {
        snprintf(line, sizeof line, "%s %d %.6f %.6f\n", a.label.c_str(), a.count, a.total_ms,
                 a.max_ms);
        out += line;
    }
    snprintf(buf, len, "%s", out.c_str());
    return out.size() < len ? SP3MM_OK : SP3MM_EINVAL;
}

int sp3mm_dcsr_upload(sp3mm_ctx* ctx, const spmat* host, int off_f, int val_type,
                      sp3mm_dcsr* out) {
    if (!ctx || !host || !out || (off_f != 0 && off_f != 1)) return SP3MM_EINVAL;
    return upload_u64(ctx, static_cast<long long>(host->M), static_cast<long long>(host->N),
                      static_cast<long long>(host->NZ),
                      reinterpret_cast<const uint64_t*>(host->IRP),
                      reinterpret_cast<const uint64_t*>(host->JA), host->AS, off_f, val_type, out);
}

int sp3mm_dcsr_upload_arrays(sp3mm_ctx* ctx, int64_t M, int64_t N, int64_t nnz,
                             const int64_t* row_ptr, const int64_t* col, const double* val,
                             int val_type, sp3mm_dcsr* out) {
    if (!ctx || !out) return SP3MM_EINVAL;
    return upload_u64(ctx, M, N, nnz, reinterpret_cast<const uint64_t*>(row_ptr),
                      reinterpret_cast<const uint64_t*>(col), val, 0, val_type, out);
}

int sp3mm_dcsr_download(sp3mm_ctx* ctx, const sp3mm_dcsr* m, int off_f, spmat** out) {
    if (!ctx || !out) return SP3MM_EINVAL;
    TRY(check_dcsr(ctx, m, "matrix"));
    *out = download_spmat(ctx, *m, off_f);
    return *out ? SP3MM_OK : SP3MM_ECUDA;
}

int sp3mm_dcsr_download_arrays(sp3mm_ctx* ctx, const sp3mm_dcsr* m, int64_t* row_ptr,
                               int64_t* col, double* val) {
    if (!ctx || !row_ptr) return SP3MM_EINVAL;
    TRY(check_dcsr(ctx, m, "matrix"));
    return download_u64(ctx, *m, 0, reinterpret_cast<uint64_t*>(row_ptr),
                        reinterpret_cast<uint64_t*>(col), val);
}

int sp3mm_dcsr_set_values(sp3mm_ctx* ctx, sp3mm_dcsr* m, const double* val) {
    if (!ctx || !m) return SP3MM_EINVAL;
    TRY(check_dcsr(ctx, m, "matrix"));
    if (m->nnz > 0 && !val) return set_error(ctx, SP3MM_EINVAL, "values are NULL");
    if (m->nnz == 0) return SP3MM_OK;
    const cudaStream_t st = ctx->stream;
    if (m->val_type == SP3MM_F64) {
        CK(ctx, cudaMemcpyAsync(m->val, val, sizeof(double) * m->nnz, cudaMemcpyHostToDevice, st));
    } else {
        DevBuf stage;
        TRY(stage.alloc(ctx, sizeof(double) * m->nnz));
        CK(ctx, cudaMemcpyAsync(stage.p, val, sizeof(double) * m->nnz, cudaMemcpyHostToDevice,
                                st));
        launch_convert_values(m->nnz, stage.p, SP3MM_F64, m->val, m->val_type, st);
        CK(ctx, cudaGetLastError());
    }
    CK(ctx, cudaStreamSynchronize(st));
    return SP3MM_OK;
}

int sp3mm_dcsr_free(sp3mm_ctx* ctx, sp3mm_dcsr* m) {
    if (!ctx || !m) return SP3MM_EINVAL;
    free_dcsr_arrays(ctx, m);
    m->nnz = 0;
    return SP3MM_OK;
}

int sp3mm_spmm(sp3mm_ctx* ctx, const sp3mm_dcsr* A, const sp3mm_dcsr* B, int flavour,
               int out_val_type, sp3mm_dcsr* C) {
    if (!ctx || !C) return SP3MM_EINVAL;
    TRY(check_dcsr(ctx, A, "A"));
    TRY(check_dcsr(ctx, B, "B"));
    return spmm_impl(ctx, *A, *B, flavour, out_val_type, C);
}

int sp3mm_rap(sp3mm_ctx* ctx, const sp3mm_dcsr* R, const sp3mm_dcsr* A, const sp3mm_dcsr* P,
              int variant, int flavour, int out_val_type, sp3mm_dcsr* C) {
    if (!ctx || !C) return SP3MM_EINVAL;
    TRY(check_dcsr(ctx, R, "R"));
    TRY(check_dcsr(ctx, A, "A"));
    TRY(check_dcsr(ctx, P, "P"));
    return rap_impl(ctx, *R, *A, *P, variant, flavour, out_val_type, C);
}

int sp3mm_spmm_rowsizes(sp3mm_ctx* ctx, const sp3mm_dcsr* A, const sp3mm_dcsr* B, int exact,
                        int32_t* rows_dev, int64_t* total) {
    if (!ctx) return SP3MM_EINVAL;
    TRY(check_dcsr(ctx, A, "A"));
    TRY(check_dcsr(ctx, B, "B"));
    if (A->N != B->M) return set_error(ctx, SP3MM_EINVAL, "inner dimensions differ");
    const int M = A->M;
    const cudaStream_t st = ctx->stream;
    DevBuf cnt_buf, need, row_cnt;
    TRY(cnt_buf.alloc(ctx, sizeof(Counters)));
    TRY(need.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
    Counters* dc = cnt_buf.as<Counters>();
    CK(ctx, cudaMemsetAsync(dc, 0, sizeof(Counters), st));
    if (!exact) {
        // The upper bound proper is the per-row flop count, without the
        // distinct-column clamp the binning uses.
        sp3mm_dcsr Bfull = *B;
        Bfull.N = INT32_MAX;
        launch_pair_bounds(view(*A), view(Bfull), rows_dev ? rows_dev : need.as<int>(),
                           &dc->total, st);
        CK(ctx, cudaGetLastError());
        Counters h{};
        CK(ctx, cudaMemcpyAsync(&h, dc, sizeof h, cudaMemcpyDeviceToHost, st));
        CK(ctx, cudaStreamSynchronize(st));
        if (total) *total = static_cast<int64_t>(h.total);
        return SP3MM_OK;
    }
    TRY(row_cnt.alloc(ctx, sizeof(int) * (static_cast<size_t>(M) + 1)));
    launch_pair_bounds(view(*A), view(*B), need.as<int>(), &dc->total, st);
    const int G = pick_group(ctx, B->M ? static_cast<double>(B->nnz) / B->M : 1.0);
    const int d1 = ctx->tune_d1 >= 0 ? ctx->tune_d1 : 2;
    Bins bins;
    TRY(bin_rows(ctx, M, need.as<int>(), d1, G, dc, row_cnt.as<int>(), bins));
    RowRunner rr{ctx, false, kSymb, {}, PairRowArgs{view(*A), view(*B)}, -1, B->max_row};
    RowParams p{};
    p.nrows = M;
    p.row_cnt = row_cnt.as<int>();
    p.err = ctx->d_err;
    TRY(rr.run(bins, p, G, 0, std::min<long long>(bins.nmax, B->N), 0, dc));
    DevBuf rp;
    long long nnz = 0;
    TRY(scan_counts(ctx, M, row_cnt.as<int>(), rp, &nnz));
    TRY(check_device_err(ctx));
    if (rows_dev)
        CK(ctx, cudaMemcpyAsync(rows_dev, row_cnt.p, sizeof(int) * M, cudaMemcpyDeviceToDevice, st));
    CK(ctx, cudaStreamSynchronize(st));
    if (total) *total = nnz;
    return SP3MM_OK;
}

int sp3mm_transpose(sp3mm_ctx* ctx, const sp3mm_dcsr* A, sp3mm_dcsr* AT) {
    if (!ctx || !AT) return SP3MM_EINVAL;
    TRY(check_dcsr(ctx, A, "A"));
    const cudaStream_t st = ctx->stream;
    DevBuf rp, ci, v, counts, cursor;
    TRY(counts.alloc(ctx, sizeof(int) * (static_cast<size_t>(A->N) + 1)));
    TRY(cursor.alloc(ctx, sizeof(int) * (static_cast<size_t>(A->N) + 1)));
    CK(ctx, cudaMemsetAsync(counts.p, 0, sizeof(int) * (static_cast<size_t>(A->N) + 1), st));
    CK(ctx, cudaMemsetAsync(cursor.p, 0, sizeof(int) * (static_cast<size_t>(A->N) + 1), st));
    launch_col_counts(A->nnz, A->col, counts.as<int>(), st);
    long long nnz = 0;
    TRY(scan_counts(ctx, A->N, counts.as<int>(), rp, &nnz));
    TRY(ci.alloc(ctx, sizeof(int) * static_cast<size_t>(A->nnz)));
    TRY(v.alloc(ctx, vbytes(A->val_type) * static_cast<size_t>(A->nnz)));
    launch_transpose_scatter(view(*A), rp.as<int>(), cursor.as<int>(), ci.as<int>(), v.p, st);
    // The scatter order within a row is arbitrary: sort (the sort kernels
    // skip the rows they do not handle, so they run without knowing the
    // longest row), then validate, which also finds the longest row.
    launch_sort_rows(A->N, rp.as<int>(), ci.as<int>(), v.p, A->val_type, INT_MAX, st);
    CK(ctx, cudaGetLastError());
    DevBuf mr;
    TRY(mr.alloc(ctx, sizeof(int)));
    CK(ctx, cudaMemsetAsync(mr.p, 0, sizeof(int), st));
    launch_validate_i32(A->N, A->M, rp.as<int>(), ci.as<int>(), mr.as<int>(), ctx->d_err, st);
    int max_row = 0;
    CK(ctx, cudaMemcpyAsync(&max_row, mr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY(check_device_err(ctx));   // synchronises: max_row is complete
    AT->M = A->N;
    AT->N = A->M;
    AT->nnz = A->nnz;
    AT->val_type = A->val_type;
    AT->max_row = max_row;
    return finish_matrix(AT, rp, ci, v);
}

int sp3mm_rap_memory_estimate(const sp3mm_dcsr* R, const sp3mm_dcsr* A, const sp3mm_dcsr* P,
                              int variant, int flavour, size_t* bytes) {
    if (!R || !A || !P || !bytes) return SP3MM_EINVAL;
    auto mr = [](const sp3mm_dcsr* m) -> double {
        return m->max_row >= 0 ? m->max_row : (m->M ? static_cast<double>(m->N) : 0.0);
    };
    // Multiply-add bounds: nnz(X) * longest row of the right operand.
    const double f_ra = R->nnz * mr(A);
    const double f_rap = f_ra * mr(P);
    const double f_ap = A->nnz * mr(P);
    double b = 0;
    const double row_ws = 32.0;   // per-row work arrays (need, level, lists, counts, offsets)
    auto spmm_bytes = [&](double M, double flops) {
        double s = M * row_ws + std::min(flops, 1e15) * 12.0 * (flavour == SP3MM_UB ? 2 : 1);
        return s;
    };
    if (variant == SP3MM_DIRECT) {
        b = spmm_bytes(R->M, f_rap);
    } else if (variant == SP3MM_PAIR) {
        b = spmm_bytes(R->M, f_ra) + f_ra * 12.0 + spmm_bytes(R->M, f_ra * mr(P));
    } else {
        b = spmm_bytes(A->M, f_ap) + f_ap * 12.0 + spmm_bytes(R->M, R->nnz * std::min(f_ap, 1e15));
    }
    b += 64.0 * 1024 * 1024;   // global-table scratch and scan temporaries
    *bytes = static_cast<size_t>(std::min(b, 1.8e19));
    return SP3MM_OK;
}

// ---------------------------------------------------------------------------
// Layer 1: reference entry points.

#define SP3MM_REF_SPMM(name, off, flav) \
    spmat* name(spmat* A, spmat* B, CONFIG* cfg) { return host_spmm(A, B, cfg, off, flav); }

SP3MM_REF_SPMM(spmmSerial_0, 0, SP3MM_UB)
SP3MM_REF_SPMM(spmmSerial_1, 1, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow_0, 0, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow_1, 1, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow1DBlocks_0, 0, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow1DBlocks_1, 1, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow2DBlocks_0, 0, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow2DBlocks_1, 1, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow2DBlocksAllocated_0, 0, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow2DBlocksAllocated_1, 1, SP3MM_UB)
SP3MM_REF_SPMM(spmmRowByRow_SymbNum_0, 0, SP3MM_SYMBNUM)
SP3MM_REF_SPMM(spmmRowByRow_SymbNum_1, 1, SP3MM_SYMBNUM)
SP3MM_REF_SPMM(spmmRowByRow1DBlocks_SymbNum_0, 0, SP3MM_SYMBNUM)
SP3MM_REF_SPMM(spmmRowByRow1DBlocks_SymbNum_1, 1, SP3MM_SYMBNUM)
SP3MM_REF_SPMM(spmmRowByRow2DBlocks_SymbNum_0, 0, SP3MM_SYMBNUM)
SP3MM_REF_SPMM(spmmRowByRow2DBlocks_SymbNum_1, 1, SP3MM_SYMBNUM)
SP3MM_REF_SPMM(spmmRowByRow2DBlocksAllocated_SymbNum_0, 0, SP3MM_SYMBNUM)
SP3MM_REF_SPMM(spmmRowByRow2DBlocksAllocated_SymbNum_1, 1, SP3MM_SYMBNUM)

spmat* sp3mmRowByRowPair_0(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, SPMM_INTERF spmm) {
    return pair_driver(R, AC, P, cfg, spmm ? spmm : &spmmRowByRow2DBlocks_0, 0, SP3MM_PAIR,
                       SP3MM_UB);
}
spmat* sp3mmRowByRowPair_1(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, SPMM_INTERF spmm) {
    return pair_driver(R, AC, P, cfg, spmm ? spmm : &spmmRowByRow2DBlocks_1, 1, SP3MM_PAIR,
                       SP3MM_UB);
}
spmat* sp3mmRowByRowPair_SymbNum_0(spmat* R, spmat* AC, spmat* P, CONFIG* cfg,
                                   SPMM_INTERF spmm) {
    return pair_driver(R, AC, P, cfg, spmm ? spmm : &spmmRowByRow_SymbNum_0, 0, SP3MM_PAIR,
                       SP3MM_SYMBNUM);
}
spmat* sp3mmRowByRowPair_SymbNum_1(spmat* R, spmat* AC, spmat* P, CONFIG* cfg,
                                   SPMM_INTERF spmm) {
    return pair_driver(R, AC, P, cfg, spmm ? spmm : &spmmRowByRow_SymbNum_1, 1, SP3MM_PAIR,
                       SP3MM_SYMBNUM);
}
spmat* sp3mmRowByRowPairRight_0(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, SPMM_INTERF spmm) {
    return pair_driver(R, AC, P, cfg, spmm, 0, SP3MM_PAIR_RIGHT, SP3MM_UB);
}
spmat* sp3mmRowByRowPairRight_1(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, SPMM_INTERF spmm) {
    return pair_driver(R, AC, P, cfg, spmm, 1, SP3MM_PAIR_RIGHT, SP3MM_UB);
}
spmat* sp3mmRowByRowMerged_0(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, SPMM_INTERF spmm) {
    (void)spmm;
    return host_sp3mm(R, AC, P, cfg, 0, SP3MM_DIRECT, SP3MM_UB);
}
spmat* sp3mmRowByRowMerged_1(spmat* R, spmat* AC, spmat* P, CONFIG* cfg, SPMM_INTERF spmm) {
    (void)spmm;
    return host_sp3mm(R, AC, P, cfg, 1, SP3MM_DIRECT, SP3MM_UB);
}
spmat* sp3mmRowByRowMerged_SymbNum_0(spmat* R, spmat* AC, spmat* P, CONFIG* cfg,
                                     SPMM_INTERF spmm) {
    (void)spmm;
    return host_sp3mm(R, AC, P, cfg, 0, SP3MM_DIRECT, SP3MM_SYMBNUM);
}
spmat* sp3mmRowByRowMerged_SymbNum_1(spmat* R, spmat* AC, spmat* P, CONFIG* cfg,
                                     SPMM_INTERF spmm) {
    (void)spmm;
    return host_sp3mm(R, AC, P, cfg, 1, SP3MM_DIRECT, SP3MM_SYMBNUM);
}

idx_t* SpMM_Symb___0(ROW_MMSYM_IMPL_MODE mode, spmat* a, spmat* b) {
    (void)mode;
    return host_rowsizes(a, b, 0, true);
}
idx_t* SpMM_Symb___1(ROW_MMSYM_IMPL_MODE mode, spmat* a, spmat* b) {
    (void)mode;
    return host_rowsizes(a, b, 1, true);
}
idx_t* spMMSizeUpperbound_0(spmat* A, spmat* B) { return host_rowsizes(A, B, 0, false); }
idx_t* spMMSizeUpperbound_1(spmat* A, spmat* B) { return host_rowsizes(A, B, 1, false); }

static idx_t* colparts_ub(spmat* A, spmat* B, unsigned short gridCols, idx_t* offs, int off) {
    sp3mm_ctx* ctx = default_ctx();
    if (!ctx) return nullptr;
    if (!A || !B || !offs || gridCols == 0) {
        set_error(ctx, SP3MM_EINVAL, "invalid column-partition arguments");
        return nullptr;
    }
    Uploaded up{ctx, {}};
    up.mats.resize(2);
    if (upload_spmat(ctx, A, off, &up.mats[0]) || upload_spmat(ctx, B, off, &up.mats[1]))
        return nullptr;
    const size_t parts = static_cast<size_t>(A->M) * gridCols;
    const size_t noff = static_cast<size_t>(B->M) * gridCols + 1;
    DevBuf d_off, d_out, d_tot;
    if (d_off.alloc(ctx, sizeof(long long) * noff) || d_out.alloc(ctx, sizeof(long long) * (parts + 1)) ||
        d_tot.alloc(ctx, sizeof(unsigned long long)))
        return nullptr;
    idx_t* out = static_cast<idx_t*>(calloc(parts + 1, sizeof(idx_t)));
    if (!out) {
        fprintf(stderr, "sp3mm_b200: colparts calloc failed\n");
        return nullptr;
    }
    unsigned long long tot = 0;
    if (cudaMemcpyAsync(d_off.p, offs, sizeof(long long) * noff, cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(d_tot.p, 0, sizeof(unsigned long long), ctx->stream) != cudaSuccess) {
        free(out);
        set_error(ctx, SP3MM_ECUDA, "colparts upload failed");
        return nullptr;
    }
    launch_colparts_ub(view(up.mats[0]), gridCols, d_off.as<long long>(), d_out.as<long long>(),
                       d_tot.as<unsigned long long>(), ctx->stream);
    if (cudaMemcpyAsync(out, d_out.p, sizeof(long long) * parts, cudaMemcpyDeviceToHost,
                        ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(&tot, d_tot.p, sizeof tot, cudaMemcpyDeviceToHost, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        free(out);
        set_error(ctx, SP3MM_ECUDA, "colparts readback failed");
        return nullptr;
    }
    out[parts] = static_cast<idx_t>(tot);
    return out;
}

idx_t* spMMSizeUpperboundColParts_0(spmat* A, spmat* B, unsigned short gridCols, idx_t* o) {
    return colparts_ub(A, B, gridCols, o, 0);
}
idx_t* spMMSizeUpperboundColParts_1(spmat* A, spmat* B, unsigned short gridCols, idx_t* o) {
    return colparts_ub(A, B, gridCols, o, 1);
}

}  // extern "C"
