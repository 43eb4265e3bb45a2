// context.cuh -- the device context and host helpers shared by the host
// runtime files (products, batches, hierarchies).  Internal to the library.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "kernels.cuh"
#include "sp3mm_internal.cuh"

struct sp3mm_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    unsigned* d_err = nullptr;           // sticky device error word
    size_t ws_limit = 0;
    size_t smem_budget = 110 * 1024;
    size_t smem_optin = 227 * 1024;      // largest dynamic shared memory per CTA
    // Row-kernel tuning: lanes per row (0: from the operands' mean row
    // length), table-size shifts d1 (first table from bound >> d1; < 0:
    // default) and d2 (direct second table = first >> d2).
    int tune_G = 0, tune_d1 = -1, tune_d2 = -1;
    std::string last_error;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Optional per-launch timing (events on the context stream).
    struct ProfRec {
        const char* label;
        cudaEvent_t a, b;
    };
    bool profiling = false;
    std::vector<ProfRec> prof;
    // Last free-memory reading (cudaMemGetInfo costs milliseconds): the
    // free bytes, the pool's reserved bytes then, and when it was taken.
    size_t free_at_check = 0;
    uint64_t reserved_at_check = 0;
    double free_checked_s = -1.0;
    // Pinned host staging for downloads (grown on demand, freed with the
    // context).
    void* host_stage = nullptr;
    size_t host_stage_bytes = 0;
    // Pinned words the product tail reads back in one round trip (row
    // count total, longest row, retry count, error word).
    unsigned* host_box = nullptr;
};

namespace sp3mm {

// Record a formatted message as the context's last error (and print it);
// returns `code`.
int set_error(sp3mm_ctx* ctx, int code, const char* fmt, ...);

#define CK(ctx, call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ::sp3mm::set_error((ctx), SP3MM_ECUDA, "%s failed: %s (%s:%d)", #call, \
                                      cudaGetErrorString(e_), __FILE__, __LINE__);      \
    } while (0)

#define TRY(expr)                        \
    do {                                 \
        int rc_ = (expr);                \
        if (rc_ != SP3MM_OK) return rc_; \
    } while (0)

// Run `f` (which launches kernels on ctx->stream), bracketed by events when
// profiling is on.
template <typename F>
void prof(sp3mm_ctx* ctx, const char* label, F&& f) {
    if (!ctx->profiling) {
        f();
        return;
    }
    sp3mm_ctx::ProfRec r{label, nullptr, nullptr};
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    cudaEventRecord(r.a, ctx->stream);
    f();
    cudaEventRecord(r.b, ctx->stream);
    ctx->prof.push_back(r);
}

// Events around a phase of several launches and host steps (profiling
// only): the span ends at end() or when it goes out of scope, on any path.
// Its time includes the gaps in which the stream waited for the host.
struct ProfSpan {
    sp3mm_ctx* ctx;
    sp3mm_ctx::ProfRec r{nullptr, nullptr, nullptr};
    ProfSpan(sp3mm_ctx* c, const char* label) : ctx(c) {
        if (!ctx->profiling) return;
        r.label = label;
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        cudaEventRecord(r.a, ctx->stream);
    }
    void end() {
        if (!r.a) return;
        cudaEventRecord(r.b, ctx->stream);
        ctx->prof.push_back(r);
        r.a = nullptr;
    }
    ~ProfSpan() { end(); }
    ProfSpan(const ProfSpan&) = delete;
    ProfSpan& operator=(const ProfSpan&) = delete;
};

// Stream-ordered device allocation from the device's memory pool.
struct DevBuf {
    sp3mm_ctx* ctx = nullptr;
    void* p = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    int alloc(sp3mm_ctx* c, size_t bytes) {
        release();
        ctx = c;
        if (bytes == 0) bytes = 16;
        cudaError_t e = cudaMallocAsync(&p, bytes, c->stream);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return set_error(c, SP3MM_ENOMEM, "device allocation of %zu bytes failed: %s", bytes,
                             cudaGetErrorString(e));
        }
        return SP3MM_OK;
    }
    void release() {
        if (p && ctx) cudaFreeAsync(p, ctx->stream);
        p = nullptr;
    }
    void* detach() {
        void* q = p;
        p = nullptr;
        return q;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

inline CsrView view(const sp3mm_dcsr& m) {
    return CsrView{m.M, m.N, m.nnz, m.row_ptr, m.col, m.val, m.val_type};
}

inline size_t vbytes(int vt) { return vt == SP3MM_F32 ? 4 : 8; }

int check_dcsr(sp3mm_ctx* ctx, const sp3mm_dcsr* m, const char* what);

// Small device block of counters used by one binning pass.
struct Counters {
    int counts[kLevels + 1];
    int cursors[kLevels];
    int nmax;
    int retry_count;
    unsigned long long total;
    unsigned long long cursor;
};

// Row lists by level, built from per-row `need`.
struct Bins {
    int counts[kLevels + 1] = {};
    int offsets[kLevels] = {};
    int nmax = 0;
    unsigned long long total = 0;
    DevBuf level, lists;
};

// Device memory available to new allocations: free HBM plus the idle part
// of the device's memory pool.
size_t free_device_bytes(sp3mm_ctx* ctx);
// Bytes the device's memory pool holds reserved but unused (a cheap query).
size_t pool_idle_bytes(sp3mm_ctx* ctx);
// Map `bytes` into the device's memory pool now (one allocation, freed at
// once; the pool keeps freed memory), unless it holds that much idle
// already: later allocations then do not wait for the pool to grow, which
// takes 0.1-0.3 s per growth step and holds up the process's other threads'
// CUDA calls meanwhile.  Failure is not an error (the pool grows on demand).
void pool_reserve(sp3mm_ctx* ctx, size_t bytes);
int read_err(sp3mm_ctx* ctx, unsigned* out);
// Read and clear the sticky device error word; map it to a return code.
int check_device_err(sp3mm_ctx* ctx);
// Bin M rows by need[i] >> shift (or est[i]) for groups of G lanes; `dcnt` is the
// device counter block (its `total` was accumulated by the bounds kernel);
// row_cnt of empty rows is zeroed when given.  Synchronises the stream once.
int bin_rows(sp3mm_ctx* ctx, int M, const int* need, int shift, int G, Counters* dcnt,
             int* row_cnt, Bins& b, const int* est = nullptr);

}  // namespace sp3mm
