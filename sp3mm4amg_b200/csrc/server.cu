// server.cu -- a setup-request server with continuous batching.
//
// A request is an operator A0 (host CSR) whose hierarchy is to be built on
// the device (the product chain of code/scripts/getLevels3MMmatrixes.py:
// 29-38): on a box grid by smoothed block aggregation, or with prolongators
// P_0, P_1, ... that the caller provides (R_l = P_l^T is formed on the
// device).  Every engine step
//
//   1. admits queued requests, first come first served, while a slot is
//      free and the request's device-memory estimate fits both the server's
//      budget (what admitted requests have reserved) and the HBM free right
//      now (cudaMemGetInfo plus the idle part of the memory pool), and hands
//      them to the loader threads, which upload them on their own contexts
//      and streams while this step's kernels run (copies overlap compute;
//      two loaders keep two uploads, each narrowing on host threads, in
//      flight);
//   2. lets the requests the loaders have finished join, waiting for them
//      only when nothing else could run;
//   3. advances every joined hierarchy by one level in one level step
//      (hierarchy_step: batched launches shared by all requests, whatever
//      their level or size, so requests admitted while others are in flight
//      share the device with them);
//   4. retires the hierarchies that are complete.
//
// Results do not depend on what else is in a step: each product's rows are
// computed by the same arithmetic whatever the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdint>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "context.cuh"
#include "hierarchy.cuh"
#include "sp3mm_b200.h"

using namespace sp3mm;

namespace {

double now_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

enum { kQueued = 0, kActive = 1, kDone = 2, kFailed = 3, kTaken = 4 };

// A borrowed host CSR (0-based int64 indices, FP64 values).
struct HostCsr {
    int64_t M = 0, N = 0, nnz = 0;
    const int64_t* rp = nullptr;
    const int64_t* ci = nullptr;
    const double* v = nullptr;
};

struct Request {
    int64_t id = 0;
    int64_t M = 0, nnz = 0;
    const int64_t* rp = nullptr;
    const int64_t* ci = nullptr;
    const double* v = nullptr;
    // Caller-provided prolongators (empty: block aggregation on dims).
    std::vector<HostCsr> P;
    int32_t dims[3] = {1, 1, 1};
    int ndim = 1, block = 2, max_levels = 1, cvt = SP3MM_F64;
    long long min_coarse = 0;
    double omega = 2.0 / 3.0;
    double t_arrival = 0, t_admit = -1, t_done = -1;
    size_t est = 0;
    size_t held = 0;   // bytes of the budget reserved while admitted
    bool loading = false;   // with a loader thread (reported as active)
    int status = kQueued;
    int error = SP3MM_OK;
    sp3mm_hierarchy* h = nullptr;
};

// Device bytes a request may hold at once: its operator and, per level,
// prolongator, restriction, the A*P0 product and the next operator (each
// at most the size of the level's operator for aggregation by blocks),
// plus the per-row work arrays of the level step.  Coarse levels shrink at
// least geometrically, which the factor 2 over level 0 covers.
size_t request_estimate(int64_t M, int64_t nnz) {
    const size_t a = static_cast<size_t>(M + 1) * 4 + static_cast<size_t>(nnz) * 12;
    const size_t level0 = a /* A0 */ + 5 * a /* P, R, A*P0, A1, booking */ +
                          static_cast<size_t>(M) * 48 /* work arrays */;
    return 2 * level0;
}

// A request with given prolongators also holds them and their transposes.
size_t request_estimate_ops(int64_t M, int64_t nnz, const std::vector<HostCsr>& P) {
    size_t e = request_estimate(M, nnz);
    for (const HostCsr& p : P)
        e += 2 * (static_cast<size_t>(p.M + 1) * 4 + static_cast<size_t>(p.N + 1) * 4 +
                  static_cast<size_t>(p.nnz) * 12);
    return e;
}

size_t free_hbm(sp3mm_ctx* ctx) { return free_device_bytes(ctx); }

}  // namespace

struct sp3mm_server {
    sp3mm_ctx* ctx = nullptr;
    int max_active = 64;
    double mem_fraction = 0.5;
    size_t budget = 0, reserved = 0;
    std::chrono::steady_clock::time_point t0;
    int64_t next_id = 0;
    std::deque<int64_t> queue;
    std::vector<int64_t> active;
    std::unordered_map<int64_t, Request> reqs;
    // Loader threads: admitted requests are uploaded on their own contexts.
    static constexpr int kLoaders = 2;
    sp3mm_ctx* loader_ctx[kLoaders] = {};
    std::thread loader[kLoaders];
    std::mutex mu;
    std::condition_variable wake, done;
    std::deque<Request*> to_load;    // guarded by mu
    std::vector<Request*> loaded;    // guarded by mu
    int in_loader = 0;               // guarded by mu
    bool stop = false;               // guarded by mu
    // Statistics.
    std::vector<double> latency;
    long long products = 0, steps = 0, admitted = 0, deferred = 0;
    int peak_active = 0;
    double busy = 0;

    ~sp3mm_server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        wake.notify_all();
        for (auto& t : loader)
            if (t.joinable()) t.join();
        for (auto& kv : reqs)
            if (kv.second.h && kv.second.status != kTaken) sp3mm_hierarchy_free(ctx, kv.second.h);
        for (sp3mm_ctx* c : loader_ctx)
            if (c) sp3mm_ctx_destroy(c);
    }
};

namespace {

// Upload a request's operator on a loader context (the call returns once
// the copy and its validation are complete) and wrap it in a hierarchy.
// The operator is freed on the server's context, after the work that uses it.
int admit(sp3mm_server* s, sp3mm_ctx* lctx, Request& r) {
    sp3mm_ctx* ctx = s->ctx;
    auto A0 = std::shared_ptr<sp3mm_dcsr>(new sp3mm_dcsr{}, [ctx](sp3mm_dcsr* m) {
        sp3mm_dcsr_free(ctx, m);
        delete m;
    });
    TRY(sp3mm_dcsr_upload_arrays(lctx, r.M, r.M, r.nnz, r.rp, r.ci, r.v, SP3MM_F64,
                                 A0.get()));
    auto* h = new sp3mm_hierarchy();
    h->ndim = r.ndim;
    h->block = r.block;
    h->omega = r.omega;
    h->min_coarse = r.min_coarse;
    h->max_levels = r.max_levels;
    h->coarse_val_type = r.cvt;
    h->owns_arrays = false;
    h->A.push_back(*A0);
    h->nx.push_back(r.dims[0]);
    h->ny.push_back(r.ndim > 1 ? r.dims[1] : 1);
    h->nz.push_back(r.ndim > 2 ? r.dims[2] : 1);
    h->nlev = 1;
    h->keep.push_back(A0);
    r.h = h;
    // Given prolongators: level 0 in FP64, coarser ones in the coarse
    // storage type (each product's operands share one value type).
    for (size_t l = 0; l < r.P.size(); ++l) {
        const HostCsr& hp = r.P[l];
        auto P = std::shared_ptr<sp3mm_dcsr>(new sp3mm_dcsr{}, [ctx](sp3mm_dcsr* m) {
            sp3mm_dcsr_free(ctx, m);
            delete m;
        });
        TRY(sp3mm_dcsr_upload_arrays(lctx, hp.M, hp.N, hp.nnz, hp.rp, hp.ci, hp.v,
                                     l == 0 ? SP3MM_F64 : r.cvt, P.get()));
        h->given_P.push_back(*P);
        h->keep.push_back(P);
    }
    return SP3MM_OK;
}

void loader_main(sp3mm_server* s, sp3mm_ctx* lctx) {
    cudaSetDevice(s->ctx->device);
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->wake.wait(lk, [&] { return s->stop || !s->to_load.empty(); });
            if (s->stop) return;
            r = s->to_load.front();
            s->to_load.pop_front();
        }
        r->error = admit(s, lctx, *r);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->loaded.push_back(r);
            --s->in_loader;
        }
        s->done.notify_all();
    }
}

void finish(sp3mm_server* s, Request& r, int status, double t) {
    r.status = status;
    r.t_done = t;
    s->reserved -= std::min(s->reserved, r.held);
    r.held = 0;
    if (status == kDone) {
        s->latency.push_back(r.t_done - r.t_arrival);
        s->products += r.h ? r.h->nlev - 1 : 0;
    }
}

}  // namespace

extern "C" {

int sp3mm_server_create(sp3mm_ctx* ctx, int max_active, double mem_fraction,
                        sp3mm_server** out) {
    if (!ctx || !out || max_active < 1 || !(mem_fraction > 0.0 && mem_fraction <= 1.0))
        return set_error(ctx, SP3MM_EINVAL, "server: invalid arguments");
    auto* s = new sp3mm_server();
    s->ctx = ctx;
    s->max_active = max_active;
    s->mem_fraction = mem_fraction;
    s->budget = static_cast<size_t>(mem_fraction * static_cast<double>(free_hbm(ctx)));
    // The budget is mapped into the memory pool up front, so that admitting
    // requests never waits for the pool to grow (which stalls the loader
    // threads' copies too).
    pool_reserve(ctx, s->budget);
    s->t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < sp3mm_server::kLoaders; ++k) {
        const int rc = sp3mm_ctx_create(ctx->device, &s->loader_ctx[k]);
        if (rc != SP3MM_OK) {
            delete s;
            return set_error(ctx, rc, "server: loader context creation failed");
        }
    }
    for (int k = 0; k < sp3mm_server::kLoaders; ++k)
        s->loader[k] = std::thread(loader_main, s, s->loader_ctx[k]);
    *out = s;
    return SP3MM_OK;
}

double sp3mm_server_now(const sp3mm_server* s) { return s ? now_s(s->t0) : 0.0; }

int sp3mm_server_submit(sp3mm_server* s, int64_t M, int64_t nnz, const int64_t* row_ptr,
                        const int64_t* col, const double* val, const int32_t* dims, int ndim,
                        int block, double omega, int64_t min_coarse, int max_levels,
                        int coarse_val_type, double arrival, int64_t* id) {
    if (!s || !row_ptr || (nnz > 0 && (!col || !val)) || !dims || !id || ndim < 1 || ndim > 3 ||
        block < 2 || max_levels < 1 || M < 1 ||
        (coarse_val_type != SP3MM_F64 && coarse_val_type != SP3MM_F32))
        return set_error(s ? s->ctx : nullptr, SP3MM_EINVAL, "server: invalid request");
    long long n = 1;
    for (int d = 0; d < ndim; ++d) {
        if (dims[d] < 1) return set_error(s->ctx, SP3MM_EINVAL, "server: invalid grid");
        n *= dims[d];
    }
    if (n != M) return set_error(s->ctx, SP3MM_EINVAL, "server: grid does not match A0");
    Request r;
    r.id = s->next_id++;
    r.M = M;
    r.nnz = nnz;
    r.rp = row_ptr;
    r.ci = col;
    r.v = val;
    for (int d = 0; d < ndim; ++d) r.dims[d] = dims[d];
    r.ndim = ndim;
    r.block = block;
    r.omega = omega;
    r.min_coarse = min_coarse;
    r.max_levels = max_levels;
    r.cvt = coarse_val_type;
    r.t_arrival = arrival >= 0 ? arrival : now_s(s->t0);
    r.est = request_estimate(M, nnz);
    s->reqs[r.id] = r;
    s->queue.push_back(r.id);
    *id = r.id;
    return SP3MM_OK;
}

int sp3mm_server_submit_ops(sp3mm_server* s, int64_t M, int64_t nnz, const int64_t* row_ptr,
                            const int64_t* col, const double* val, int np,
                            const int64_t* p_rows, const int64_t* p_cols, const int64_t* p_nnz,
                            const int64_t* const* p_row_ptr, const int64_t* const* p_col,
                            const double* const* p_val, int coarse_val_type, double arrival,
                            int64_t* id) {
    if (!s || !row_ptr || (nnz > 0 && (!col || !val)) || !id || M < 1 || np < 1 ||
        !p_rows || !p_cols || !p_nnz || !p_row_ptr || !p_col || !p_val ||
        (coarse_val_type != SP3MM_F64 && coarse_val_type != SP3MM_F32))
        return set_error(s ? s->ctx : nullptr, SP3MM_EINVAL, "server: invalid request");
    Request r;
    int64_t rows = M;
    for (int l = 0; l < np; ++l) {
        if (p_rows[l] != rows || p_cols[l] < 1 || p_nnz[l] < 0 || !p_row_ptr[l] ||
            (p_nnz[l] > 0 && (!p_col[l] || !p_val[l])))
            return set_error(s->ctx, SP3MM_EINVAL,
                             "server: prolongator %d does not follow its level's size", l);
        HostCsr hp;
        hp.M = p_rows[l];
        hp.N = p_cols[l];
        hp.nnz = p_nnz[l];
        hp.rp = p_row_ptr[l];
        hp.ci = p_col[l];
        hp.v = p_val[l];
        r.P.push_back(hp);
        rows = p_cols[l];
    }
    r.id = s->next_id++;
    r.M = M;
    r.nnz = nnz;
    r.rp = row_ptr;
    r.ci = col;
    r.v = val;
    r.dims[0] = static_cast<int32_t>(std::min<int64_t>(M, INT32_MAX));
    r.ndim = 1;
    r.max_levels = np + 1;
    r.cvt = coarse_val_type;
    r.t_arrival = arrival >= 0 ? arrival : now_s(s->t0);
    r.est = request_estimate_ops(M, nnz, r.P);
    const int64_t rid = r.id;
    s->reqs[rid] = std::move(r);
    s->queue.push_back(rid);
    *id = rid;
    return SP3MM_OK;
}

int sp3mm_server_step(sp3mm_server* s, int* pending) {
    if (!s) return SP3MM_EINVAL;
    sp3mm_ctx* ctx = s->ctx;
    const double t_begin = now_s(s->t0);
    int in_loader = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        in_loader = s->in_loader + static_cast<int>(s->loaded.size());
    }
    // 1. Admission, first come first served; uploads go to the loaders.
    std::vector<Request*> handed;
    while (!s->queue.empty() &&
           static_cast<int>(s->active.size()) + in_loader < s->max_active) {
        Request& r = s->reqs[s->queue.front()];
        if (r.est > s->budget) {   // can never fit: refuse instead of blocking
            r.error = SP3MM_ENOMEM;
            s->queue.pop_front();
            finish(s, r, kFailed, now_s(s->t0));
            continue;
        }
        if (s->reserved + r.est > s->budget || r.est > free_hbm(ctx)) {
            ++s->deferred;
            break;
        }
        s->queue.pop_front();
        r.status = kActive;
        r.loading = true;
        r.t_admit = now_s(s->t0);
        s->reserved += r.est;
        r.held = r.est;
        handed.push_back(&r);
        ++in_loader;
        ++s->admitted;
    }
    if (!handed.empty()) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (Request* r : handed) s->to_load.push_back(r);
            s->in_loader += static_cast<int>(handed.size());
        }
        s->wake.notify_all();
    }
    // 2. Requests the loaders have finished join; wait only when nothing
    //    else could run.
    {
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->active.empty() && s->loaded.empty() && s->in_loader > 0)
            s->done.wait(lk, [&] { return !s->loaded.empty(); });
        for (Request* r : s->loaded) {
            r->loading = false;
            r->rp = nullptr;
            r->ci = nullptr;
            r->v = nullptr;
            r->P.clear();
            if (r->error != SP3MM_OK) {
                if (r->h) sp3mm_hierarchy_free(ctx, r->h);
                r->h = nullptr;
                finish(s, *r, kFailed, now_s(s->t0));
            } else {
                s->active.push_back(r->id);
            }
        }
        s->loaded.clear();
        in_loader = s->in_loader;
    }
    s->peak_active = std::max(s->peak_active, static_cast<int>(s->active.size()));
    // 3. One level for every joined hierarchy.
    std::vector<sp3mm_hierarchy*> hs;
    for (int64_t id : s->active) hs.push_back(s->reqs[id].h);
    if (!hs.empty()) {
        int rc = hierarchy_step(ctx, hs);
        if (rc != SP3MM_OK) {
            // Find the failing requests: step each one alone.
            for (int64_t id : s->active) {
                Request& r = s->reqs[id];
                if (!r.h->wants_level()) continue;
                const int rc1 = hierarchy_step(ctx, {r.h});
                if (rc1 != SP3MM_OK) {
                    r.error = rc1;
                    finish(s, r, kFailed, now_s(s->t0));
                }
            }
            cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), ctx->stream);
        }
        ++s->steps;
    }
    // 4. Retire complete hierarchies.
    const double t = now_s(s->t0);
    std::vector<int64_t> still;
    for (int64_t id : s->active) {
        Request& r = s->reqs[id];
        if (r.status == kFailed) continue;
        if (r.h->wants_level()) still.push_back(id);
        else finish(s, r, kDone, t);
    }
    s->active.swap(still);
    s->busy += t - t_begin;
    if (pending)
        *pending = static_cast<int>(s->queue.size() + s->active.size()) + in_loader;
    return SP3MM_OK;
}

int sp3mm_server_poll(const sp3mm_server* s, int64_t id, int* status, double* latency,
                      double* queued) {
    if (!s) return SP3MM_EINVAL;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return SP3MM_EINVAL;
    const Request& r = it->second;
    if (status) *status = r.status;
    if (latency) *latency = r.t_done >= 0 ? r.t_done - r.t_arrival : -1.0;
    if (queued) *queued = r.t_admit >= 0 ? r.t_admit - r.t_arrival : -1.0;
    return r.status == kFailed ? r.error : SP3MM_OK;
}

int sp3mm_server_take(sp3mm_server* s, int64_t id, sp3mm_hierarchy** h) {
    if (!s || !h) return SP3MM_EINVAL;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end() || it->second.status != kDone) return SP3MM_EINVAL;
    *h = it->second.h;
    it->second.h = nullptr;
    it->second.status = kTaken;
    return SP3MM_OK;
}

int sp3mm_server_stats(const sp3mm_server* s, int64_t* completed, int64_t* products,
                       double* p50, double* p99, double* busy_s, int64_t* steps,
                       int* peak_active, int64_t* deferred) {
    if (!s) return SP3MM_EINVAL;
    std::vector<double> l = s->latency;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
        if (l.empty()) return 0.0;
        const size_t k = static_cast<size_t>(q * (l.size() - 1) + 0.5);
        return l[std::min(k, l.size() - 1)];
    };
    if (completed) *completed = static_cast<int64_t>(l.size());
    if (products) *products = s->products;
    if (p50) *p50 = pct(0.50);
    if (p99) *p99 = pct(0.99);
    if (busy_s) *busy_s = s->busy;
    if (steps) *steps = s->steps;
    if (peak_active) *peak_active = s->peak_active;
    if (deferred) *deferred = s->deferred;
    return SP3MM_OK;
}

int sp3mm_server_free(sp3mm_server* s) {
    if (!s) return SP3MM_EINVAL;
    delete s;
    return SP3MM_OK;
}

}  // extern "C"
