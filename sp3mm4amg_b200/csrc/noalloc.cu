// noalloc.cu -- sp3mm_rap_direct_noalloc: the direct R*A*P product
// (symbolic + numeric) without any device allocation.
//
// Why it exists: some callers cannot let a library allocate device memory
// while they run -- code whose device memory is entirely owned by another
// allocator (a framework or solver that reserved the GPU's memory up front),
// and latency-critical loops that must not reach the CUDA allocator.  Such a
// caller passes the inputs and preallocated output arrays; every temporary
// this product needs (per-row bounds, bins, counts, scan storage, error word)
// lives in one fixed file-scope device array instead of memory from
// cudaMalloc or the stream-ordered pool.
//
// The array is `kScratchBytes` (64 MiB) per device, allocated when the
// library is loaded and kept until the process exits.  Host code finds its
// device address once per device with cudaGetSymbolAddress (the first call
// on a device does this set-up, so make that first call before any stream
// capture); device code of this file could name the array directly.  Every
// call shares the array and it keeps the last call's contents: each call
// clears what must start at zero.  Calls whose GPU work overlaps (two
// streams, two host threads) race on the array and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <mutex>

#include "kernels.cuh"
#include "sp3mm_b200.h"
#include "sp3mm_internal.cuh"

namespace sp3mm {
namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the scratch array and SM count per device (set-up once
// per device).
unsigned char* g_scratch_addr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};
std::mutex g_setup_mutex;

struct Head {
    int counts[kLevels + 1];
    int cursors[kLevels];
    int nmax;
    int retry_count;
    unsigned long long total;
    unsigned err;
    // Filled after the binning passes (run_direct clears the fields above):
    // longest rows of A and P when the operands do not record them, and
    // the longest C row with the 64-bit total of C's row counts.
    int a_max, p_max, c_max;
    unsigned long long c_total;
};

int fail(int code, const char* msg) {
    fprintf(stderr, "sp3mm_rap_direct_noalloc: %s\n", msg);
    return code;
}

// Map a device error word as sp3mm_rap does: malformed input is EINVAL.
int device_fail(unsigned err, const char* pass) {
    fprintf(stderr, "sp3mm_rap_direct_noalloc: device error flags 0x%x in the %s pass%s\n", err,
            pass, (err & kErrInput) ? " (malformed CSR input)" : "");
    return (err & kErrInput) ? SP3MM_EINVAL : SP3MM_EDEVICE;
}

#define NA_CK(call)                                                                     \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            fprintf(stderr, "sp3mm_rap_direct_noalloc: %s failed: %s\n", #call,         \
                    cudaGetErrorString(e_));                                            \
            return SP3MM_ECUDA;                                                         \
        }                                                                               \
    } while (0)

// The scratch array's device address on `dev` (the current device) and its
// SM count, looked up on the first call on that device.
unsigned char* scratch_for(int dev, int* sms) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (dev < 0 || dev >= kMaxDevices) {
        fprintf(stderr, "sp3mm_rap_direct_noalloc: device %d out of range\n", dev);
        return nullptr;
    }
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        int n = 0;
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) {
            fprintf(stderr, "sp3mm_rap_direct_noalloc: device set-up failed: %s\n",
                    cudaGetErrorString(e));
            return nullptr;
        }
        g_sms[dev] = n;
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *sms = g_sms[dev];
    return g_scratch_addr[dev];
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Bytes of the scratch layout for R with M rows (the offsets carve() uses).
size_t layout_bytes(int M) {
    const size_t rows = static_cast<size_t>(M) + 1;
    return align256(sizeof(Head)) + 5 * align256(4 * rows) + align256(rows) +
           align256(scan_temp_bytes(M));
}

// Largest row count of R whose layout fits the scratch array.
int max_rows_fitting() {
    int lo = 0, hi = INT_MAX - 1;
    while (lo < hi) {
        const int mid = lo + (hi - lo + 1) / 2;
        if (layout_bytes(mid) <= kScratchBytes) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Carve the per-row arrays out of the scratch array; returns the bytes used.
struct Layout {
    Head* head;
    int *need, *row_cnt, *row_cnt1, *retry, *lists;
    signed char* level;
    void* scan_tmp;
    size_t scan_bytes, total;
};

Layout carve(unsigned char* base, int M) {
    Layout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += align256(bytes);
        return p;
    };
    const size_t rows = static_cast<size_t>(M) + 1;
    L.head = reinterpret_cast<Head*>(take(sizeof(Head)));
    L.need = reinterpret_cast<int*>(take(4 * rows));
    L.row_cnt = reinterpret_cast<int*>(take(4 * rows));
    L.row_cnt1 = reinterpret_cast<int*>(take(4 * rows));
    L.retry = reinterpret_cast<int*>(take(4 * rows));
    L.lists = reinterpret_cast<int*>(take(4 * rows));
    L.level = reinterpret_cast<signed char*>(take(rows));
    L.scan_bytes = scan_temp_bytes(M);
    L.scan_tmp = take(L.scan_bytes);
    L.total = off;
    return L;
}

struct Geo {
    int sms;
    size_t smem_budget;
};

// Bin rows by need >> shift and run the direct row kernel over every level,
// tables in shared memory only.  Rows that overflow an optimistic table are
// rerun once with tables from the proven bounds (s1_max, s2_max).
int run_direct(const Layout& L, const DirectRowArgs& da, RowParams base, int mode, int G,
               int shift, int d2, long long s1_max_bound, long long s2_bound, double pmax,
               int a_max, int p_max, const Geo& geo, cudaStream_t st) {
    const int M = base.nrows;
    NA_CK(cudaMemsetAsync(L.head, 0, sizeof(Head), st));
    launch_bin_levels(M, L.need, shift, G, L.level, L.head->counts, &L.head->nmax,
                      mode == kSymb ? L.row_cnt : nullptr, st);
    Head h{};
    NA_CK(cudaMemcpyAsync(&h, L.head, sizeof h, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    int off = 0, offsets[kLevels];
    for (int l = 0; l < kLevels; ++l) {
        offsets[l] = off;
        h.cursors[l] = off;
        off += h.counts[l];
    }
    NA_CK(cudaMemcpyAsync(L.head->cursors, h.cursors, sizeof h.cursors, cudaMemcpyHostToDevice,
                          st));
    launch_bin_scatter(M, L.level, L.head->cursors, L.lists, st);

    auto launch = [&](RowParams p, int g) -> int {
        const size_t per_group = row_table_bytes(true, mode, g, p.S1, p.S2);
        const int gpw = 32 / g;
        int warps = static_cast<int>(geo.smem_budget / (per_group * gpw));
        if (warps > 8) warps = 8;
        if (warps < 1)
            return fail(SP3MM_ELIMIT,
                        "a row needs hash tables larger than shared memory; use sp3mm_rap");
        RowGeom rg{};
        rg.G = g;
        rg.block = 32 * warps;
        rg.smem = per_group * gpw * warps;
        const int gpc = gpw * warps;
        const long long grid = (p.nrows + gpc - 1) / gpc;
        rg.grid = static_cast<int>(std::min<long long>(grid, static_cast<long long>(geo.sms) * 16));
        const int cover = row_prefetch_cover(g);
        p.a_long = a_max < 0 || a_max > cover;
        p.b_long = p_max < 0 || p_max > cover;
        const cudaError_t e = launch_direct_rows(da, p, mode, rg, st);
        if (e != cudaSuccess) {
            fprintf(stderr, "sp3mm_rap_direct_noalloc: row kernel: %s\n", cudaGetErrorString(e));
            return SP3MM_ECUDA;
        }
        return SP3MM_OK;
    };
    NA_CK(cudaMemsetAsync(&L.head->retry_count, 0, sizeof(int), st));
    for (int l = 0; l < kLevels; ++l) {
        if (!h.counts[l]) continue;
        RowParams p = base;
        p.rows = L.lists + offsets[l];
        p.nrows = h.counts[l];
        p.S1 = 32 << l;
        p.S2 = std::max(32, p.S1 >> d2);
        p.retry_rows = L.retry;
        p.retry_count = &L.head->retry_count;
        const int rc = launch(p, G);
        if (rc) return rc;
    }
    int nretry = 0;
    NA_CK(cudaMemcpyAsync(&nretry, &L.head->retry_count, sizeof(int), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (nretry > 0) {
        RowParams p = base;
        p.rows = L.retry;
        p.nrows = nretry;
        const long long s1 = std::min<long long>(h.nmax, s1_max_bound);
        const long long s2 = std::min<long long>(
            static_cast<long long>(static_cast<double>(h.nmax) * pmax), s2_bound);
        p.S1 = slots_for_need(s1, 32);
        p.S2 = slots_for_need(s2, 32);
        if (p.S1 < p.S2) p.S1 = p.S2;
        p.retry_rows = nullptr;
        p.retry_count = nullptr;
        const int rc = launch(p, 32);
        if (rc) return rc;
    }
    return SP3MM_OK;
}

}  // namespace
}  // namespace sp3mm

using namespace sp3mm;

extern "C" SP3MM_API int sp3mm_rap_direct_noalloc(const sp3mm_dcsr* R, const sp3mm_dcsr* A,
                                                  const sp3mm_dcsr* P, int32_t* c_row_ptr,
                                                  int32_t* c_col, double* c_val,
                                                  int64_t c_capacity, int64_t* c_nnz,
                                                  void* stream) {
    if (!R || !A || !P || !c_row_ptr || !c_nnz || c_capacity < 0)
        return fail(SP3MM_EINVAL, "NULL argument or negative capacity");
    if (R->N != A->M || A->N != P->M)
        return fail(SP3MM_EINVAL, "inner dimensions differ");
    if (R->val_type != SP3MM_F64 || A->val_type != SP3MM_F64 || P->val_type != SP3MM_F64)
        return fail(SP3MM_EINVAL, "operands must hold FP64 values");
    if (c_capacity > 0 && (!c_col || !c_val))
        return fail(SP3MM_EINVAL, "NULL output arrays");
    const int M = R->M;
    int dev = 0, sms = 0;
    NA_CK(cudaGetDevice(&dev));
    unsigned char* base = scratch_for(dev, &sms);
    if (!base) return SP3MM_ECUDA;
    if (layout_bytes(M) > kScratchBytes) {
        char msg[200];
        snprintf(msg, sizeof msg, "R has %d rows; the %zu MiB scratch array holds at most %d",
                 M, kScratchBytes >> 20, max_rows_fitting());
        return fail(SP3MM_ELIMIT, msg);
    }
    const Layout L = carve(base, M);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Geo geo{sms, 110 * 1024};

    const CsrView vR{R->M, R->N, R->nnz, R->row_ptr, R->col, R->val, R->val_type};
    const CsrView vA{A->M, A->N, A->nnz, A->row_ptr, A->col, A->val, A->val_type};
    const CsrView vP{P->M, P->N, P->nnz, P->row_ptr, P->col, P->val, P->val_type};
    const DirectRowArgs da{vR, vA, vP};
    const double meanA = A->M ? static_cast<double>(A->nnz) / A->M : 1.0;
    const double meanP = P->M ? static_cast<double>(P->nnz) / P->M : 1.0;
    const double mean = std::max(meanA, meanP);
    const int G = mean <= 4 ? 4 : mean <= 8 ? 8 : mean <= 16 ? 16 : 32;

    // Start-of-call state: error word and counters cleared.
    NA_CK(cudaMemsetAsync(L.head, 0, sizeof(Head), st));
    // Longest rows the operands do not record are measured (the bounds and
    // the retry tables need P's; the kernels' prefetch needs both).
    int a_max = A->max_row, p_max = P->max_row;
    if (a_max < 0 || p_max < 0) {
        if (a_max < 0) launch_count_max(A->M, nullptr, A->row_ptr, &L.head->a_max, st);
        if (p_max < 0) launch_count_max(P->M, nullptr, P->row_ptr, &L.head->p_max, st);
        Head h{};
        NA_CK(cudaMemcpyAsync(&h, L.head, sizeof h, cudaMemcpyDeviceToHost, st));
        NA_CK(cudaStreamSynchronize(st));
        if (a_max < 0) a_max = h.a_max;
        if (p_max < 0) p_max = h.p_max;
    }
    const double pmax = p_max;
    launch_direct_bounds(vR, vA, p_max, L.need, &L.head->total, st);

    RowParams p{};
    p.nrows = M;
    p.row_cnt = L.row_cnt;
    p.row_cnt1 = L.row_cnt1;
    p.err = &L.head->err;
    p.c_vt = SP3MM_F64;
    NA_CK(cudaMemsetAsync(L.row_cnt1, 0, sizeof(int) * (static_cast<size_t>(M) + 1), st));
    int rc = run_direct(L, da, p, kSymb, G, 1, 1, A->N, P->N, pmax, a_max, p_max, geo, st);
    if (rc) return rc;
    // The 64-bit total of the row counts decides whether C fits int32
    // offsets before the 32-bit scan result is trusted.
    launch_count_max(M, L.row_cnt, nullptr, &L.head->c_max, st, &L.head->c_total);
    Head h{};
    NA_CK(cudaMemcpyAsync(&h, L.head, sizeof h, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (h.err) return device_fail(h.err, "symbolic");
    const long long nnz = static_cast<long long>(h.c_total);
    *c_nnz = nnz;
    if (nnz >= INT32_MAX) {
        fprintf(stderr, "sp3mm_rap_direct_noalloc: C has %lld nonzeros, beyond int32 offsets\n",
                nnz);
        return SP3MM_ELIMIT;
    }
    launch_scan(M, L.row_cnt, c_row_ptr, L.scan_tmp, L.scan_bytes, st);
    if (nnz > c_capacity) {
        // c_row_ptr is complete on return, so the caller can size C's arrays.
        NA_CK(cudaStreamSynchronize(st));
        fprintf(stderr,
                "sp3mm_rap_direct_noalloc: C has %lld nonzeros, the output arrays hold %lld\n",
                nnz, static_cast<long long>(c_capacity));
        return SP3MM_ENOMEM;
    }
    launch_need_from_counts(M, L.row_cnt, L.row_cnt1, L.need, st);
    p.row_cnt1 = nullptr;
    p.c_rp = c_row_ptr;
    p.c_ci = c_col;
    p.c_v = c_val;
    rc = run_direct(L, da, p, kNumExact, G, 0, 0, A->N, P->N, pmax, a_max, p_max, geo, st);
    if (rc) return rc;
    unsigned err = 0;
    NA_CK(cudaMemcpyAsync(&err, &L.head->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (err) return device_fail(err, "numeric");
    return SP3MM_OK;
}
