// batch.cuh -- descriptors and launchers of the batch row kernels.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

struct sp3mm_batch;

namespace sp3mm {

enum : int { kBatchPair = 0, kBatchDirect = 1 };

// One product of a batch: C = X*Y (pair) or C = X*Y*Z (direct).
struct BItem {
    CsrView X, Y, Z;
    int kind;
    int M, N;              // shape of C
    long long row_base;    // first global row
    int zmax;              // direct: longest row of Z (-1: unknown)
};

struct BatchRowParams {
    const int* rows;        // global rows of this launch
    const int* nrows_dev;   // when set, the row count is read from here
    int nrows;
    int scap;               // slots per table in each warp's region
    int d1, d2;             // symbolic: optimistic table shifts
    int slack;              // numeric: tables 2^slack times the exact size
    int reverse;            // walk the list from its end (largest rows first)
    const int* need;        // symbolic: first-table bound per global row
    const int* need_opt;    // symbolic: optimistic first-table size (null: need >> d1)
    int* cnt1;              // direct R*A distinct count (out: symbolic, in: numeric)
    int* cnt2;              // C row length (out: symbolic, in: numeric)
    const int* c_rp;        // numeric: global row pointers into c_ci / c_v
    int* c_ci;
    void* c_v;
    int* retry_rows;        // rows whose proven tables exceed scap
    int* retry_count;
    int* retry_need;        // largest proven table bound among them
    unsigned char* gtab;    // global-memory regions (GT), gstride bytes each
    long long gstride;
    unsigned* err;
    // Booking (upper-bound flavour): each finished row books its exact
    // length from `cursor` (capacity `cap` entries) and is written there.
    unsigned long long* cursor;
    unsigned long long cap;
    long long* row_off;
    int* ub_ci;
    void* ub_v;
};

// Sets the kernel's dynamic shared memory limit to `max_smem` and returns
// how many CTAs of `block` threads with `smem` bytes each fit one SM.
cudaError_t batch_rows_configure(int mode, bool gt, int tv, int to, int block, size_t smem,
                                 size_t max_smem, int* ctas_per_sm);
cudaError_t launch_batch_rows(int mode, bool gt, int tv, int to, int grid, int block,
                              size_t smem, cudaStream_t st, const BItem* items,
                              const int* row_item, const BatchRowParams& p);
size_t batch_row_region_bytes(bool num, int scap);
// Heavy direct rows of a batch, one CTA of 512 threads per row (symbolic or
// booked pass); batch_dense_smem(): its dynamic shared memory per CTA.
cudaError_t launch_batch_dense(int mode, int tv, int to, int grid, cudaStream_t st,
                               const BItem* items, const int* row_item, const BatchRowParams& p);
size_t batch_dense_smem();
// Release a planned, executed batch's planning state and graph; its
// results stay valid, execute is no longer possible.
void batch_trim(::sp3mm_batch* b);
int batch_slots_for(long long need);

}  // namespace sp3mm
