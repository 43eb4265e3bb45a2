// kernels.cuh -- host-side launchers of the Sp3MM device kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace sp3mm {

// Internal read-only view of a device CSR.
struct CsrView {
    int M, N;
    long long nnz;
    const int* rp;
    const int* ci;
    const void* v;
    int vtype;   // SP3MM_F64 / SP3MM_F32
};

// Row-kernel modes.
enum Mode : int { kSymb = 0, kNumExact = 1, kNumBook = 2 };

// Table-size levels: level L uses 32 << L slots.
constexpr int kMinLogSlots = 5;
constexpr int kLevels = 24;

struct DirectRowArgs {
    CsrView R, A, P;   // C = R*A*P, one output row per row of R
};
struct PairRowArgs {
    CsrView A, B;      // C = A*B, one output row per row of A
};

// Per-launch parameters shared by both row-kernel families.
struct RowParams {
    const int* rows;          // the rows of this launch
    int nrows;
    const int* nrows_dev;     // CTA-per-row kernel: row count on the device (set: nrows bounds it)
    int S1, S2;               // table slots (powers of two >= 32); S2: direct only
    unsigned char* gtab;      // tables in global memory (nullptr: shared memory)
    long long gstride;        // bytes per group in gtab
    int* retry_rows;          // rows whose table overflowed (nullptr: error)
    int* retry_count;
    int* row_cnt;             // kSymb: C row length; kNumBook: booked length
    int* row_cnt1;            // kSymb, direct: R*A row length (may be null)
    const int* c_rp;          // kNumExact: output row pointers
    int* c_ci;
    void* c_v;
    int c_vt;
    unsigned long long* cursor;   // kNumBook: booking cursor
    unsigned long long cap;       //           and capacity (entries)
    long long* row_off;           //           offset of each row
    int* ub_ci;
    void* ub_v;
    unsigned* err;
    // Some row of the first (a_long, direct only) / last (b_long) right
    // operand is longer than the entries the kernel prefetches per step.
    bool a_long, b_long;
    // Layout of the register-product direct kernel's batches (rowlanes.cuh)
    // in stage 1 (R*A, A rows) and stage 2 (RA*P, P rows): lanes per
    // left-row step (log2, at most 5, every right row at most that long), or
    // -1 for packed batches (any row length).
    int lg1, lg2;
};

// Launch geometry of one row-kernel launch.
struct RowGeom {
    int G;        // lanes per row
    int grid, block;
    size_t smem;  // dynamic shared memory per CTA
};

// Table bytes of one row (G lanes; G == 32: the warp kernels, incl. staging).
size_t row_table_bytes(bool direct, int mode, int G, int S1, int S2);
int row_table_limit(int S, int G);
// Right-row entries a G-lane group prefetches per step (0: none).
int row_prefetch_cover(int G);
cudaError_t launch_direct_rows(const DirectRowArgs& a, const RowParams& p, int mode,
                               const RowGeom& geo, cudaStream_t st);
// Direct rows with the products formed in registers (rowlanes.cuh):
// shared-memory tables, batch layouts p.lg1 / p.lg2.  lanes_row_bytes:
// table bytes per warp.
cudaError_t launch_direct_lanes(const DirectRowArgs& a, const RowParams& p, int mode,
                                const RowGeom& geo, cudaStream_t st);
size_t lanes_row_bytes(int mode, int S1, int S2);
// Tuning value of "lanes per row" that runs every direct row on the
// CTA-per-row kernel.
constexpr int kDenseLanes = 512;
// Direct rows with heavy work, one CTA per row (rowdense.cuh); rows that do
// not fit its shared-memory slice go to the retry list.  dense_row_smem():
// its dynamic shared memory per CTA.
cudaError_t launch_direct_dense(const DirectRowArgs& a, const RowParams& p, int mode, int grid,
                                cudaStream_t st);
size_t dense_row_smem();
// The same kernel in half the shared memory, two CTAs per SM
// (rows_dense_small.cu), for products whose A has at least
// kDenseSmallMinCols columns (coarse rows then reach a small fraction of
// them: 1,227 of 32,768 at 128^3 level 2); rows whose R*A row outgrows its
// 2,048-column list are run again by the default configuration.
// dense_small_ctas_per_sm(): its resident CTAs per SM (0 when it cannot
// run).
constexpr int kDenseSmallMinCols = 16384;
cudaError_t launch_direct_dense_small(const DirectRowArgs& a, const RowParams& p, int mode,
                                      int grid, cudaStream_t st);
int dense_small_ctas_per_sm();
cudaError_t launch_pair_rows(const PairRowArgs& a, const RowParams& p, int mode,
                             const RowGeom& geo, cudaStream_t st);

// Bounds: need[i] = distinct-key bound of the first table (A*B: min(flops,
// N); R*A*P: min(len of the R*A products, A.N)); total += the multiply-add
// bound of the output (A*B: flops; R*A*P: R*A flops times P's longest row).
void launch_pair_bounds(const CsrView& A, const CsrView& B, int* need,
                        unsigned long long* total, cudaStream_t st);
// need_opt (optional): optimistic first-table size per row, min(need >> d1,
// 8 sqrt(R*A products)).
void launch_direct_bounds(const CsrView& R, const CsrView& A, int p_max_row, int* need,
                          unsigned long long* total, cudaStream_t st, int* need_opt = nullptr,
                          int d1 = 0);
// *out = max(*out, largest cnt[i]) (cnt null: largest row length of rp) and,
// when `sum` is given, *sum += the 64-bit total of the row lengths (the
// caller zeroes both).
void launch_count_max(int M, const int* cnt, const int* rp, int* out, cudaStream_t st,
                      unsigned long long* sum = nullptr);
// need from exact counts: max(cnt[i], cnt1[i]) (cnt1 may be null).
void launch_need_from_counts(int M, const int* cnt, const int* cnt1, int* need,
                             cudaStream_t st);

// Binning: level of every row from need[i] >> shift -- or est[i] when est is
// given -- for a group of G lanes (counts[kLevels] = empty rows, whose
// row_cnt is zeroed when given); nmax = largest need.
void launch_bin_levels(int M, const int* need, int shift, int G, signed char* level,
                       int* counts, int* nmax, int* row_cnt_zero, cudaStream_t st,
                       const int* est = nullptr);
void launch_bin_scatter(int M, const signed char* level, int* cursors, int* lists,
                        cudaStream_t st);
// Smallest slot count (power of two >= 32) whose load limit for G lanes
// admits `need` distinct keys.
int slots_for_need(long long need, int G);
int level_for_need(long long need, int G);

// Upper-bound flavour: copy each booked row into exact CSR.
void launch_compact(int M, const int* row_cnt, const long long* row_off, const int* ub_ci,
                    const void* ub_v, const int* c_rp, int* c_ci, void* c_v, int vtype,
                    cudaStream_t st);

// row_ptr[0..M] = exclusive scan of cnt[0..M-1] (row_ptr[M] = total).
size_t scan_temp_bytes(int M);
void launch_scan(int M, const int* cnt, int* row_ptr, void* temp, size_t temp_bytes,
                 cudaStream_t st);

// Upload / download conversions.
void launch_narrow_rowptr(long long M, long long nnz, const unsigned long long* src, int off,
                          int* dst, unsigned* err, cudaStream_t st);
void launch_narrow_cols(long long M, long long N, const int* rp, const unsigned long long* src,
                        int off, int* dst, int* max_row, unsigned* err, cudaStream_t st);
void launch_widen(long long n, const int* src, int off, unsigned long long* dst,
                  cudaStream_t st);
void launch_convert_values(long long n, const void* src, int src_type, void* dst,
                           int dst_type, cudaStream_t st);
void launch_validate_i32(int M, int N, const int* rp, const int* ci, int* max_row,
                         unsigned* err, cudaStream_t st);

// Transpose (count, scan, scatter, per-row sort).
void launch_col_counts(long long nnz, const int* ci, int* counts, cudaStream_t st);
void launch_transpose_scatter(const CsrView& A, const int* t_rp, int* cursor, int* t_ci,
                              void* t_v, cudaStream_t st);
void launch_sort_rows(int M, const int* rp, int* ci, void* v, int vtype, int max_row,
                      cudaStream_t st);

// 2D column-partition upper bounds.
void launch_colparts_ub(const CsrView& A, int gridCols, const long long* bColOffsets,
                        long long* out, unsigned long long* total, cudaStream_t st);

void note_launch();
uint64_t launch_count();

}  // namespace sp3mm

struct sp3mm_ctx;
namespace sp3mm {
// Record `msg` as the context's last error (and print it); returns `code`.
int report_error(sp3mm_ctx* ctx, int code, const char* msg);

}  // namespace sp3mm
