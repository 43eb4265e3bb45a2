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

// Table-size levels: level L holds slots = 32 << L.  Levels below
// kSharedLevels keep their tables in shared memory; the last level keeps
// them in global memory.
constexpr int kMinLogSlots = 5;
constexpr int kSharedLevels = 8;          // 32 .. 4096 slots
constexpr int kLevels = kSharedLevels + 1;
constexpr int kGlobalLevel = kSharedLevels;

// Slots a row needs for `bound` distinct keys (load factor <= 0.8).
inline unsigned slots_for(long long bound) {
    long long need = bound + bound / 4 + 1;
    unsigned s = 32;
    while ((long long)s < need && s < (1u << 30)) s <<= 1;
    return s;
}

// Bytes of table state per slot for a kernel family/mode.
inline int bytes_per_slot(bool direct, int mode) {
    if (direct) return mode == kSymb ? 12 : 28;
    return mode == kSymb ? 8 : 24;
}

// Shared-memory plan of one level: group size, groups per CTA, bytes.
struct LevelPlan {
    int G;
    int groups_per_cta;
    int slots;
    size_t smem_bytes;   // per CTA (0 for the global level)
    bool global;
};

// Per-launch row set of one level.
struct RowSet {
    const int* rows;
    int nrows;
    int slots;
    int shift;
    unsigned char* gtab;     // global tables (nullptr: shared memory)
    long long gtab_stride;   // bytes per group in gtab
};

struct PairArgs {
    CsrView A, B;            // C = A*B, rows of A processed
    int* row_cnt;            // kSymb: exact length; kNumBook: booked length
    const int* c_rp;         // kNumExact: output row pointers
    int* c_ci;
    void* c_v;
    int c_vtype;
    unsigned long long* book_cursor;
    unsigned long long book_cap;
    long long* row_off;      // kNumBook: offset of each row in the UB space
    int* ub_ci;
    void* ub_v;
    unsigned* err;
};

struct DirectArgs {
    CsrView R, A, P;         // C = R*A*P, rows of R processed
    int* row_cnt;            // kSymb: exact C row length; kNumBook: booked
    int* row_cnt1;           // kSymb: distinct R*A row length (may be null)
    const int* c_rp;
    int* c_ci;
    void* c_v;
    int c_vtype;
    unsigned long long* book_cursor;
    unsigned long long book_cap;
    long long* row_off;
    int* ub_ci;
    void* ub_v;
    unsigned* err;
};

// Choose the group size (lanes per row) from the right operand's mean row
// length, and derive the per-level launch plan.
int choose_group(double mean_right_row_len);
LevelPlan plan_level(int level, bool direct, int mode, int G, size_t smem_budget);

// Bounds: per-row table size requirement (`need`, distinct-key bound) and
// the total multiply-add count (upper bound of the output size).
void launch_pair_bounds(const CsrView& A, const CsrView& B, int* need,
                        unsigned long long* total_flops, cudaStream_t st);
void launch_direct_bounds(const CsrView& R, const CsrView& A, const CsrView& P, int* need,
                          unsigned long long* total_flops, cudaStream_t st);
// need from exact counts: max(cnt[i], cnt1[i]) (cnt1 may be null).
void launch_need_from_counts(int M, const int* cnt, const int* cnt1, int* need,
                             cudaStream_t st);

// Binning: level of every row from `need`; counts[kLevels+1] (the extra
// entry counts empty rows, whose row_cnt is zeroed); global_need_max.
void launch_bin_levels(int M, const int* need, signed char* level, int* counts,
                       int* global_need_max, int* row_cnt_zero, cudaStream_t st);
void launch_bin_scatter(int M, const signed char* level, int* cursors, int* lists,
                        cudaStream_t st);

// Row kernels.
void launch_pair_rows(const PairArgs& a, int mode, const LevelPlan& plan, const RowSet& rs,
                      int grid, cudaStream_t st);
void launch_direct_rows(const DirectArgs& a, int mode, const LevelPlan& plan,
                        const RowSet& rs, int grid, cudaStream_t st);
size_t row_kernel_max_smem();

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
void launch_colparts_ub(const CsrView& A, const CsrView& B, int gridCols,
                        const long long* bColOffsets, int off, long long* out,
                        unsigned long long* total, cudaStream_t st);

uint64_t launch_count();

}  // namespace sp3mm
