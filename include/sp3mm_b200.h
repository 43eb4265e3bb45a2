/*
 * sp3mm_b200.h -- C ABI of libsp3mm_b200.so, a B200 (sm_100a) implementation
 * of the Sp3MM4AMG Galerkin triple product C = R*AC*P on ordered CSR.
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the reference's names, signatures, structs,
 *     ownership and error behaviour (andreadiiorio/Sp3MM4AMG; paths below are
 *     relative to that project).  Inputs are host `spmat`s (64-bit IRP/JA,
 *     FP64 AS), borrowed and not modified; the result is a fresh host `spmat`
 *     whose AS/JA/IRP come from malloc/calloc so the caller's freeSpmat()
 *     releases it.  Errors return NULL after a message on stderr.  The `_1`
 *     variants take and return 1-based (FORTRAN) IRP/JA.
 *
 *  2. A device-resident layer (sp3mm_*): a context (device + CUDA stream),
 *     CSR matrices resident in HBM with 32-bit indices, and products that
 *     keep their operands and results on the device.  Functions return 0 on
 *     success or a SP3MM_E* code.
 *
 * Every product of layer 1 and 2 runs on the GPU; there is no CPU fallback.
 *
 * Result semantics (both layers): row pointers and column indices equal the
 * reference's; every value is accumulated in the reference's order with
 * separately rounded FP64 multiplies and adds, so values are bit-identical to
 * the reference's pair-wise functions (pair variants) and to
 * sp3mmRowByRowMerged_ (direct variants).
 *
 * Limits: M, N < 2^31 and every matrix (inputs, intermediate, result) has
 * fewer than 2^31 nonzeros; each input row's column indices must be strictly
 * ascending (ordered CSR).  Violations return NULL / SP3MM_EINVAL.
 */
#ifndef SP3MM_B200_H
#define SP3MM_B200_H

#include <stdint.h>
#include <stddef.h>

#if defined(__GNUC__)
#define SP3MM_API __attribute__((visibility("default")))
#else
#define SP3MM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference ABI types (same layout; skipped when the reference's own
 * headers were included first) ------------------------------------------ */
#ifndef CONFIG_H
/* code/src/include/config.h:51 */
typedef unsigned long idx_t;
/* code/src/include/config.h:34-37 */
typedef enum { RBTREE, IDXMAP } ROW_MMSYM_IMPL_MODE;
/* code/src/include/config.h:42-49.  gridRows/gridCols/threadNum are accepted
 * and ignored (the GPU partitions by row bins); chunkDistrbFunc, when not
 * NULL, is called once per SpMM with (rows, matrix, cfg) as the reference
 * does (code/src/Sp3MM_CSR_OMP_UB_Generic.c:83). */
typedef struct {
    unsigned short gridRows;
    unsigned short gridCols;
    ROW_MMSYM_IMPL_MODE symbMMRowImplID;
    unsigned int threadNum;
    void *chunkDistrbFunc;
} CONFIG;
#endif

#ifndef SPARSEMATRIX
/* code/src/include/sparseMatrix.h:41-53 (ROWLENS off). */
typedef struct {
    idx_t NZ, M, N;
    double *AS;
    idx_t *JA;
    idx_t *IRP;
    idx_t MAX_ROW_NZ;
} spmat;
#endif

#ifndef SP3MM_CSR_OMP_MULTI_H
/* code/src/include/Sp3MM_CSR_OMP_Multi.h:50-53 */
typedef spmat *(SPMM)(spmat *, spmat *, CONFIG *);
typedef spmat *(*SPMM_INTERF)(spmat *, spmat *, CONFIG *);
typedef spmat *(SP3MM)(spmat *, spmat *, spmat *, CONFIG *, SPMM_INTERF);
typedef spmat *(*SP3MM_INTERF)(spmat *, spmat *, spmat *, CONFIG *, SPMM_INTERF);
#endif

/* Timing globals of code/src/Sp3MM_CSR_OMP_Multi.c:54.  ElapsedInternal is
 * set to the device time (seconds) of the last product's compute, without
 * host<->device copies; Start/End bracket it in omp_get_wtime-like seconds. */
SP3MM_API extern double Start, End, Elapsed, ElapsedInternal;

/* ---- layer 1: drop-in entry points ------------------------------------- */

/* Triple product as a pair of SpMMs, (R*AC)*P.
 * Replaces code/src/Sp3MM_CSR_OMP_UB_Generic.c:456-494.  spmm == NULL selects
 * spmmRowByRow2DBlocks_ as the reference does (:462-465).  When spmm is one
 * of this library's SpMM entry points the intermediate stays on the device;
 * any other function pointer is called twice on host matrices, as the
 * reference does. */
SP3MM_API SP3MM sp3mmRowByRowPair_0, sp3mmRowByRowPair_1;
/* Direct row-forwarding triple product, upper-bound flavour.  Each R*AC row
 * is forwarded into P in first-touch order.  spmm is ignored.
 * Replaces code/src/Sp3MM_CSR_OMP_UB_Generic.c:498-573. */
SP3MM_API SP3MM sp3mmRowByRowMerged_0, sp3mmRowByRowMerged_1;
/* Pair-wise triple product with the symbolic-numeric SpMM; spmm == NULL
 * selects spmmRowByRow_SymbNum_.  Declared but never defined by the
 * reference (code/src/include/Sp3MM_CSR_OMP_Num_Generic.h:44). */
SP3MM_API SP3MM sp3mmRowByRowPair_SymbNum_0, sp3mmRowByRowPair_SymbNum_1;
/* Direct triple product, symbolic-numeric flavour: an exact symbolic pass
 * sizes C, then the numeric pass writes it in place.  Same values as
 * sp3mmRowByRowMerged_.  Declared, never defined, by the reference
 * (code/src/include/Sp3MM_CSR_OMP_Num_Generic.h:51). */
SP3MM_API SP3MM sp3mmRowByRowMerged_SymbNum_0, sp3mmRowByRowMerged_SymbNum_1;
/* R*(AC*P): the right association, which the reference lacks.  spmm selects
 * the flavour as in sp3mmRowByRowPair_ (NULL: upper bound). */
SP3MM_API SP3MM sp3mmRowByRowPairRight_0, sp3mmRowByRowPairRight_1;

/* SpMM, upper-bound flavour: per-row upper bounds, accumulation, atomic
 * space booking and a compaction into exact CSR.  All five return the same
 * matrix; the reference's 1D/2D OpenMP partitionings have no GPU meaning.
 * Replace code/src/Sp3MM_CSR_OMP_UB_Generic.c:38-53 (spmmSerial_, broken in
 * the reference), :56-124, :126-201, :205-338, :340-454. */
SP3MM_API SPMM spmmSerial_0, spmmSerial_1;
SP3MM_API SPMM spmmRowByRow_0, spmmRowByRow_1;
SP3MM_API SPMM spmmRowByRow1DBlocks_0, spmmRowByRow1DBlocks_1;
SP3MM_API SPMM spmmRowByRow2DBlocks_0, spmmRowByRow2DBlocks_1;
SP3MM_API SPMM spmmRowByRow2DBlocksAllocated_0, spmmRowByRow2DBlocksAllocated_1;

/* SpMM, symbolic-numeric flavour: exact row sizes, a scan to IRP, then the
 * numeric pass writes sorted rows in place.
 * Replace code/src/Sp3MM_CSR_OMP_Num_Generic.c:93-146, :147-210 and the
 * 2D stub :211-239 (which always returns NULL in the reference). */
SP3MM_API SPMM spmmRowByRow_SymbNum_0, spmmRowByRow_SymbNum_1;
SP3MM_API SPMM spmmRowByRow1DBlocks_SymbNum_0, spmmRowByRow1DBlocks_SymbNum_1;
SP3MM_API SPMM spmmRowByRow2DBlocks_SymbNum_0, spmmRowByRow2DBlocks_SymbNum_1;
SP3MM_API SPMM spmmRowByRow2DBlocksAllocated_SymbNum_0, spmmRowByRow2DBlocksAllocated_SymbNum_1;

/* Exact row sizes of a*b: malloc'd idx_t[a->M + 1], the total at [a->M].
 * Both modes return the same counts.
 * Replaces code/src/Sp3MM_CSR_OMP_SymbStep_Generic.c:281-412 (SpMM_Symb_). */
SP3MM_API idx_t *SpMM_Symb___0(ROW_MMSYM_IMPL_MODE mode, spmat *a, spmat *b);
SP3MM_API idx_t *SpMM_Symb___1(ROW_MMSYM_IMPL_MODE mode, spmat *a, spmat *b);

/* Upper-bound row sizes of A*B (sum of the B row lengths selected by each A
 * row): malloc'd idx_t[A->M + 1], the total at [A->M].
 * Replaces code/src/include/SpMMUtilsGeneric.h:112-139. */
SP3MM_API idx_t *spMMSizeUpperbound_0(spmat *A, spmat *B);
SP3MM_API idx_t *spMMSizeUpperbound_1(spmat *A, spmat *B);

/* Upper-bound sizes per (row of A, column partition of B):
 * malloc'd idx_t[A->M*gridCols + 1], row-major, the total at the end.
 * bColPartOffsets is B's column-partition offset matrix
 * (code/src/commons/sparseUtilsGeneric.c:284-311).
 * Replaces code/src/include/SpMMUtilsGeneric.h:146-174. */
SP3MM_API idx_t *spMMSizeUpperboundColParts_0(spmat *A, spmat *B, unsigned short gridCols,
                                    idx_t *bColPartOffsets);
SP3MM_API idx_t *spMMSizeUpperboundColParts_1(spmat *A, spmat *B, unsigned short gridCols,
                                    idx_t *bColPartOffsets);

/* 2D column partitioning of a host CSR into gridCols uniform column ranges
 * (the first N % gridCols ranges one column wider).
 * colsOffsetsPartitioningUnifRanges_: malloc'd idx_t[A->M*gridCols + 1],
 * entry [r*gridCols + gc] the 0-based JA/AS position of row r's first entry
 * in range gc, NZ at the end (the input spMMSizeUpperboundColParts_ takes).
 * colsPartitioningUnifRanges_ / ...OffsetsAux_: a calloc'd array of gridCols
 * spmat, range gc as an A->M x width matrix with 0-based IRP and JA/AS
 * copies (column indices unchanged); free each one's IRP, JA and AS, then
 * the array, with free() (the reference's freeSpmatInternal + free).  The Aux form also returns the offsets through
 * *colPartsOffsets when that pointer is not NULL.  NULL plus a message on
 * stderr on error (including gridCols == 0); an empty range gets NULL JA/AS
 * where the reference fails the call.
 * Replace code/src/include/sparseUtilsGeneric.h:43-52
 * (code/src/commons/sparseUtilsGeneric.c:284-400). */
SP3MM_API idx_t *colsOffsetsPartitioningUnifRanges_0(spmat *A, unsigned int gridCols);
SP3MM_API idx_t *colsOffsetsPartitioningUnifRanges_1(spmat *A, unsigned int gridCols);
SP3MM_API spmat *colsPartitioningUnifRanges_0(spmat *A, unsigned int gridCols);
SP3MM_API spmat *colsPartitioningUnifRanges_1(spmat *A, unsigned int gridCols);
SP3MM_API spmat *colsPartitioningUnifRangesOffsetsAux_0(spmat *A, unsigned int gridCols,
                                                        idx_t **colPartsOffsets);
SP3MM_API spmat *colsPartitioningUnifRangesOffsetsAux_1(spmat *A, unsigned int gridCols,
                                                        idx_t **colPartsOffsets);

/* MatrixMarket coordinate file -> host CSR spmat, 0-based, the arrays from
 * malloc/calloc (freeSpmat releases them); NULL plus a message on stderr on
 * error.  Replaces code/src/lib/parser.c:126-330 (MMtoCSR over MMRead,
 * MMtoCOO, COOtoCSR): real / integer / pattern (value 1.0) fields;
 * "symmetric" files expanded with each off-diagonal item mirrored right
 * after it; every row keeps the file's entry order, so files written row by
 * row in ascending column order give the ordered CSR the products require
 * (sp3mm_spmat_sort_rows orders the others).  Errors where the reference's
 * behaviour is undefined: a count of items different from the size line's,
 * an index outside the declared shape, complex or array files. */
SP3MM_API spmat *MMtoCSR(char *matPath);
/* New, no counterpart in the reference: write a host CSR (index base off_f,
 * 0 or 1) as a "matrix coordinate real general" MatrixMarket file with
 * 1-based indices and values printed to round-trip exactly (%.17g).
 * Returns SP3MM_OK or SP3MM_EINVAL (invalid CSR or unwritable path). */
SP3MM_API int sp3mm_write_mm(const spmat *m, int off_f, const char *path);
/* New, no counterpart in the reference: sort every row of a host CSR (index
 * base off_f) by column index in place, keeping the order of equal columns.
 * Returns SP3MM_OK or SP3MM_EINVAL. */
SP3MM_API int sp3mm_spmat_sort_rows(spmat *m, int off_f);

/* Dispatch tables with the reference's names and orders
 * (code/src/include/Sp3MM_CSR_OMP_UB_Generic.h:86-95,
 *  code/src/include/Sp3MM_CSR_OMP_Num_Generic.h:86-95), so that the
 * reference's test driver relinks unchanged.  The SymbNum direct table gains
 * its (new) entry. */
#ifndef SP3MM_B200_NO_TABLES
static SPMM_INTERF Spmm_UB_Funcs_0[] = {
    &spmmRowByRow_0, &spmmRowByRow1DBlocks_0, &spmmRowByRow2DBlocks_0,
    &spmmRowByRow2DBlocksAllocated_0};
static SP3MM_INTERF Sp3mm_UB_Funcs_0[] = {&sp3mmRowByRowMerged_0};
static SPMM_INTERF Spmm_SymbNum_Funcs_0[] = {
    &spmmRowByRow_SymbNum_0, &spmmRowByRow1DBlocks_SymbNum_0};
static SP3MM_INTERF Sp3mm_SymbNum_Funcs_0[] = {&sp3mmRowByRowMerged_SymbNum_0};
static SPMM_INTERF Spmm_UB_Funcs_1[] = {
    &spmmRowByRow_1, &spmmRowByRow1DBlocks_1, &spmmRowByRow2DBlocks_1,
    &spmmRowByRow2DBlocksAllocated_1};
static SP3MM_INTERF Sp3mm_UB_Funcs_1[] = {&sp3mmRowByRowMerged_1};
static SPMM_INTERF Spmm_SymbNum_Funcs_1[] = {
    &spmmRowByRow_SymbNum_1, &spmmRowByRow1DBlocks_SymbNum_1};
static SP3MM_INTERF Sp3mm_SymbNum_Funcs_1[] = {&sp3mmRowByRowMerged_SymbNum_1};
#endif

/* ---- layer 2: device-resident products --------------------------------- */

enum {
    SP3MM_OK = 0,
    SP3MM_ECUDA = 1,     /* a CUDA call failed (message on stderr) */
    SP3MM_EINVAL = 2,    /* invalid argument or malformed CSR input */
    SP3MM_ENOMEM = 3,    /* device allocation failed or budget exceeded */
    SP3MM_ELIMIT = 4,    /* a size exceeds the 32-bit device index limits */
    SP3MM_EDEVICE = 5    /* a kernel reported an internal error flag */
};

/* Flavours and variants of a product. */
enum { SP3MM_UB = 0, SP3MM_SYMBNUM = 1 };
enum { SP3MM_PAIR = 0, SP3MM_DIRECT = 1, SP3MM_PAIR_RIGHT = 2 };
/* Value storage of a device matrix. */
enum { SP3MM_F64 = 0, SP3MM_F32 = 1 };

/* A CSR matrix resident in device memory: 0-based int32 row_ptr[M+1] and
 * col[nnz] (ascending within each row), values in FP64 or FP32.  Arrays are
 * owned by the library when created by it (free with sp3mm_dcsr_free). */
typedef struct {
    int32_t M, N;
    int64_t nnz;
    int32_t *row_ptr;
    int32_t *col;
    void *val;
    int32_t val_type;   /* SP3MM_F64 or SP3MM_F32 */
    int32_t max_row;    /* longest row, or -1 when unknown */
} sp3mm_dcsr;

typedef struct sp3mm_ctx sp3mm_ctx;

/* Context on `device` with its own non-blocking stream. */
SP3MM_API int sp3mm_ctx_create(int device, sp3mm_ctx **out);
SP3MM_API int sp3mm_ctx_destroy(sp3mm_ctx *ctx);
/* Run subsequent work on a caller-owned stream (cudaStream_t as void*);
 * NULL restores the context's own stream. */
SP3MM_API int sp3mm_ctx_set_stream(sp3mm_ctx *ctx, void *stream);
SP3MM_API void *sp3mm_ctx_stream(sp3mm_ctx *ctx);
/* Bytes of device memory the context may hold for workspace (0: no limit). */
SP3MM_API int sp3mm_ctx_set_workspace_limit(sp3mm_ctx *ctx, size_t bytes);
/* Release cached workspace: the device memory pool's idle memory, this
 * context's page-locked staging and the process-wide cache of staging
 * buffers that destroyed contexts gave back. */
SP3MM_API int sp3mm_ctx_trim(sp3mm_ctx *ctx);
/* Last error message of this context (static storage of the context). */
SP3MM_API const char *sp3mm_ctx_last_error(sp3mm_ctx *ctx);
/* Kernel launches issued by this context since creation. */
SP3MM_API uint64_t sp3mm_ctx_launches(sp3mm_ctx *ctx);
/* Block until the context's stream is idle. */
SP3MM_API int sp3mm_ctx_sync(sp3mm_ctx *ctx);
/* Row-kernel tuning (results never depend on it): lanes per output row
 * (4, 8, 16, 32; 512: a CTA of 16 warps per row of a direct product, with
 * dense shared-memory accumulators; 0 = default: a warp per row, and the
 * CTA per row for direct rows with thousands of distinct columns); d1: the
 * first hash table of a row is sized for its distinct-key bound >> d1; d2:
 * the direct product's second table is the first >> d2 (d1, d2 < 0:
 * defaults).  Rows whose tables overflow are recomputed with proven-size
 * tables. */
SP3MM_API int sp3mm_ctx_set_tuning(sp3mm_ctx *ctx, int lanes_per_row, int d1, int d2);
/* Time every kernel launch with CUDA events on the context stream (on != 0);
 * switching clears the records. */
SP3MM_API int sp3mm_ctx_set_profiling(sp3mm_ctx *ctx, int on);
/* Per-kernel totals since profiling was switched on, one line per kernel
 * family: "<label> <launches> <total_ms> <max_ms>\n". */
SP3MM_API int sp3mm_ctx_profile_report(sp3mm_ctx *ctx, char *buf, size_t len);

/* Upload a host spmat (0- or 1-based per off_f), validating it, narrowing
 * the indices to int32 and storing values as val_type. */
SP3MM_API int sp3mm_dcsr_upload(sp3mm_ctx *ctx, const spmat *host, int off_f, int val_type,
                      sp3mm_dcsr *out);
/* Upload from plain host arrays (int64 row pointers and columns, FP64 values). */
SP3MM_API int sp3mm_dcsr_upload_arrays(sp3mm_ctx *ctx, int64_t M, int64_t N, int64_t nnz,
                             const int64_t *row_ptr, const int64_t *col,
                             const double *val, int val_type, sp3mm_dcsr *out);
/* Copy to a fresh host spmat (malloc'd arrays, indices shifted by off_f). */
SP3MM_API int sp3mm_dcsr_download(sp3mm_ctx *ctx, const sp3mm_dcsr *m, int off_f, spmat **out);
/* Copy into caller arrays (int64 row_ptr[M+1], int64 col[nnz], FP64 val[nnz]). */
SP3MM_API int sp3mm_dcsr_download_arrays(sp3mm_ctx *ctx, const sp3mm_dcsr *m, int64_t *row_ptr,
                               int64_t *col, double *val);
SP3MM_API int sp3mm_dcsr_free(sp3mm_ctx *ctx, sp3mm_dcsr *m);
/* Overwrite the values of m (same pattern) from host FP64 val[nnz],
 * converted to m's value type; returns once the copy is complete. */
SP3MM_API int sp3mm_dcsr_set_values(sp3mm_ctx *ctx, sp3mm_dcsr *m, const double *val);

/* C = A*B on the device, flavour SP3MM_UB or SP3MM_SYMBNUM; C's values are
 * stored as out_val_type.  C is allocated by the library. */
SP3MM_API int sp3mm_spmm(sp3mm_ctx *ctx, const sp3mm_dcsr *A, const sp3mm_dcsr *B, int flavour,
               int out_val_type, sp3mm_dcsr *C);
/* C = R*A*P on the device: variant SP3MM_PAIR, SP3MM_DIRECT or
 * SP3MM_PAIR_RIGHT; flavour SP3MM_UB or SP3MM_SYMBNUM. */
SP3MM_API int sp3mm_rap(sp3mm_ctx *ctx, const sp3mm_dcsr *R, const sp3mm_dcsr *A,
              const sp3mm_dcsr *P, int variant, int flavour, int out_val_type,
              sp3mm_dcsr *C);
/* Exact row sizes / upper bounds of A*B into device int32 rows[M] (any of
 * the pointers may be NULL); returns the totals through *total. */
SP3MM_API int sp3mm_spmm_rowsizes(sp3mm_ctx *ctx, const sp3mm_dcsr *A, const sp3mm_dcsr *B,
                        int exact, int32_t *rows_dev, int64_t *total);
/* Device transpose (R = P^T), values kept in their storage type. */
SP3MM_API int sp3mm_transpose(sp3mm_ctx *ctx, const sp3mm_dcsr *A, sp3mm_dcsr *AT);
/* C = R*A*P, direct variant, symbolic-numeric flavour, allocating nothing.
 * No counterpart in the reference: it serves callers that cannot let a
 * library allocate device memory while they run (their device memory is
 * owned by another allocator, or the call sits in a latency-critical loop).
 * Inputs are FP64 device CSRs; the caller passes C's arrays: c_row_ptr
 * (R->M + 1 entries), c_col / c_val (c_capacity entries).  *c_nnz receives
 * C's nonzero count; when it exceeds c_capacity the call returns
 * SP3MM_ENOMEM having written only c_row_ptr (call again with larger
 * arrays).  Temporaries live in a fixed 64 MiB device array inside the
 * library (held on every device that uses it until the process exits), which
 * bounds R->M to about 3.19 million rows (SP3MM_ELIMIT beyond, with the
 * exact limit in the message) and requires every row's hash tables to fit
 * in shared memory; C's nonzero count must stay below 2^31.  Operands whose
 * max_row is -1 are measured on the device.  The first call on a
 * device looks up that array's address; make it before any stream capture.
 * Calls whose GPU work overlaps share the array and race: serialise them.
 * `stream` is a cudaStream_t (NULL: the legacy default stream). */
SP3MM_API int sp3mm_rap_direct_noalloc(const sp3mm_dcsr *R, const sp3mm_dcsr *A,
                                       const sp3mm_dcsr *P, int32_t *c_row_ptr, int32_t *c_col,
                                       double *c_val, int64_t c_capacity, int64_t *c_nnz,
                                       void *stream);
/* Upper bound of the device bytes a sp3mm_rap call may allocate. */
SP3MM_API int sp3mm_rap_memory_estimate(const sp3mm_dcsr *R, const sp3mm_dcsr *A,
                              const sp3mm_dcsr *P, int variant, int flavour,
                              size_t *bytes);

/* ---- Batches: many independent products in one pass --------------------
 * Product i is C_i = X_i*Y_i (SP3MM_BATCH_SPMM, the symbolic-numeric SpMM)
 * or C_i = X_i*Y_i*Z_i (SP3MM_BATCH_RAP, the direct row-forwarding triple
 * product); results equal the single-product calls bit for bit.  All
 * operands share one value type; results are stored as out_val_type.
 * The operands are borrowed: they must stay allocated, with unchanged
 * patterns, while the batch is used.
 *
 * sp3mm_batch_plan sizes every product at once (a few host round trips
 * per batch) and allocates the results.  sp3mm_batch_execute replays the
 * numeric pass, captured as a CUDA graph, on the context stream without
 * host synchronisation; it may be repeated after the operands' values
 * change.  sp3mm_batch_run = plan (when needed; values computed) or
 * execute, then an error check.  Results are views owned by the batch. */
enum { SP3MM_BATCH_SPMM = 0, SP3MM_BATCH_RAP = 1 };
typedef struct sp3mm_batch sp3mm_batch;
SP3MM_API int sp3mm_batch_create(sp3mm_ctx *ctx, int n, const int *kinds, const sp3mm_dcsr *X,
                                 const sp3mm_dcsr *Y, const sp3mm_dcsr *Z, int out_val_type,
                                 sp3mm_batch **out);
/* Symbolic table shifts d1, d2 (first table from its bound >> d1; second
 * from its bound >> d2), numeric table slack (2^slack times the exact
 * size), and the table levels at which a new numeric tier (one persistent
 * launch) starts: nsplits < 0 for one tier per level, 0 for a single tier. */
SP3MM_API int sp3mm_batch_set_tuning(sp3mm_batch *b, int d1, int d2, int slack, int nsplits,
                                     const int32_t *splits);
/* SP3MM_UB (default): the plan runs one numeric pass in which every row
 * books its exact length from one cursor, then compacts (the plan computes
 * the values; the replay graph is built at the first execute).
 * SP3MM_SYMBNUM: the plan runs a symbolic pass and builds the graph; values
 * come from execute.  Both give the same results. */
SP3MM_API int sp3mm_batch_set_flavour(sp3mm_batch *b, int flavour);
SP3MM_API int sp3mm_batch_plan(sp3mm_batch *b);
SP3MM_API int sp3mm_batch_execute(sp3mm_batch *b);
SP3MM_API int sp3mm_batch_run(sp3mm_batch *b);
/* Times `reps` replays of each candidate tiering and slack, keeps the
 * fastest; one line per candidate is written to report (may be NULL). */
SP3MM_API int sp3mm_batch_autotune(sp3mm_batch *b, int reps, char *report, size_t len);
SP3MM_API int sp3mm_batch_result(const sp3mm_batch *b, int i, sp3mm_dcsr *C);
/* Rows and nonzeros of the batch, numeric tiers (of which in global
 * memory), and rows the last plan redid with proven table sizes. */
SP3MM_API int sp3mm_batch_info(const sp3mm_batch *b, int64_t *rows, int64_t *nnz, int *tiers,
                               int *global_tiers, int64_t *retried);
SP3MM_API int sp3mm_batch_free(sp3mm_batch *b);

/* ---- Smoothed-aggregation setup around the product --------------------
 * The level-by-level chain that produces the reference's test operators
 * (code/scripts/getLevels3MMmatrixes.py:29-38) applied on the
 * device.  A is a square operator on a box grid of ndim (1..3) dimensions
 * dims[] with lexicographic numbering (x fastest) and a non-zero diagonal.
 *
 * sp3mm_block_prolongator: P = (I - omega D^-1 A) P0, P0 the aggregation of
 * non-overlapping block^ndim grid blocks (partial blocks at the high edges),
 * on the pattern of A*P0, values stored as out_val_type.  A row without a
 * diagonal entry returns SP3MM_EINVAL. */
SP3MM_API int sp3mm_block_prolongator(sp3mm_ctx *ctx, const sp3mm_dcsr *A, const int32_t *dims,
                                      int ndim, int block, double omega, int out_val_type,
                                      sp3mm_dcsr *P);

/* A device-resident hierarchy A_0 (the caller's, borrowed) .. A_{L-1} with
 * P_l = sp3mm_block_prolongator(A_l), R_l = P_l^T and
 * A_{l+1} = R_l A_l P_l by sp3mm_rap(variant, flavour).  Coarsening stops
 * at max_levels levels or once A_l has fewer than min_coarse rows.
 * coarse_val_type SP3MM_F32 keeps level 0 in A_0's type and stores every
 * coarse operator and coarse prolongator in FP32 (FP64 accumulation). */
typedef struct sp3mm_hierarchy sp3mm_hierarchy;
SP3MM_API int sp3mm_hierarchy_build(sp3mm_ctx *ctx, const sp3mm_dcsr *A0, const int32_t *dims,
                                    int ndim, int block, double omega, int64_t min_coarse,
                                    int max_levels, int variant, int flavour,
                                    int coarse_val_type, sp3mm_hierarchy **out);
SP3MM_API int sp3mm_hierarchy_levels(const sp3mm_hierarchy *h);
/* Views of level `level`'s operator and (for all but the last level) its
 * prolongator and restriction; owned by the hierarchy. */
SP3MM_API int sp3mm_hierarchy_get(const sp3mm_hierarchy *h, int level, sp3mm_dcsr *A,
                                  sp3mm_dcsr *P, sp3mm_dcsr *R);
SP3MM_API int sp3mm_hierarchy_free(sp3mm_ctx *ctx, sp3mm_hierarchy *h);
/* n hierarchies built level-synchronously: each step forms the next level
 * of every unfinished hierarchy with batched launches (one SpMM batch for
 * the A*P0 products, one batch of direct triple products), so results equal
 * n calls of sp3mm_hierarchy_build with variant SP3MM_DIRECT.  dims holds
 * 3 entries per hierarchy (the first ndims[i] are used). */
SP3MM_API int sp3mm_hierarchy_build_batch(sp3mm_ctx *ctx, int n, const sp3mm_dcsr *A0,
                                          const int32_t *dims, const int32_t *ndims, int block,
                                          double omega, int64_t min_coarse, int max_levels,
                                          int coarse_val_type, sp3mm_hierarchy **out);

/* ---- Request server: continuous batching of hierarchy setups ------------
 * Each request is a host CSR operator A0 (0-based int64 row_ptr/col, FP64
 * values; borrowed until the request is done or has failed) on a box grid
 * (sp3mm_server_submit: smoothed block aggregation), or A0 with the
 * caller's prolongators (sp3mm_server_submit_ops).
 * Every sp3mm_server_step admits queued requests first come first served
 * while fewer than max_active are in flight and the request's device-memory
 * estimate fits both the budget (mem_fraction of the HBM free at creation,
 * less what admitted requests reserve) and the HBM free now, and hands them
 * to the server's two loader threads, which upload them on their own
 * contexts and streams while the step computes; then advances every uploaded hierarchy by one level
 * with batched launches shared by all of them (results equal the single
 * build's); then retires complete ones.  A request is reported active from
 * admission on.
 * Times are seconds on the server's clock (sp3mm_server_now); a request's
 * latency runs from its arrival (given, or its submission) to the end of
 * the step that completed it.  Status: 0 queued, 1 active, 2 done,
 * 3 failed (poll returns the error), 4 taken. */
typedef struct sp3mm_server sp3mm_server;
SP3MM_API int sp3mm_server_create(sp3mm_ctx *ctx, int max_active, double mem_fraction,
                                  sp3mm_server **out);
SP3MM_API double sp3mm_server_now(const sp3mm_server *s);
SP3MM_API int sp3mm_server_submit(sp3mm_server *s, int64_t M, int64_t nnz,
                                  const int64_t *row_ptr, const int64_t *col, const double *val,
                                  const int32_t *dims, int ndim, int block, double omega,
                                  int64_t min_coarse, int max_levels, int coarse_val_type,
                                  double arrival, int64_t *id);
/* Submit a request whose prolongators the caller provides (the setup
 * requests of an AMG caller such as AMG4PSBLAS, which aggregates by its own
 * rules): host CSRs A0 (M x M) and P_0 .. P_{np-1}, P_l of p_rows[l] x
 * p_cols[l] with p_rows[0] = M and p_rows[l] = p_cols[l-1] (0-based int64
 * indices, FP64 values, ascending columns; borrowed until the request is
 * done or has failed).  The server forms R_l = P_l^T and A_{l+1} =
 * R_l A_l P_l (direct product) on the device, level by level, batched with
 * the other requests in flight; coarse levels (l >= 1, their P included)
 * are stored as coarse_val_type.  The hierarchy's levels and results are
 * read as for the other requests; its grid sizes are the row counts. */
SP3MM_API int sp3mm_server_submit_ops(sp3mm_server *s, int64_t M, int64_t nnz,
                                      const int64_t *row_ptr, const int64_t *col,
                                      const double *val, int np, const int64_t *p_rows,
                                      const int64_t *p_cols, const int64_t *p_nnz,
                                      const int64_t *const *p_row_ptr,
                                      const int64_t *const *p_col, const double *const *p_val,
                                      int coarse_val_type, double arrival, int64_t *id);
SP3MM_API int sp3mm_server_step(sp3mm_server *s, int *pending);
SP3MM_API int sp3mm_server_poll(const sp3mm_server *s, int64_t id, int *status,
                                double *latency, double *queued);
/* Hand a done request's hierarchy (with its uploaded A0) to the caller,
 * who frees it with sp3mm_hierarchy_free. */
SP3MM_API int sp3mm_server_take(sp3mm_server *s, int64_t id, sp3mm_hierarchy **h);
SP3MM_API int sp3mm_server_stats(const sp3mm_server *s, int64_t *completed, int64_t *products,
                                 double *p50, double *p99, double *busy_s, int64_t *steps,
                                 int *peak_active, int64_t *deferred);
SP3MM_API int sp3mm_server_free(sp3mm_server *s);

#ifdef __cplusplus
}
#endif
#endif /* SP3MM_B200_H */
