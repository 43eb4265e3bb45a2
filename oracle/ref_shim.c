/*
 * ref_shim.c -- TEST INFRASTRUCTURE ONLY (oracle/_ref build).
 *
 * Linked beside the reference's own, unmodified sources (compiled in place
 * from the reference tree by oracle/Makefile) to make a shared library that
 * ctypes can drive.  The reference keeps a few helpers as C99 `inline`
 * functions in its headers; C99 only emits an external definition for such
 * a function in a translation unit that also declares it without `inline`.
 * The reference's own test driver does the same for its binary
 * (code/test/Sp3MM_test.c:48-77).  This file declares the handful that a
 * caller of the Sp3MM entry points needs, and adds a no-op chunk-division
 * callback for CONFIG.chunkDistrbFunc (code/src/include/config.h:42-49),
 * which every reference SpMM calls unconditionally
 * (code/src/Sp3MM_CSR_OMP_UB_Generic.c:83).
 */
#include <omp.h>
#include "Sp3MM_CSR_OMP_Multi.h"
#include "sparseUtilsMulti.h"
#include "ompChunksDivide.h"

/* External definitions of the header-inline helpers. */
spmat *allocSpMatrix(idx_t rows, idx_t cols);
int allocSpMatrixInternal(idx_t rows, idx_t cols, spmat *mat);
void freeSpmatInternal(spmat *mat);
void freeSpmat(spmat *mat);
void C_FortranShiftIdxs(spmat *m);
void Fortran_C_ShiftIdxs(spmat *m);
void chunksNOOP(ulong r, spmat *mat, CONFIG *cfg);
void chunksFairFolded(ulong r, spmat *mat, CONFIG *cfg);

/* Addresses for ctypes, which cannot take the address of an inline. */
void *refshim_chunks_noop(void) { return (void *)&chunksNOOP; }
void *refshim_chunks_fair_folded(void) { return (void *)&chunksFairFolded; }

/* omp_sched_t kind of the runtime schedule, as the test driver reads it
 * (code/test/Sp3MM_test.c:296-308). */
int refshim_runtime_sched_kind(void) {
    omp_sched_t kind; int chunk;
    omp_get_schedule(&kind, &chunk);
    return (int)kind;
}
void refshim_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int refshim_max_threads(void) { return omp_get_max_threads(); }

/* Reads the reference's timing global written by the Sp3MM drivers. */
extern double ElapsedInternal;
double refshim_elapsed_internal(void) { return ElapsedInternal; }
