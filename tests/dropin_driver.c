/* dropin_driver.c -- a plain C11 consumer of include/sp3mm_b200.h, written
 * the way the reference's own test driver uses its library
 * (code/test/Sp3MM_test.c:318-419): load R, AC and P from MatrixMarket files,
 * walk every dispatch table -- the pair-wise SpMMs through
 * sp3mmRowByRowPair_, the direct triple products directly, the
 * symbolic-numeric ones under both symbolic modes -- and release every
 * result with free() as the reference's freeSpmat does.  Each result is
 * written to <out_dir>/<tag>.mtx for the calling test to compare.
 *
 * usage: dropin_driver r.mtx ac.mtx p.mtx out_dir off_f
 *   off_f = 1 hands the library 1-based IRP/JA, as a FORTRAN caller does
 *   (the _1 tables); 0 uses the _0 tables.
 * Exit status 0 when every call returned a matrix; the number of results is
 * printed on stdout. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sp3mm_b200.h"

#define COUNT(a) (sizeof(a) / sizeof((a)[0]))

static void free_spmat(spmat *m) {
    if (!m) return;
    free(m->AS);
    free(m->JA);
    free(m->IRP);
    free(m);
}

static void shift(spmat *m, idx_t by) {
    for (idx_t i = 0; i <= m->M; ++i) m->IRP[i] += by;
    for (idx_t i = 0; i < m->NZ; ++i) m->JA[i] += by;
}

static int emit(spmat *c, const char *dir, const char *tag, int off) {
    char path[4096];
    if (!c) {
        fprintf(stderr, "dropin_driver: %s returned NULL\n", tag);
        return 1;
    }
    snprintf(path, sizeof path, "%s/%s.mtx", dir, tag);
    const int rc = sp3mm_write_mm(c, off, path);
    free_spmat(c);
    if (rc != SP3MM_OK) {
        fprintf(stderr, "dropin_driver: writing %s failed\n", path);
        return 1;
    }
    return 0;
}

int main(int argc, char **argv) {
    if (argc != 6) {
        fprintf(stderr, "usage: %s r.mtx ac.mtx p.mtx out_dir off_f\n", argv[0]);
        return 2;
    }
    const int off = atoi(argv[5]) ? 1 : 0;
    spmat *R = MMtoCSR(argv[1]), *AC = MMtoCSR(argv[2]), *P = MMtoCSR(argv[3]);
    if (!R || !AC || !P) return 1;
    if (off) {
        shift(R, 1);
        shift(AC, 1);
        shift(P, 1);
    }
    SPMM_INTERF *spmm_ub = off ? Spmm_UB_Funcs_1 : Spmm_UB_Funcs_0;
    const size_t n_spmm_ub = off ? COUNT(Spmm_UB_Funcs_1) : COUNT(Spmm_UB_Funcs_0);
    SP3MM_INTERF *rap_ub = off ? Sp3mm_UB_Funcs_1 : Sp3mm_UB_Funcs_0;
    const size_t n_rap_ub = off ? COUNT(Sp3mm_UB_Funcs_1) : COUNT(Sp3mm_UB_Funcs_0);
    SPMM_INTERF *spmm_sn = off ? Spmm_SymbNum_Funcs_1 : Spmm_SymbNum_Funcs_0;
    const size_t n_spmm_sn = off ? COUNT(Spmm_SymbNum_Funcs_1) : COUNT(Spmm_SymbNum_Funcs_0);
    SP3MM_INTERF *rap_sn = off ? Sp3mm_SymbNum_Funcs_1 : Sp3mm_SymbNum_Funcs_0;
    const size_t n_rap_sn = off ? COUNT(Sp3mm_SymbNum_Funcs_1) : COUNT(Sp3mm_SymbNum_Funcs_0);
    SP3MM_INTERF pair = off ? sp3mmRowByRowPair_1 : sp3mmRowByRowPair_0;

    CONFIG cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.gridRows = 2;
    cfg.gridCols = 3;
    cfg.threadNum = 1;
    char tag[64];
    int fails = 0, results = 0;
    for (size_t f = 0; f < n_spmm_ub; ++f, ++results) {
        snprintf(tag, sizeof tag, "pair_ub_%zu", f);
        fails += emit(pair(R, AC, P, &cfg, spmm_ub[f]), argv[4], tag, off);
    }
    for (size_t f = 0; f < n_rap_ub; ++f, ++results) {
        snprintf(tag, sizeof tag, "direct_ub_%zu", f);
        fails += emit(rap_ub[f](R, AC, P, &cfg, NULL), argv[4], tag, off);
    }
    const ROW_MMSYM_IMPL_MODE modes[2] = {RBTREE, IDXMAP};
    for (int m = 0; m < 2; ++m) {
        cfg.symbMMRowImplID = modes[m];
        for (size_t f = 0; f < n_spmm_sn; ++f, ++results) {
            snprintf(tag, sizeof tag, "pair_sn%d_%zu", m, f);
            fails += emit(pair(R, AC, P, &cfg, spmm_sn[f]), argv[4], tag, off);
        }
        for (size_t f = 0; f < n_rap_sn; ++f, ++results) {
            snprintf(tag, sizeof tag, "direct_sn%d_%zu", m, f);
            fails += emit(rap_sn[f](R, AC, P, &cfg, NULL), argv[4], tag, off);
        }
    }
    if (off) {
        shift(R, (idx_t)-1);
        shift(AC, (idx_t)-1);
        shift(P, (idx_t)-1);
    }
    free_spmat(R);
    free_spmat(AC);
    free_spmat(P);
    printf("%d\n", results);
    return fails ? 1 : 0;
}
