// colparts.cu -- the reference's 2D column-partition utilities for host CSR
// `spmat`s (host code): uniform column ranges, per (row, range) offsets, and
// the ranges copied out as separate matrices.
//
// Follows code/src/commons/sparseUtilsGeneric.c:284-400 and its helpers
// :217-275, compiled per index base OFF_F like the reference
// (code/src/Sp3MM_CSR_OMP_Multi.c:56-66):
//
// * range gc of gridCols covers columns [gc*(N/gridCols) + min(gc, N%gridCols),
//   +N/gridCols + (gc < N%gridCols)) -- the first N%gridCols ranges one
//   column wider (code/src/include/macros.h:50-55);
// * offsets[r*gridCols + gc] = the 0-based position in JA/AS of row r's first
//   entry at or past range gc's first column; offsets[M*gridCols] = NZ
//   (malloc'd, idx_t[M*gridCols + 1]);
// * a partition is a calloc'd array of gridCols spmat structs: M rows, N =
//   the range's width, IRP calloc'd idx_t[M+1] with 0-based running offsets
//   (also for OFF_F = 1, as in the reference), JA / AS malloc'd copies of
//   the range's entries with JA unchanged (original column indices, OFF_F
//   included), NZ the entry count, MAX_ROW_NZ 0.  Free each with
//   freeSpmatInternal and the array with free().
//
// Differences, where the reference fails or has undefined behaviour: a NULL
// matrix or gridCols == 0 (a division by zero there) returns NULL with a
// message; a range with no entries gets NULL JA / AS (the reference's
// realloc to 0 bytes returns NULL and fails the whole call).
//
// Rows are independent: offsets and copies run on host threads by row
// chunks; each range's row pointers come from one scan of the per-row
// lengths.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "sp3mm_b200.h"

namespace {

void cp_error(const char* fn, const char* what) {
    fprintf(stderr, "sp3mm_b200: %s: %s\n", fn, what);
}

template <typename F>
void cp_parallel(idx_t rows, idx_t work, F&& f) {
    const unsigned hw = std::thread::hardware_concurrency();
    size_t t = static_cast<size_t>(work >> 20) + 1;
    if (t > 16) t = 16;
    if (hw && t > hw) t = hw;
    if (t > rows) t = rows ? rows : 1;
    if (t <= 1) {
        f(idx_t(0), rows);
        return;
    }
    std::vector<std::thread> th;
    for (size_t k = 0; k < t; ++k) {
        const idx_t b = rows * k / t, e = rows * (k + 1) / t;
        th.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto& x : th) x.join();
}

bool cp_valid(const char* fn, const spmat* A, unsigned gridCols) {
    if (!A || gridCols == 0) {
        cp_error(fn, "NULL matrix or gridCols == 0");
        return false;
    }
    if (A->M && (!A->IRP || (A->NZ && (!A->JA || !A->AS)))) {
        cp_error(fn, "matrix without IRP / JA / AS arrays");
        return false;
    }
    return true;
}

// offsets[r*gc_n + gc] for rows [rb, re) (0-based positions).
template <int OFF>
void row_offsets(const spmat* A, unsigned gridCols, idx_t rb, idx_t re, idx_t* offsets) {
    const idx_t blk = A->N / gridCols, rem = A->N % gridCols;
    for (idx_t r = rb; r < re; ++r) {
        idx_t j = A->IRP[r] - OFF;
        const idx_t end = A->IRP[r + 1] - OFF;
        offsets[r * gridCols] = j;
        for (idx_t gc = 1; gc < gridCols; ++gc) {
            const idx_t start = gc * blk + std::min<idx_t>(gc, rem);
            while (j < end && A->JA[j] - OFF < start) ++j;
            offsets[r * gridCols + gc] = j;
        }
    }
}

template <int OFF>
idx_t* col_offsets(const char* fn, spmat* A, unsigned gridCols) {
    if (!cp_valid(fn, A, gridCols)) return nullptr;
    const idx_t n = A->M * gridCols;
    idx_t* offsets = static_cast<idx_t*>(malloc((n + 1) * sizeof(idx_t)));
    if (!offsets) {
        cp_error(fn, "offsets malloc failed");
        return nullptr;
    }
    cp_parallel(A->M, A->NZ + n,
                [&](idx_t rb, idx_t re) { row_offsets<OFF>(A, gridCols, rb, re, offsets); });
    offsets[n] = A->NZ;
    return offsets;
}

void free_parts(spmat* parts, unsigned gridCols) {
    if (!parts) return;
    for (unsigned i = 0; i < gridCols; ++i) {
        free(parts[i].AS);
        free(parts[i].JA);
        free(parts[i].IRP);
    }
    free(parts);
}

// The column ranges of A as gridCols matrices, from A's offsets.
spmat* parts_from_offsets(const char* fn, const spmat* A, unsigned gridCols,
                          const idx_t* offsets) {
    const idx_t blk = A->N / gridCols, rem = A->N % gridCols, M = A->M;
    spmat* parts = static_cast<spmat*>(calloc(gridCols, sizeof(spmat)));
    if (!parts) {
        cp_error(fn, "partitions calloc failed");
        return nullptr;
    }
    for (unsigned gc = 0; gc < gridCols; ++gc) {
        spmat& p = parts[gc];
        p.M = M;
        p.N = blk + (gc < rem ? 1 : 0);
        p.IRP = static_cast<idx_t*>(calloc(M + 1, sizeof(idx_t)));
        if (!p.IRP) {
            cp_error(fn, "IRP calloc failed");
            free_parts(parts, gridCols);
            return nullptr;
        }
        // Running offsets of the range's rows (0-based, as the reference).
        idx_t run = 0;
        for (idx_t r = 0; r < M; ++r) {
            p.IRP[r] = run;
            run += offsets[r * gridCols + gc + 1] - offsets[r * gridCols + gc];
        }
        p.IRP[M] = run;
        p.NZ = run;
        if (run) {
            p.JA = static_cast<idx_t*>(malloc(run * sizeof(idx_t)));
            p.AS = static_cast<double*>(malloc(run * sizeof(double)));
            if (!p.JA || !p.AS) {
                cp_error(fn, "partition JA / AS malloc failed");
                free_parts(parts, gridCols);
                return nullptr;
            }
        }
    }
    cp_parallel(M, A->NZ, [&](idx_t rb, idx_t re) {
        for (idx_t r = rb; r < re; ++r)
            for (unsigned gc = 0; gc < gridCols; ++gc) {
                const idx_t s = offsets[r * gridCols + gc];
                const idx_t len = offsets[r * gridCols + gc + 1] - s;
                if (!len) continue;
                spmat& p = parts[gc];
                memcpy(p.JA + p.IRP[r], A->JA + s, len * sizeof(idx_t));
                memcpy(p.AS + p.IRP[r], A->AS + s, len * sizeof(double));
            }
    });
    return parts;
}

template <int OFF>
spmat* col_parts(const char* fn, spmat* A, unsigned gridCols, idx_t** offsets_out) {
    if (offsets_out) *offsets_out = nullptr;
    idx_t* offsets = col_offsets<OFF>(fn, A, gridCols);
    if (!offsets) return nullptr;
    spmat* parts = parts_from_offsets(fn, A, gridCols, offsets);
    if (parts && offsets_out)
        *offsets_out = offsets;
    else
        free(offsets);
    return parts;
}

}  // namespace

extern "C" {

SP3MM_API idx_t* colsOffsetsPartitioningUnifRanges_0(spmat* A, unsigned int gridCols) {
    return col_offsets<0>("colsOffsetsPartitioningUnifRanges_0", A, gridCols);
}
SP3MM_API idx_t* colsOffsetsPartitioningUnifRanges_1(spmat* A, unsigned int gridCols) {
    return col_offsets<1>("colsOffsetsPartitioningUnifRanges_1", A, gridCols);
}
SP3MM_API spmat* colsPartitioningUnifRanges_0(spmat* A, unsigned int gridCols) {
    return col_parts<0>("colsPartitioningUnifRanges_0", A, gridCols, nullptr);
}
SP3MM_API spmat* colsPartitioningUnifRanges_1(spmat* A, unsigned int gridCols) {
    return col_parts<1>("colsPartitioningUnifRanges_1", A, gridCols, nullptr);
}
SP3MM_API spmat* colsPartitioningUnifRangesOffsetsAux_0(spmat* A, unsigned int gridCols,
                                                        idx_t** colPartsOffsets) {
    return col_parts<0>("colsPartitioningUnifRangesOffsetsAux_0", A, gridCols, colPartsOffsets);
}
SP3MM_API spmat* colsPartitioningUnifRangesOffsetsAux_1(spmat* A, unsigned int gridCols,
                                                        idx_t** colPartsOffsets) {
    return col_parts<1>("colsPartitioningUnifRangesOffsetsAux_1", A, gridCols, colPartsOffsets);
}

}  // extern "C"
