// hierarchy.cuh -- the device hierarchy object shared by the single and the
// batched (level-synchronous) builds and the request server.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "sp3mm_b200.h"

struct sp3mm_hierarchy {
    int nlev = 0;
    std::vector<sp3mm_dcsr> A, P, R;   // A[0] is the caller's (borrowed)
    std::vector<int> nx, ny, nz;
    // Build parameters.
    int ndim = 3, block = 2, max_levels = 1, coarse_val_type = SP3MM_F64;
    long long min_coarse = 0;
    double omega = 2.0 / 3.0;
    // Matrices built by the batched build live in shared device arenas
    // (kept alive here) instead of owning their arrays.
    bool owns_arrays = true;
    std::vector<std::shared_ptr<void>> keep;
    // Prolongators the caller provides, one per level to build (device
    // copies kept alive through `keep`); empty: block aggregation on the
    // box grid.
    std::vector<sp3mm_dcsr> given_P;

    // Whether another level should be built.
    bool wants_level() const {
        if (!given_P.empty()) return A.size() <= given_P.size();
        const sp3mm_dcsr& a = A.back();
        return static_cast<int>(A.size()) < max_levels && a.M >= min_coarse && a.M > 1;
    }
};

namespace sp3mm {

// Advance every hierarchy of hs that wants another level by one level,
// level-synchronously: all their prolongators, restrictions and Galerkin
// products are formed by a few batched launches (direct triple product).
int hierarchy_step(sp3mm_ctx* ctx, const std::vector<sp3mm_hierarchy*>& hs);

// A*P0 for the aggregation P0 given by agg (fine point -> one of nc blocks,
// value 1.0) computed directly, one thread per row; A's rows must hold at
// most kAggProductRow entries (A.max_row known).  The result's arrays are
// the caller's (free with sp3mm_dcsr_free); bit-identical to the SpMM.
constexpr int kAggProductRow = 32;
int agg_product(sp3mm_ctx* ctx, const sp3mm_dcsr& A, const int* agg, int nc, sp3mm_dcsr* AP0);

}  // namespace sp3mm
