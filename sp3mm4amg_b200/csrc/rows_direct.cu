// rows_direct.cu -- instantiations and launcher of the direct R*A*P row
// kernel (rows.cuh).
#include "rowdense.cuh"

namespace sp3mm {

using namespace dbig;   // the default CTA-per-row configuration (rowdense.cuh)

template <int MODE, bool GT>
static cudaError_t direct_warp_typed(const DirectRowArgs& a, const RowParams& p,
                                     const RowGeom& geo, cudaStream_t st) {
    const int tv = a.R.vtype, to = p.c_vt;
    if (MODE == kSymb)
        return launch_row_kernel(k_direct_warp<kSymb, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F64)
        return launch_row_kernel(k_direct_warp<MODE, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_warp<MODE, double, float, GT>, a, p, geo, st);
    if (tv == SP3MM_F32 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_warp<MODE, float, float, GT>, a, p, geo, st);
    return launch_row_kernel(k_direct_warp<MODE, float, double, GT>, a, p, geo, st);
}

template <bool GT>
static cudaError_t direct_warp_mode(const DirectRowArgs& a, const RowParams& p, int mode,
                                    const RowGeom& geo, cudaStream_t st) {
    if (mode == kSymb) return direct_warp_typed<kSymb, GT>(a, p, geo, st);
    if (mode == kNumExact) return direct_warp_typed<kNumExact, GT>(a, p, geo, st);
    return direct_warp_typed<kNumBook, GT>(a, p, geo, st);
}

template <int G, int MODE, bool GT>
static cudaError_t direct_typed(const DirectRowArgs& a, const RowParams& p, const RowGeom& geo,
                                cudaStream_t st) {
    const int tv = a.R.vtype, to = p.c_vt;
    if (MODE == kSymb)
        return launch_row_kernel(k_direct_rows<G, kSymb, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F64)
        return launch_row_kernel(k_direct_rows<G, MODE, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_rows<G, MODE, double, float, GT>, a, p, geo, st);
    if (tv == SP3MM_F32 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_rows<G, MODE, float, float, GT>, a, p, geo, st);
    return launch_row_kernel(k_direct_rows<G, MODE, float, double, GT>, a, p, geo, st);
}

template <int G, bool GT>
static cudaError_t direct_mode(const DirectRowArgs& a, const RowParams& p, int mode,
                               const RowGeom& geo, cudaStream_t st) {
    if (mode == kSymb) return direct_typed<G, kSymb, GT>(a, p, geo, st);
    if (mode == kNumExact) return direct_typed<G, kNumExact, GT>(a, p, geo, st);
    return direct_typed<G, kNumBook, GT>(a, p, geo, st);
}

template <int MODE>
static cudaError_t dense_typed(const DirectRowArgs& a, const RowParams& p, int grid,
                               cudaStream_t st) {
    const int tv = a.R.vtype, to = p.c_vt;
    RowGeom geo{};
    geo.G = 32 * kDWarps;
    geo.grid = grid;
    geo.block = 32 * kDWarps;
    geo.smem = dense_smem_bytes();
    if (MODE == kSymb)
        return launch_row_kernel(k_direct_dense<kSymb, double, double>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F64)
        return launch_row_kernel(k_direct_dense<MODE, double, double>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_dense<MODE, double, float>, a, p, geo, st);
    if (tv == SP3MM_F32 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_dense<MODE, float, float>, a, p, geo, st);
    return launch_row_kernel(k_direct_dense<MODE, float, double>, a, p, geo, st);
}

size_t dense_row_smem() { return dense_smem_bytes(); }

cudaError_t launch_direct_dense(const DirectRowArgs& a, const RowParams& p, int mode, int grid,
                                cudaStream_t st) {
    if (p.nrows <= 0) return cudaSuccess;
    note_launch();
    if (grid > p.nrows) grid = p.nrows;
    if (mode == kSymb) return dense_typed<kSymb>(a, p, grid, st);
    if (mode == kNumExact) return dense_typed<kNumExact>(a, p, grid, st);
    return dense_typed<kNumBook>(a, p, grid, st);
}

cudaError_t launch_direct_rows(const DirectRowArgs& a, const RowParams& p, int mode,
                               const RowGeom& geo, cudaStream_t st) {
    if (p.nrows <= 0) return cudaSuccess;
    note_launch();
    // A whole warp per row (and every global-table launch): warp kernels;
    // 4 / 8 / 16 lanes per row: the group kernels.
    if (p.gtab) return direct_warp_mode<true>(a, p, mode, geo, st);
    switch (geo.G) {
        case 4: return direct_mode<4, false>(a, p, mode, geo, st);
        case 8: return direct_mode<8, false>(a, p, mode, geo, st);
        case 16: return direct_mode<16, false>(a, p, mode, geo, st);
        default: return direct_warp_mode<false>(a, p, mode, geo, st);
    }
}

}  // namespace sp3mm
// Out-of-line helpers of the row kernels.
#include "rowwarp.cuh"

namespace sp3mm {

size_t row_table_bytes(bool direct, int mode, int G, int S1, int S2) {
    const bool num = mode != kSymb;
    if (G == 32) return direct ? wdirect_bytes(num, S1, S2) : wpair_bytes(num, S1);
    if (direct) return static_cast<size_t>(num ? 16 : 8) * (S1 + S2);
    return static_cast<size_t>(num ? 28 : 8) * S1;
}

int row_table_limit(int S, int G) { return table_limit(S, G); }

int row_prefetch_cover(int G) {
    switch (G) {
        case 4: return 4 * prefetch_depth<4>();
        case 8: return 8 * prefetch_depth<8>();
        case 16: return 16 * prefetch_depth<16>();
        default: return 32 * prefetch_depth<32>();
    }
}

}  // namespace sp3mm
