// rows_pair.cu -- instantiations and launcher of the pair-wise A*B row
// kernel (rows.cuh).
#include "rowwarp.cuh"

namespace sp3mm {

template <int MODE, bool GT>
static cudaError_t pair_warp_typed(const PairRowArgs& a, const RowParams& p, const RowGeom& geo,
                                   cudaStream_t st) {
    const int tv = a.A.vtype, to = p.c_vt;
    if (MODE == kSymb)
        return launch_row_kernel(k_pair_warp<kSymb, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F64)
        return launch_row_kernel(k_pair_warp<MODE, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F32)
        return launch_row_kernel(k_pair_warp<MODE, double, float, GT>, a, p, geo, st);
    if (tv == SP3MM_F32 && to == SP3MM_F32)
        return launch_row_kernel(k_pair_warp<MODE, float, float, GT>, a, p, geo, st);
    return launch_row_kernel(k_pair_warp<MODE, float, double, GT>, a, p, geo, st);
}

template <bool GT>
static cudaError_t pair_warp_mode(const PairRowArgs& a, const RowParams& p, int mode,
                                  const RowGeom& geo, cudaStream_t st) {
    if (mode == kSymb) return pair_warp_typed<kSymb, GT>(a, p, geo, st);
    if (mode == kNumExact) return pair_warp_typed<kNumExact, GT>(a, p, geo, st);
    return pair_warp_typed<kNumBook, GT>(a, p, geo, st);
}

template <int G, int MODE, bool GT>
static cudaError_t pair_typed(const PairRowArgs& a, const RowParams& p, const RowGeom& geo,
                                cudaStream_t st) {
    const int tv = a.A.vtype, to = p.c_vt;
    if (MODE == kSymb)
        return launch_row_kernel(k_pair_rows<G, kSymb, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F64)
        return launch_row_kernel(k_pair_rows<G, MODE, double, double, GT>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F32)
        return launch_row_kernel(k_pair_rows<G, MODE, double, float, GT>, a, p, geo, st);
    if (tv == SP3MM_F32 && to == SP3MM_F32)
        return launch_row_kernel(k_pair_rows<G, MODE, float, float, GT>, a, p, geo, st);
    return launch_row_kernel(k_pair_rows<G, MODE, float, double, GT>, a, p, geo, st);
}

template <int G, bool GT>
static cudaError_t pair_mode(const PairRowArgs& a, const RowParams& p, int mode,
                               const RowGeom& geo, cudaStream_t st) {
    if (mode == kSymb) return pair_typed<G, kSymb, GT>(a, p, geo, st);
    if (mode == kNumExact) return pair_typed<G, kNumExact, GT>(a, p, geo, st);
    return pair_typed<G, kNumBook, GT>(a, p, geo, st);
}

cudaError_t launch_pair_rows(const PairRowArgs& a, const RowParams& p, int mode,
                               const RowGeom& geo, cudaStream_t st) {
    if (p.nrows <= 0) return cudaSuccess;
    note_launch();
    if (p.gtab) return pair_warp_mode<true>(a, p, mode, geo, st);
    switch (geo.G) {
        case 4: return pair_mode<4, false>(a, p, mode, geo, st);
        case 8: return pair_mode<8, false>(a, p, mode, geo, st);
        case 16: return pair_mode<16, false>(a, p, mode, geo, st);
        default: return pair_warp_mode<false>(a, p, mode, geo, st);
    }
}

}  // namespace sp3mm
