// rows_lanes.cu -- instantiations and launcher of the register-product direct
// R*A*P row kernel (rowlanes.cuh).
#include "rowlanes.cuh"

namespace sp3mm {

template <int MODE, bool PACK>
static cudaError_t lanes_typed(const DirectRowArgs& a, const RowParams& p, const RowGeom& geo,
                               cudaStream_t st) {
    const int tv = a.R.vtype, to = p.c_vt;
    if (MODE == kSymb)
        return launch_row_kernel(k_direct_lanes<kSymb, double, double, PACK>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F64)
        return launch_row_kernel(k_direct_lanes<MODE, double, double, PACK>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_lanes<MODE, double, float, PACK>, a, p, geo, st);
    if (tv == SP3MM_F32 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_lanes<MODE, float, float, PACK>, a, p, geo, st);
    return launch_row_kernel(k_direct_lanes<MODE, float, double, PACK>, a, p, geo, st);
}

template <bool PACK>
static cudaError_t lanes_mode(const DirectRowArgs& a, const RowParams& p, int mode,
                              const RowGeom& geo, cudaStream_t st) {
    if (mode == kSymb) return lanes_typed<kSymb, PACK>(a, p, geo, st);
    if (mode == kNumExact) return lanes_typed<kNumExact, PACK>(a, p, geo, st);
    return lanes_typed<kNumBook, PACK>(a, p, geo, st);
}

size_t lanes_row_bytes(int mode, int S1, int S2) {
    return wlanes_bytes(mode != kSymb, S1, S2);
}

cudaError_t launch_direct_lanes(const DirectRowArgs& a, const RowParams& p, int mode,
                                const RowGeom& geo, cudaStream_t st) {
    if (p.nrows <= 0) return cudaSuccess;
    if (p.lg1 > 5 || p.lg2 > 5 || p.S2 > p.S1 || p.gtab) return cudaErrorInvalidValue;
    note_launch();
    // Packed batches when either stage needs them (they take any row).
    if (p.lg1 < 0 || p.lg2 < 0) return lanes_mode<true>(a, p, mode, geo, st);
    return lanes_mode<false>(a, p, mode, geo, st);
}

}  // namespace sp3mm
