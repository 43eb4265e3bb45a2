// rows_lanes.cu -- instantiations and launcher of the register-product direct
// R*A*P row kernel (rowlanes.cuh).
#include "rowlanes.cuh"

namespace sp3mm {

template <int MODE>
static cudaError_t lanes_typed(const DirectRowArgs& a, const RowParams& p, const RowGeom& geo,
                               cudaStream_t st) {
    const int tv = a.R.vtype, to = p.c_vt;
    if (MODE == kSymb)
        return launch_row_kernel(k_direct_lanes<kSymb, double, double>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F64)
        return launch_row_kernel(k_direct_lanes<MODE, double, double>, a, p, geo, st);
    if (tv == SP3MM_F64 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_lanes<MODE, double, float>, a, p, geo, st);
    if (tv == SP3MM_F32 && to == SP3MM_F32)
        return launch_row_kernel(k_direct_lanes<MODE, float, float>, a, p, geo, st);
    return launch_row_kernel(k_direct_lanes<MODE, float, double>, a, p, geo, st);
}

size_t lanes_row_bytes(int mode, int S1, int S2) {
    return wlanes_bytes(mode != kSymb, S1, S2);
}

cudaError_t launch_direct_lanes(const DirectRowArgs& a, const RowParams& p, int mode,
                                const RowGeom& geo, cudaStream_t st) {
    if (p.nrows <= 0) return cudaSuccess;
    if (p.lg1 < 0 || p.lg1 > 5 || p.lg2 < 0 || p.lg2 > 5 || p.S2 > p.S1 || p.gtab)
        return cudaErrorInvalidValue;
    note_launch();
    if (mode == kSymb) return lanes_typed<kSymb>(a, p, geo, st);
    if (mode == kNumExact) return lanes_typed<kNumExact>(a, p, geo, st);
    return lanes_typed<kNumBook>(a, p, geo, st);
}

}  // namespace sp3mm
