// rows_dense_small.cu -- the CTA-per-row direct kernel (rowdense.cuh) in its
// small configuration: half the dense slice (4,096 columns) and list (2,048
// R*A columns) in half the shared memory, at most 64 registers a thread, so
// two CTAs share an SM and hide each other's latency.  The heavy rows of
// products whose A has at least kDenseSmallMinCols columns run here first
// (128^3 level 2: 10.2 -> 8.6 ms); a row that outgrows the list or slice
// joins this launch's own retry list, which the default configuration
// runs next.
#define SP3MM_DENSE_NS dsmall
#define SP3MM_DENSE_SPAN 4096
#define SP3MM_DENSE_LIST 2048
#define SP3MM_DENSE_STAGE 64
#define SP3MM_DENSE_MINB 2
#include "rowdense.cuh"

namespace sp3mm {
namespace {

template <int MODE>
cudaError_t dense_small_typed(const DirectRowArgs& a, const RowParams& p, int grid,
                              cudaStream_t st) {
    using namespace dsmall;
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

}  // namespace

int dense_small_ctas_per_sm() {
    static int per_sm = -1;   // the same on every device of one kind
    if (per_sm < 0) {
        const void* f = reinterpret_cast<const void*>(
            dsmall::k_direct_dense<kNumBook, double, double>);
        const int smem = static_cast<int>(dsmall::dense_smem_bytes());
        int n = 0;
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, 32 * dsmall::kDWarps, smem) !=
                cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        per_sm = n;
    }
    return per_sm;
}

cudaError_t launch_direct_dense_small(const DirectRowArgs& a, const RowParams& p, int mode,
                                      int grid, cudaStream_t st) {
    if (p.nrows <= 0) return cudaSuccess;
    note_launch();
    if (grid > p.nrows) grid = p.nrows;
    if (mode == kSymb) return dense_small_typed<kSymb>(a, p, grid, st);
    if (mode == kNumExact) return dense_small_typed<kNumExact>(a, p, grid, st);
    return dense_small_typed<kNumBook>(a, p, grid, st);
}

}  // namespace sp3mm
