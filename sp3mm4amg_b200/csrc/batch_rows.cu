// batch_rows.cu -- instantiations and launcher of the batch row kernels.
#include "batch.cuh"
#include "rowbatch.cuh"

namespace sp3mm {
namespace {

using KFn = void (*)(const BItem*, const int*, BatchRowParams);

template <int MODE, bool GT>
KFn pick_types(int tv, int to) {
    const bool f_in = tv == SP3MM_F32, f_out = to == SP3MM_F32;
    if constexpr (MODE == kSymb) {   // no values: one instantiation per layout
        (void)f_in;
        (void)f_out;
        return &k_batch_rows<MODE, double, double, GT>;
    } else {
        if (!f_in && !f_out) return &k_batch_rows<MODE, double, double, GT>;
        if (!f_in && f_out) return &k_batch_rows<MODE, double, float, GT>;
        if (f_in && f_out) return &k_batch_rows<MODE, float, float, GT>;
        return &k_batch_rows<MODE, float, double, GT>;
    }
}

KFn pick(int mode, bool gt, int tv, int to) {
    if (mode == kSymb) return gt ? pick_types<kSymb, true>(tv, to) : pick_types<kSymb, false>(tv, to);
    if (mode == kNumBook)
        return gt ? pick_types<kNumBook, true>(tv, to) : pick_types<kNumBook, false>(tv, to);
    return gt ? pick_types<kNumExact, true>(tv, to) : pick_types<kNumExact, false>(tv, to);
}

}  // namespace

cudaError_t batch_rows_configure(int mode, bool gt, int tv, int to, int block, size_t smem,
                                 size_t max_smem, int* ctas_per_sm) {
    const KFn f = pick(mode, gt, tv, to);
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(f),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(max_smem));
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, block, smem);
    *ctas_per_sm = n;
    return e;
}

cudaError_t launch_batch_rows(int mode, bool gt, int tv, int to, int grid, int block,
                              size_t smem, cudaStream_t st, const BItem* items,
                              const int* row_item, const BatchRowParams& p) {
    const KFn f = pick(mode, gt, tv, to);
    f<<<grid, block, smem, st>>>(items, row_item, p);
    note_launch();
    return cudaGetLastError();
}

size_t batch_row_region_bytes(bool num, int scap) { return batch_region_bytes(num, scap); }
int batch_slots_for(long long need) { return batch_slots(need); }

}  // namespace sp3mm
