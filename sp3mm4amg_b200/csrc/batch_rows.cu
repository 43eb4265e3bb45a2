// batch_rows.cu -- instantiations and launcher of the batch row kernels.
#include "batch.cuh"
#include "rowbatch.cuh"
#include "rowdense.cuh"

namespace sp3mm {

using namespace dbig;   // the default CTA-per-row configuration (rowdense.cuh)
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

// Direct rows of a batch, one CTA per row with dense accumulators (the
// rows of the batch's heavy levels; rowdense.cuh).  In the symbolic and
// booked passes a row it cannot hold joins the retry rounds of the plan; the
// exact numeric pass (the captured graph) gets only rows whose R*A list fits.
template <int MODE, typename TV, typename TO>
__global__ void __launch_bounds__(kDWarps * 32, 1)
    k_batch_dense(const BItem* __restrict__ items, const int* __restrict__ row_item,
                  BatchRowParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_n1, s_lo, s_hi, s_cnt[kDWarps];
    __shared__ long long s_base;
    const DenseSmem d = dense_smem(smem, &s_n1, &s_lo, &s_hi, s_cnt, &s_base);
    dense_clear(d);
    const int nrows = p.nrows_dev ? *p.nrows_dev : p.nrows;
    for (long long it = blockIdx.x; it < nrows; it += gridDim.x) {
        const int g = p.rows[p.reverse ? nrows - 1 - it : it];
        const BItem* I = items + __ldg(row_item + g);
        if (I->kind != kBatchDirect) {
            // Only direct rows are routed here; anything else is redone by
            // the warp kernels of the retry rounds.
            if (threadIdx.x == 0) batch_retry(p, g, __ldg(p.need + g));
            continue;
        }
        const int i = static_cast<int>(g - I->row_base);
        const long long eb = MODE == kNumExact ? __ldg(p.c_rp + g) : 0;
        const long long ee = MODE == kNumExact ? eb + __ldg(p.cnt2 + g) : 0;
        int* oc = MODE == kNumExact ? p.c_ci : p.ub_ci;
        TO* ov = static_cast<TO*>(MODE == kNumExact ? p.c_v : p.ub_v);
        dense_row<MODE, TV, TO>(d, I->X, I->Y, I->Z, i, oc, ov, eb, ee,
                                [&](int n1, int n2, bool fail) -> long long {
            if (MODE == kNumExact) {
                // Routed only where the list fits; a count that differs
                // from the plan's is an error, as in the warp kernels.
                if (fail || n2 != ee - eb) atomicOr(p.err, kErrCount);
                return -1;
            }
            if (fail) {
                batch_retry(p, g, __ldg(p.need + g));
                return -1;
            }
            p.cnt1[g] = n1;
            p.cnt2[g] = n2;
            if (MODE == kSymb) return -1;
            const unsigned long long off =
                n2 > 0 ? atomicAdd(p.cursor, static_cast<unsigned long long>(n2)) : 0ULL;
            if (off + n2 > p.cap) {
                atomicOr(p.err, kErrBook);
                return -1;
            }
            p.row_off[g] = static_cast<long long>(off);
            return static_cast<long long>(off);
        });
    }
}

template <int MODE>
KFn pick_dense_types(int tv, int to) {
    const bool f_in = tv == SP3MM_F32, f_out = to == SP3MM_F32;
    if constexpr (MODE == kSymb) {
        (void)f_in;
        (void)f_out;
        return &k_batch_dense<MODE, double, double>;
    } else {
        if (!f_in && !f_out) return &k_batch_dense<MODE, double, double>;
        if (!f_in && f_out) return &k_batch_dense<MODE, double, float>;
        if (f_in && f_out) return &k_batch_dense<MODE, float, float>;
        return &k_batch_dense<MODE, float, double>;
    }
}

}  // namespace

size_t batch_dense_smem() { return dense_smem_bytes(); }

cudaError_t launch_batch_dense(int mode, int tv, int to, int grid, cudaStream_t st,
                               const BItem* items, const int* row_item, const BatchRowParams& p) {
    const KFn f = mode == kSymb      ? pick_dense_types<kSymb>(tv, to)
                  : mode == kNumBook ? pick_dense_types<kNumBook>(tv, to)
                                     : pick_dense_types<kNumExact>(tv, to);
    const size_t smem = dense_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(f),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    f<<<grid, kDWarps * 32, smem, st>>>(items, row_item, p);
    note_launch();
    return cudaGetLastError();
}

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
