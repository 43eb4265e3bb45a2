// hbatch.cu -- level-synchronous construction of many hierarchies.
//
// Every step advances a set of hierarchies by one level with the same
// arithmetic as the single build (hierarchy.cu): P = (I - omega D^-1 A) P0
// on the pattern of A*P0, R = P^T, A_c = R A P (direct product).  Instead of
// a dozen launches and several host round trips per hierarchy, a step runs
//
//   labels + diagonals        one launch over the rows of all hierarchies
//   A*P0                      one thread per row when every operator's rows
//                             hold at most kAggRow entries (count, scan,
//                             fill), else one batch (sp3mm_batch, SpMM)
//   Jacobi combine            one launch
//   transpose                 column counts, scan, scatter, row sort and
//                             local row pointers over the block-diagonal
//                             concatenation of all P (five launches)
//   R*A*P                     one batch (direct triple products)
//
// Matrices built by a step live in arenas shared by the step's hierarchies
// (the two batches' result arrays and the restriction arrays); each
// hierarchy keeps them alive.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <memory>
#include <vector>

#include "batch.cuh"
#include "context.cuh"
#include "hierarchy.cuh"
#include "sp3mm_b200.h"

using namespace sp3mm;

namespace {

// One hierarchy of a step (device descriptor).
struct HStep {
    CsrView A;             // the hierarchy's coarsest operator
    int nx, ny, nz, block;
    int nc;                // coarse size
    long long row_base;    // first global fine row
    long long col_base;    // first global coarse column
    double omega;
    CsrView AP0;           // A*P0: the pattern of P, FP64 values
    void* pv;              // P values (AP0's array when FP64)
    int pvt;
    long long r_base;      // first entry of this R in the step's R arrays
};

__device__ __forceinline__ int find_base(const long long* __restrict__ bases, int n, long long g) {
    int lo = 0, hi = n;   // largest b with bases[b] <= g (bases[n] = total)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(bases + mid) <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double vload(const void* p, int vt, long long i) {
    return vt == SP3MM_F32 ? static_cast<double>(static_cast<const float*>(p)[i])
                           : static_cast<const double*>(p)[i];
}
__device__ __forceinline__ void vstore(void* p, int vt, long long i, double v) {
    if (vt == SP3MM_F32) static_cast<float*>(p)[i] = __double2float_rn(v);
    else static_cast<double*>(p)[i] = v;
}

// agg[g] = block of fine point g on its hierarchy's coarse grid (local
// coarse index); d[g] = diagonal entry (flag when missing or zero).
__global__ void k_hs_labels(const HStep* __restrict__ hs, const long long* __restrict__ bases,
                            int n, long long rows, int* agg, double* d, unsigned* err) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const HStep& h = hs[find_base(bases, n, g)];
        const long long i = g - h.row_base;
        const int b = h.block;
        const int cx = (h.nx + b - 1) / b, cy = (h.ny + b - 1) / b;
        const long long x = i % h.nx, y = (i / h.nx) % h.ny,
                        z = i / (static_cast<long long>(h.nx) * h.ny);
        agg[g] = static_cast<int>(x / b + cx * (y / b + static_cast<long long>(cy) * (z / b)));
        int lo = h.A.rp[i], hi = h.A.rp[i + 1];
        double v = 0.0;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const int c = h.A.ci[mid];
            if (c == i) {
                v = vload(h.A.v, h.A.vtype, mid);
                break;
            }
            if (c < i) lo = mid + 1;
            else hi = mid;
        }
        if (v == 0.0) atomicOr(err, kErrInput);
        d[g] = v;
    }
}

// P = (I - omega D^-1 A) P0 on the pattern of A*P0: s = omega / d_i, then
// [j == agg(i)] - s * (A P0)_ij, separately rounded (the single build's
// arithmetic).
__global__ void k_hs_jacobi(const HStep* __restrict__ hs, const long long* __restrict__ bases,
                            int n, long long rows, const int* agg, const double* d) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const HStep& h = hs[find_base(bases, n, g)];
        const int i = static_cast<int>(g - h.row_base);
        const double s = __ddiv_rn(h.omega, d[g]);
        const int a = agg[g];
        const double* x = static_cast<const double*>(h.AP0.v);
        for (int j = h.AP0.rp[i]; j < h.AP0.rp[i + 1]; ++j) {
            const double y = __dmul_rn(s, x[j]);
            vstore(h.pv, h.pvt, j, h.AP0.ci[j] == a ? __dsub_rn(1.0, y) : -y);
        }
    }
}

// Transpose of the block-diagonal concatenation of all P: entries per
// global coarse column.
__global__ void k_hs_colcount(const HStep* __restrict__ hs, const long long* __restrict__ bases,
                              int n, long long rows, int* cnt) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const HStep& h = hs[find_base(bases, n, g)];
        const int i = static_cast<int>(g - h.row_base);
        for (int j = h.AP0.rp[i]; j < h.AP0.rp[i + 1]; ++j)
            atomicAdd(cnt + h.col_base + h.AP0.ci[j], 1);
    }
}

__global__ void k_hs_scatter(const HStep* __restrict__ hs, const long long* __restrict__ bases,
                             int n, long long rows, const int* grp, int* cursor, int* r_ci,
                             void* r_v, int vt) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const HStep& h = hs[find_base(bases, n, g)];
        const int i = static_cast<int>(g - h.row_base);
        for (int j = h.AP0.rp[i]; j < h.AP0.rp[i + 1]; ++j) {
            const long long c = h.col_base + h.AP0.ci[j];
            const long long pos = grp[c] + atomicAdd(cursor + c, 1);
            r_ci[pos] = i;
            vstore(r_v, vt, pos, vload(h.pv, h.pvt, j));
        }
    }
}

// Local row pointers of every R: r_rp[r_rp_off[h] + j] = grp[col_base + j]
// - grp[col_base] for j = 0..nc.
__global__ void k_hs_local_rp(const HStep* __restrict__ hs, const long long* __restrict__ cbases,
                              int n, long long cols, const int* grp, const long long* r_rp_off,
                              int* r_rp) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cols;
         c += (long long)gridDim.x * blockDim.x) {
        const int b = find_base(cbases, n, c);
        const HStep& h = hs[b];
        const int j = static_cast<int>(c - h.col_base);
        const int c0 = grp[h.col_base];
        int* out = r_rp + r_rp_off[b];
        out[j] = grp[c] - c0;
        if (j == h.nc - 1) out[j + 1] = grp[c + 1] - c0;
    }
}

__global__ void k_hs_fill(long long n, int* iota, void* ones, int vt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= n;
         i += (long long)gridDim.x * blockDim.x) {
        iota[i] = static_cast<int>(i);
        if (i < n) vstore(ones, vt, i, 1.0);
    }
}

// A*P0 for an aggregation P0 (one 1.0 per row: fine point j -> its
// block agg(j)) on operators whose rows hold at most kAggRow entries (the
// fine levels' stencils), one thread per row: (A P0)_ic is the sum, over
// the row's entries j in order, of A_ij * 1.0 with agg(j) = c -- the same
// rounded products (x * 1.0 = x), added in the same order onto the same
// 0.0 start as the SpMM row kernels, so the result is bit-identical to the
// SpMM batch that the coarser levels still take.
constexpr int kAggRow = kAggProductRow;

// The row's distinct blocks in first-touch order (lab) and, SUMS, their
// sums; the row has at most kAggRow entries.
template <bool SUMS>
__device__ __forceinline__ int agg_row(const HStep& h, int i, const int* __restrict__ agg,
                                       int* lab, double* sum) {
    int n = 0;
    const int e1 = h.A.rp[i + 1];
    for (int e = h.A.rp[i]; e < e1; ++e) {
        const int c = agg[h.row_base + h.A.ci[e]];
        int q = 0;
        while (q < n && lab[q] != c) ++q;
        if (q == n) {
            lab[n] = c;
            if (SUMS) sum[n] = 0.0;
            ++n;
        }
        if (SUMS) sum[q] = __dadd_rn(sum[q], __dmul_rn(1.0, vload(h.A.v, h.A.vtype, e)));
    }
    return n;
}

// cnt[g] = distinct blocks of row g; maxrow[t] = the longest of
// hierarchy t (a longer A row than kAggRow flags kErrInput).
__global__ void k_hs_ap0_count(const HStep* __restrict__ hs, const long long* __restrict__ bases,
                               int n, long long rows, const int* __restrict__ agg, int* cnt,
                               int* maxrow, unsigned* err) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const int t = find_base(bases, n, g);
        const HStep& h = hs[t];
        const int i = static_cast<int>(g - h.row_base);
        int c = 0;
        if (h.A.rp[i + 1] - h.A.rp[i] > kAggRow) {
            atomicOr(err, kErrInput);
        } else {
            int lab[kAggRow];
            c = agg_row<false>(h, i, agg, lab, nullptr);
        }
        cnt[g] = c;
        const unsigned peers = __match_any_sync(__activemask(), t);
        const int m = static_cast<int>(__reduce_max_sync(peers, static_cast<unsigned>(c)));
        if ((peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0) atomicMax(maxrow + t, m);
    }
}

// Row g of A*P0 at grp[g]: blocks ascending with their sums.
__global__ void k_hs_ap0_fill(const HStep* __restrict__ hs, const long long* __restrict__ bases,
                              int n, long long rows, const int* __restrict__ agg,
                              const int* __restrict__ grp, int* ci, double* v) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const HStep& h = hs[find_base(bases, n, g)];
        const int i = static_cast<int>(g - h.row_base);
        if (h.A.rp[i + 1] - h.A.rp[i] > kAggRow) continue;
        int lab[kAggRow];
        double sum[kAggRow];
        const int c = agg_row<true>(h, i, agg, lab, sum);
        for (int a = 1; a < c; ++a) {
            const int l = lab[a];
            const double x = sum[a];
            int b = a - 1;
            while (b >= 0 && lab[b] > l) {
                lab[b + 1] = lab[b];
                sum[b + 1] = sum[b];
                --b;
            }
            lab[b + 1] = l;
            sum[b + 1] = x;
        }
        const int o = grp[g];
        for (int q = 0; q < c; ++q) {
            ci[o + q] = lab[q];
            v[o + q] = sum[q];
        }
    }
}

// Local row pointers of every hierarchy's A*P0 (hierarchy t's at
// lrp[bases[t] + t]), and off[t] = its first entry in the step's arrays
// (off[n] = the total).
__global__ void k_hs_ap0_rp(const long long* __restrict__ bases, int n, long long rows,
                            const int* __restrict__ grp, int* lrp, int* off) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
         g += (long long)gridDim.x * blockDim.x) {
        const int t = find_base(bases, n, g);
        const long long base = bases[t];
        const int b0 = grp[base];
        lrp[g + t] = grp[g] - b0;
        if (g + 1 == bases[t + 1]) lrp[g + t + 1] = grp[g + 1] - b0;
        if (g == base) off[t] = b0;
        if (g + 1 == rows) off[n] = grp[rows];
    }
}

int grid_of(long long work) {
    const long long g = (work + 255) / 256;
    return static_cast<int>(std::max<long long>(1, std::min<long long>(g, 148LL * 32)));
}

// Device memory released when the last hierarchy holding it is freed.
struct Arena {
    sp3mm_ctx* ctx;
    std::vector<void*> ptrs;
    explicit Arena(sp3mm_ctx* c) : ctx(c) {}
    ~Arena() {
        for (void* p : ptrs) cudaFreeAsync(p, ctx->stream);
    }
    void* take(DevBuf& b) {
        void* p = b.detach();
        ptrs.push_back(p);
        return p;
    }
};

std::shared_ptr<sp3mm_batch> hold(sp3mm_batch* b) {
    return std::shared_ptr<sp3mm_batch>(b, [](sp3mm_batch* p) { sp3mm_batch_free(p); });
}

}  // namespace

namespace {

// One step for hierarchies whose coarsest operators share a value type
// and whose coarse levels share a storage type.
int step_group(sp3mm_ctx* ctx, const std::vector<sp3mm_hierarchy*>& hs) {
    const cudaStream_t st = ctx->stream;
    const int k = static_cast<int>(hs.size());
    const int tv = hs[0]->A.back().val_type;
    const int cvt = hs[0]->coarse_val_type;
    const size_t vb = vbytes(tv);
    std::vector<HStep> H(k);
    std::vector<long long> bases(k + 1), cbases(k + 1);
    long long rows = 0, cols = 0, maxn = 0;
    for (int t = 0; t < k; ++t) {
        const sp3mm_hierarchy* h = hs[t];
        const sp3mm_dcsr& A = h->A.back();
        const int nx = h->nx.back(), ny = h->ny.back(), nz = h->nz.back(), b = h->block;
        if (static_cast<long long>(nx) * ny * nz != A.M || A.M != A.N)
            return set_error(ctx, SP3MM_EINVAL, "hierarchy step: grid does not match operator");
        HStep& s = H[t];
        s = HStep{};
        s.A = view(A);
        s.nx = nx;
        s.ny = ny;
        s.nz = nz;
        s.block = b;
        s.nc = ((nx + b - 1) / b) * ((ny + b - 1) / b) * ((nz + b - 1) / b);
        s.row_base = rows;
        s.col_base = cols;
        s.omega = h->omega;
        s.pvt = tv;
        bases[t] = rows;
        cbases[t] = cols;
        rows += A.M;
        cols += s.nc;
        maxn = std::max<long long>(maxn, A.M);
    }
    bases[k] = rows;
    cbases[k] = cols;
    if (rows >= INT32_MAX || cols >= INT32_MAX)
        return set_error(ctx, SP3MM_ELIMIT, "hierarchy step: too many rows");

    ProfSpan whole(ctx, "hstep");
    ProfSpan phase(ctx, "hstep.labels");
    DevBuf dH, dB, dCB, agg, d, iota, ones, cnt, cursor, grp, tmp, rrp_off;
    TRY(dH.alloc(ctx, sizeof(HStep) * k));
    TRY(dB.alloc(ctx, sizeof(long long) * (k + 1)));
    TRY(dCB.alloc(ctx, sizeof(long long) * (k + 1)));
    TRY(agg.alloc(ctx, sizeof(int) * rows));
    TRY(d.alloc(ctx, sizeof(double) * rows));
    TRY(iota.alloc(ctx, sizeof(int) * (maxn + 1)));
    TRY(ones.alloc(ctx, vb * maxn));
    CK(ctx, cudaMemcpyAsync(dH.p, H.data(), sizeof(HStep) * k, cudaMemcpyHostToDevice, st));
    CK(ctx, cudaMemcpyAsync(dB.p, bases.data(), sizeof(long long) * (k + 1),
                            cudaMemcpyHostToDevice, st));
    CK(ctx, cudaMemcpyAsync(dCB.p, cbases.data(), sizeof(long long) * (k + 1),
                            cudaMemcpyHostToDevice, st));
    k_hs_fill<<<grid_of(maxn + 1), 256, 0, st>>>(maxn, iota.as<int>(), ones.p, tv);
    k_hs_labels<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), k, rows,
                                               agg.as<int>(), d.as<double>(), ctx->d_err);
    note_launch();
    note_launch();
    CK(ctx, cudaGetLastError());

    // A*P0 for every hierarchy: directly when every operator's rows are
    // short (the fine levels), else one SpMM batch.
    phase.end();
    ProfSpan phase_ap0(ctx, "hstep.ap0");
    std::vector<sp3mm_dcsr> X(k), Y(k), Z(k);
    std::vector<sp3mm_dcsr> AP0(k), P(k), R(k);
    auto arena = std::make_shared<Arena>(ctx);
    std::shared_ptr<sp3mm_batch> b1;
    sp3mm_batch* raw = nullptr;
    bool short_rows = true;
    for (int t = 0; t < k; ++t) {
        const int mr = hs[t]->A.back().max_row;
        short_rows = short_rows && mr >= 0 && mr <= kAggRow;
    }
    if (short_rows) {
        DevBuf acnt, agrp, amax, aoff, arp, aci, av;
        TRY(acnt.alloc(ctx, sizeof(int) * rows));
        TRY(agrp.alloc(ctx, sizeof(int) * (rows + 1)));
        TRY(amax.alloc(ctx, sizeof(int) * k));
        TRY(aoff.alloc(ctx, sizeof(int) * (k + 1)));
        TRY(arp.alloc(ctx, sizeof(int) * (rows + k)));
        CK(ctx, cudaMemsetAsync(amax.p, 0, sizeof(int) * k, st));
        k_hs_ap0_count<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), k,
                                                      rows, agg.as<int>(), acnt.as<int>(),
                                                      amax.as<int>(), ctx->d_err);
        note_launch();
        const size_t atb = scan_temp_bytes(static_cast<int>(rows));
        TRY(tmp.alloc(ctx, atb));
        launch_scan(static_cast<int>(rows), acnt.as<int>(), agrp.as<int>(), tmp.p, atb, st);
        k_hs_ap0_rp<<<grid_of(rows), 256, 0, st>>>(dB.as<long long>(), k, rows, agrp.as<int>(),
                                                   arp.as<int>(), aoff.as<int>());
        note_launch();
        CK(ctx, cudaGetLastError());
        std::vector<int> hoff(k + 1), hmax(k);
        CK(ctx, cudaMemcpyAsync(hoff.data(), aoff.p, sizeof(int) * (k + 1),
                                cudaMemcpyDeviceToHost, st));
        CK(ctx, cudaMemcpyAsync(hmax.data(), amax.p, sizeof(int) * k, cudaMemcpyDeviceToHost,
                                st));
        TRY(check_device_err(ctx));   // synchronises: hoff and hmax are complete
        const long long total = hoff[k];
        TRY(aci.alloc(ctx, sizeof(int) * std::max<long long>(total, 1)));
        TRY(av.alloc(ctx, sizeof(double) * std::max<long long>(total, 1)));
        k_hs_ap0_fill<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), k,
                                                     rows, agg.as<int>(), agrp.as<int>(),
                                                     aci.as<int>(), av.as<double>());
        note_launch();
        CK(ctx, cudaGetLastError());
        int* a_rp = static_cast<int*>(arena->take(arp));
        int* a_ci = static_cast<int*>(arena->take(aci));
        double* a_v = static_cast<double*>(arena->take(av));
        for (int t = 0; t < k; ++t) {
            AP0[t] = sp3mm_dcsr{static_cast<int>(bases[t + 1] - bases[t]), H[t].nc,
                                static_cast<long long>(hoff[t + 1] - hoff[t]),
                                a_rp + bases[t] + t, a_ci + hoff[t], a_v + hoff[t], SP3MM_F64,
                                hmax[t]};
        }
    } else {
        std::vector<int> kinds(k, SP3MM_BATCH_SPMM);
        for (int t = 0; t < k; ++t) {
            X[t] = hs[t]->A.back();
            sp3mm_dcsr& p0 = Y[t];
            p0.M = static_cast<int>(bases[t + 1] - bases[t]);
            p0.N = H[t].nc;
            p0.nnz = p0.M;
            p0.row_ptr = iota.as<int>();
            p0.col = agg.as<int>() + bases[t];
            p0.val = ones.p;
            p0.val_type = tv;
            p0.max_row = 1;
        }
        TRY(sp3mm_batch_create(ctx, k, kinds.data(), X.data(), Y.data(), nullptr, SP3MM_F64,
                               &raw));
        b1 = hold(raw);
        TRY(sp3mm_batch_run(b1.get()));
        batch_trim(b1.get());
        for (int t = 0; t < k; ++t) TRY(sp3mm_batch_result(b1.get(), t, &AP0[t]));
    }

    // P values (in place when FP64) and the restriction arrays.
    phase_ap0.end();
    ProfSpan phase_jac(ctx, "hstep.jacobi");
    long long nnz_p = 0;
    std::vector<long long> r_base(k), rrp(k);
    long long rrp_total = 0;
    for (int t = 0; t < k; ++t) {
        r_base[t] = nnz_p;
        nnz_p += AP0[t].nnz;
        rrp[t] = rrp_total;
        rrp_total += H[t].nc + 1;
    }
    if (nnz_p >= INT32_MAX) return set_error(ctx, SP3MM_ELIMIT, "hierarchy step: P too large");
    void* p32 = nullptr;
    if (tv != SP3MM_F64) {
        DevBuf pv;
        TRY(pv.alloc(ctx, vb * nnz_p));
        p32 = arena->take(pv);
    }
    for (int t = 0; t < k; ++t) {
        H[t].AP0 = view(AP0[t]);
        H[t].pv = p32 ? static_cast<unsigned char*>(p32) + vb * r_base[t] : AP0[t].val;
        H[t].r_base = r_base[t];
    }
    CK(ctx, cudaMemcpyAsync(dH.p, H.data(), sizeof(HStep) * k, cudaMemcpyHostToDevice, st));
    k_hs_jacobi<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), k, rows,
                                               agg.as<int>(), d.as<double>());
    note_launch();
    CK(ctx, cudaGetLastError());

    // R = P^T of the block-diagonal concatenation.
    phase_jac.end();
    ProfSpan phase_tr(ctx, "hstep.transpose");
    TRY(cnt.alloc(ctx, sizeof(int) * (cols + 1)));
    TRY(cursor.alloc(ctx, sizeof(int) * (cols + 1)));
    TRY(grp.alloc(ctx, sizeof(int) * (cols + 1)));
    CK(ctx, cudaMemsetAsync(cnt.p, 0, sizeof(int) * (cols + 1), st));
    CK(ctx, cudaMemsetAsync(cursor.p, 0, sizeof(int) * (cols + 1), st));
    k_hs_colcount<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), k, rows,
                                                 cnt.as<int>());
    note_launch();
    const size_t tb = scan_temp_bytes(static_cast<int>(cols));
    TRY(tmp.alloc(ctx, tb));
    launch_scan(static_cast<int>(cols), cnt.as<int>(), grp.as<int>(), tmp.p, tb, st);
    DevBuf rci, rv, rrpb;
    TRY(rci.alloc(ctx, sizeof(int) * nnz_p));
    TRY(rv.alloc(ctx, vb * nnz_p));
    TRY(rrpb.alloc(ctx, sizeof(int) * rrp_total));
    TRY(rrp_off.alloc(ctx, sizeof(long long) * k));
    CK(ctx, cudaMemcpyAsync(rrp_off.p, rrp.data(), sizeof(long long) * k, cudaMemcpyHostToDevice,
                            st));
    k_hs_scatter<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), k, rows,
                                                grp.as<int>(), cursor.as<int>(), rci.as<int>(),
                                                rv.p, tv);
    note_launch();
    launch_sort_rows(static_cast<int>(cols), grp.as<int>(), rci.as<int>(), rv.p, tv, INT_MAX, st);
    k_hs_local_rp<<<grid_of(cols), 256, 0, st>>>(dH.as<HStep>(), dCB.as<long long>(), k, cols,
                                                 grp.as<int>(), rrp_off.as<long long>(),
                                                 rrpb.as<int>());
    note_launch();
    CK(ctx, cudaGetLastError());
    int* r_ci = static_cast<int*>(arena->take(rci));
    unsigned char* r_v = static_cast<unsigned char*>(arena->take(rv));
    int* r_rp = static_cast<int*>(arena->take(rrpb));
    for (int t = 0; t < k; ++t) {
        const int n = static_cast<int>(bases[t + 1] - bases[t]);
        P[t] = sp3mm_dcsr{n, H[t].nc, AP0[t].nnz, AP0[t].row_ptr, AP0[t].col,
                          H[t].pv, tv, AP0[t].max_row};
        R[t] = sp3mm_dcsr{H[t].nc, n, AP0[t].nnz, r_rp + rrp[t], r_ci + r_base[t],
                          r_v + vb * r_base[t], tv, -1};
    }

    // A_c = R*A*P for every hierarchy: one batch of direct products.
    phase_tr.end();
    ProfSpan phase_rap(ctx, "hstep.rap");
    std::vector<int> rk(k, SP3MM_BATCH_RAP);
    for (int t = 0; t < k; ++t) X[t] = R[t];
    raw = nullptr;
    std::vector<sp3mm_dcsr> Aop(k);
    for (int t = 0; t < k; ++t) Aop[t] = hs[t]->A.back();
    TRY(sp3mm_batch_create(ctx, k, rk.data(), X.data(), Aop.data(), P.data(), cvt, &raw));
    auto b2 = hold(raw);
    TRY(sp3mm_batch_run(b2.get()));
    batch_trim(b2.get());
    for (int t = 0; t < k; ++t) {
        sp3mm_hierarchy* h = hs[t];
        sp3mm_dcsr Ac{};
        TRY(sp3mm_batch_result(b2.get(), t, &Ac));
        const int b = h->block;
        h->P.push_back(P[t]);
        h->R.push_back(R[t]);
        h->A.push_back(Ac);
        h->nx.push_back((h->nx.back() + b - 1) / b);
        h->ny.push_back((h->ny.back() + b - 1) / b);
        h->nz.push_back((h->nz.back() + b - 1) / b);
        h->nlev = static_cast<int>(h->A.size());
        h->keep.push_back(b1);
        h->keep.push_back(b2);
        h->keep.push_back(arena);
    }
    return SP3MM_OK;
}

// One step for hierarchies whose prolongators the caller provides (same
// value types within the group): R = P^T by a device transpose per
// hierarchy, then one batch of direct R*A*P products for all of them.
int step_given(sp3mm_ctx* ctx, const std::vector<sp3mm_hierarchy*>& hs) {
    const int k = static_cast<int>(hs.size());
    const int cvt = hs[0]->coarse_val_type;
    ProfSpan whole(ctx, "hstep.given");
    std::vector<sp3mm_dcsr> X(k), Aop(k), P(k);
    std::vector<std::shared_ptr<void>> rkeep(k);
    for (int t = 0; t < k; ++t) {
        sp3mm_hierarchy* h = hs[t];
        const sp3mm_dcsr& A = h->A.back();
        P[t] = h->given_P[h->A.size() - 1];
        if (P[t].M != A.M || A.M != A.N || P[t].val_type != A.val_type)
            return set_error(ctx, SP3MM_EINVAL,
                             "hierarchy step: prolongator %zu does not match its operator",
                             h->A.size() - 1);
        auto R = std::shared_ptr<sp3mm_dcsr>(new sp3mm_dcsr{}, [ctx](sp3mm_dcsr* m) {
            sp3mm_dcsr_free(ctx, m);
            delete m;
        });
        TRY(sp3mm_transpose(ctx, &P[t], R.get()));
        X[t] = *R;
        Aop[t] = A;
        rkeep[t] = R;
    }
    std::vector<int> rk(k, SP3MM_BATCH_RAP);
    sp3mm_batch* raw = nullptr;
    TRY(sp3mm_batch_create(ctx, k, rk.data(), X.data(), Aop.data(), P.data(), cvt, &raw));
    auto b = hold(raw);
    TRY(sp3mm_batch_run(b.get()));
    batch_trim(b.get());
    for (int t = 0; t < k; ++t) {
        sp3mm_hierarchy* h = hs[t];
        sp3mm_dcsr Ac{};
        TRY(sp3mm_batch_result(b.get(), t, &Ac));
        h->P.push_back(P[t]);
        h->R.push_back(X[t]);
        h->A.push_back(Ac);
        h->nx.push_back(Ac.M);
        h->ny.push_back(1);
        h->nz.push_back(1);
        h->nlev = static_cast<int>(h->A.size());
        h->keep.push_back(rkeep[t]);
        h->keep.push_back(b);
    }
    return SP3MM_OK;
}

}  // namespace

namespace sp3mm {

int hierarchy_step(sp3mm_ctx* ctx, const std::vector<sp3mm_hierarchy*>& all) {
    // Group by (operator value type, coarse storage type), block-aggregation
    // hierarchies apart from those with given prolongators.
    std::vector<sp3mm_hierarchy*> groups[8];
    for (sp3mm_hierarchy* h : all)
        if (h->wants_level())
            groups[(h->given_P.empty() ? 0 : 4) + (h->A.back().val_type == SP3MM_F32 ? 2 : 0) +
                   (h->coarse_val_type == SP3MM_F32 ? 1 : 0)]
                .push_back(h);
    for (int g = 0; g < 8; ++g)
        if (!groups[g].empty()) TRY(g < 4 ? step_group(ctx, groups[g]) : step_given(ctx, groups[g]));
    return SP3MM_OK;
}

}  // namespace sp3mm

extern "C" {

int sp3mm_hierarchy_build_batch(sp3mm_ctx* ctx, int n, const sp3mm_dcsr* A0, const int32_t* dims,
                                const int32_t* ndims, int block, double omega,
                                int64_t min_coarse, int max_levels, int coarse_val_type,
                                sp3mm_hierarchy** out) {
    if (!ctx || n < 0 || (n > 0 && (!A0 || !dims || !ndims || !out)) || block < 2 ||
        max_levels < 1 || (coarse_val_type != SP3MM_F64 && coarse_val_type != SP3MM_F32))
        return set_error(ctx, SP3MM_EINVAL, "hierarchy_build_batch: invalid arguments");
    std::vector<sp3mm_hierarchy*> hs(n, nullptr);
    auto free_all = [&] {
        for (auto* h : hs)
            if (h) sp3mm_hierarchy_free(ctx, h);
    };
    for (int i = 0; i < n; ++i) {
        const int nd = ndims[i];
        const int32_t* dm = dims + 3 * i;
        int rc = check_dcsr(ctx, &A0[i], "A0");
        if (rc == SP3MM_OK && (nd < 1 || nd > 3))
            rc = set_error(ctx, SP3MM_EINVAL, "hierarchy_build_batch: bad dimension count");
        const int nx = dm[0], ny = nd > 1 ? dm[1] : 1, nz = nd > 2 ? dm[2] : 1;
        if (rc == SP3MM_OK && (nx < 1 || ny < 1 || nz < 1 ||
                               static_cast<long long>(nx) * ny * nz != A0[i].M ||
                               A0[i].M != A0[i].N))
            rc = set_error(ctx, SP3MM_EINVAL, "hierarchy_build_batch: grid does not match A0");
        if (rc != SP3MM_OK) {
            free_all();
            return rc;
        }
        auto* h = new sp3mm_hierarchy();
        h->ndim = nd;
        h->block = block;
        h->omega = omega;
        h->min_coarse = min_coarse;
        h->max_levels = max_levels;
        h->coarse_val_type = coarse_val_type;
        h->owns_arrays = false;
        h->A.push_back(A0[i]);
        h->nx.push_back(nx);
        h->ny.push_back(ny);
        h->nz.push_back(nz);
        h->nlev = 1;
        hs[i] = h;
    }
    for (;;) {
        bool any = false;
        for (auto* h : hs) any = any || h->wants_level();
        if (!any) break;
        const int rc = hierarchy_step(ctx, hs);
        if (rc != SP3MM_OK) {
            free_all();
            return rc;
        }
    }
    for (int i = 0; i < n; ++i) out[i] = hs[i];
    return SP3MM_OK;
}

}  // extern "C"

namespace sp3mm {

int agg_product(sp3mm_ctx* ctx, const sp3mm_dcsr& A, const int* agg, int nc, sp3mm_dcsr* AP0) {
    const cudaStream_t st = ctx->stream;
    if (A.max_row < 0 || A.max_row > kAggRow || A.M < 1) return SP3MM_EINVAL;
    const long long rows = A.M;
    HStep h{};
    h.A = view(A);
    h.nc = nc;
    const long long bases[2] = {0, rows};
    DevBuf dH, dB, cnt, grp, mx, off, tmp, rp, ci, v;
    TRY(dH.alloc(ctx, sizeof(HStep)));
    TRY(dB.alloc(ctx, sizeof(bases)));
    TRY(cnt.alloc(ctx, sizeof(int) * rows));
    TRY(grp.alloc(ctx, sizeof(int) * (rows + 1)));
    TRY(mx.alloc(ctx, sizeof(int)));
    TRY(off.alloc(ctx, sizeof(int) * 2));
    TRY(rp.alloc(ctx, sizeof(int) * (rows + 1)));
    CK(ctx, cudaMemcpyAsync(dH.p, &h, sizeof(HStep), cudaMemcpyHostToDevice, st));
    CK(ctx, cudaMemcpyAsync(dB.p, bases, sizeof(bases), cudaMemcpyHostToDevice, st));
    CK(ctx, cudaMemsetAsync(mx.p, 0, sizeof(int), st));
    k_hs_ap0_count<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), 1, rows,
                                                  agg, cnt.as<int>(), mx.as<int>(), ctx->d_err);
    note_launch();
    const size_t tb = scan_temp_bytes(static_cast<int>(rows));
    TRY(tmp.alloc(ctx, tb));
    launch_scan(static_cast<int>(rows), cnt.as<int>(), grp.as<int>(), tmp.p, tb, st);
    k_hs_ap0_rp<<<grid_of(rows), 256, 0, st>>>(dB.as<long long>(), 1, rows, grp.as<int>(),
                                               rp.as<int>(), off.as<int>());
    note_launch();
    CK(ctx, cudaGetLastError());
    int hoff[2] = {0, 0}, hmax = 0;
    CK(ctx, cudaMemcpyAsync(hoff, off.p, sizeof(hoff), cudaMemcpyDeviceToHost, st));
    CK(ctx, cudaMemcpyAsync(&hmax, mx.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY(check_device_err(ctx));   // synchronises: hoff and hmax are complete
    const long long total = hoff[1];
    TRY(ci.alloc(ctx, sizeof(int) * std::max<long long>(total, 1)));
    TRY(v.alloc(ctx, sizeof(double) * std::max<long long>(total, 1)));
    k_hs_ap0_fill<<<grid_of(rows), 256, 0, st>>>(dH.as<HStep>(), dB.as<long long>(), 1, rows,
                                                 agg, grp.as<int>(), ci.as<int>(),
                                                 v.as<double>());
    note_launch();
    CK(ctx, cudaGetLastError());
    *AP0 = sp3mm_dcsr{A.M, nc, total, rp.as<int>(), ci.as<int>(), v.p, SP3MM_F64, hmax};
    rp.detach();
    ci.detach();
    v.detach();
    return SP3MM_OK;
}

}  // namespace sp3mm
