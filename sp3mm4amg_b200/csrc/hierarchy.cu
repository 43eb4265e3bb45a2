// hierarchy.cu -- smoothed-aggregation prolongators and the device-resident
// AMG setup loop around the triple product.
//
// The reference computes one Galerkin product per call; its callers (the
// AMG4PSBLAS setup, and the level-by-level chain behind its test matrices,
// code/scripts/getLevels3MMmatrixes.py:29-38) repeat
// A_{l+1} = R_l A_l P_l until the operator is small.  This file keeps that
// loop on the device:
//
//   P0_l  tentative aggregation of non-overlapping block^d grid blocks of
//         level l's grid (one 1.0 per row),
//   P_l   = (I - omega D_l^-1 A_l) P0_l, one damped-Jacobi step, computed as
//         the SpGEMM A_l P0_l followed by an elementwise combine,
//   R_l   = P_l^T (device transpose),
//   A_l+1 = R_l A_l P_l with the library's product (direct or pair-wise).
//
// Arithmetic of the combine: s = omega / d_i (IEEE division), then
// p_ij = [j == agg(i)] - s * (A P0)_ij with separately rounded operations,
// the order of the host generator's (I - s A) P0 evaluation, so host and
// device prolongators agree bit for bit.
//
// Mixed precision: with coarse_val_type = SP3MM_F32, level 0 stays FP64
// (A_0, P_0, R_0 and the product accumulation), and every coarse operator
// and coarse prolongator is stored in FP32; products still accumulate in
// FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "hierarchy.cuh"
#include "kernels.cuh"
#include "sp3mm_b200.h"
#include "sp3mm_internal.cuh"

namespace sp3mm {
namespace {

template <typename T>
__device__ __forceinline__ double hv(const void* p, long long i) {
    return static_cast<double>(static_cast<const T*>(p)[i]);
}
__device__ __forceinline__ double hload(const void* p, int vt, long long i) {
    return vt == SP3MM_F32 ? hv<float>(p, i) : hv<double>(p, i);
}
__device__ __forceinline__ void hstore(void* p, int vt, long long i, double v) {
    if (vt == SP3MM_F32) static_cast<float*>(p)[i] = __double2float_rn(v);
    else static_cast<double*>(p)[i] = v;
}

// Aggregate of every grid point (lexicographic numbering, x fastest):
// the index of its block^d block on the coarse grid.
__global__ void k_block_labels(long long n, int nx, int ny, int nz, int block, int* agg) {
    const int cx = (nx + block - 1) / block, cy = (ny + block - 1) / block;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long x = i % nx, y = (i / nx) % ny, z = i / (static_cast<long long>(nx) * ny);
        agg[i] = static_cast<int>((x / block) + cx * ((y / block) + static_cast<long long>(cy) * (z / block)));
    }
}

// P0: row i has the single entry (agg[i], 1.0).
__global__ void k_p0(long long n, const int* agg, int* rp, int* ci, void* v, int vt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= n;
         i += (long long)gridDim.x * blockDim.x) {
        rp[i] = static_cast<int>(i);
        if (i < n) {
            ci[i] = agg[i];
            hstore(v, vt, i, 1.0);
        }
    }
}

// d[i] = A(i, i) (0 when the row has no diagonal entry), binary search in
// the row's ascending columns.
__global__ void k_diag(CsrView A, double* d, unsigned* err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.M; i += gridDim.x * blockDim.x) {
        int lo = A.rp[i], hi = A.rp[i + 1];
        double v = 0.0;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const int c = A.ci[mid];
            if (c == i) {
                v = hload(A.v, A.vtype, mid);
                break;
            }
            if (c < i) lo = mid + 1;
            else hi = mid;
        }
        if (v == 0.0) atomicOr(err, kErrInput);
        d[i] = v;
    }
}

// P = (I - omega D^-1 A) P0 on the pattern of A*P0 (which holds P0's
// pattern because every row of A has its diagonal).
__global__ void k_jacobi(CsrView AP0, const double* d, const int* agg, double omega, void* pv,
                         int pvt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < AP0.M; i += gridDim.x * blockDim.x) {
        const double s = __ddiv_rn(omega, d[i]);
        const int a = agg[i];
        for (int j = AP0.rp[i]; j < AP0.rp[i + 1]; ++j) {
            const double y = __dmul_rn(s, hload(AP0.v, AP0.vtype, j));
            const double v = AP0.ci[j] == a ? __dsub_rn(1.0, y) : -y;
            hstore(pv, pvt, j, v);
        }
    }
}

int grid_of(long long work) {
    long long g = (work + 255) / 256;
    return static_cast<int>(std::max<long long>(1, std::min<long long>(g, 148 * 16)));
}

CsrView dview(const sp3mm_dcsr& m) {
    return CsrView{m.M, m.N, m.nnz, m.row_ptr, m.col, m.val, m.val_type};
}

int fail(sp3mm_ctx* ctx, int code, const char* msg) { return report_error(ctx, code, msg); }

#define H_CK(call)                                                                      \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            return fail(ctx, SP3MM_ECUDA, cudaGetErrorString(e_));                       \
        }                                                                               \
    } while (0)

#define H_TRY(expr)                      \
    do {                                 \
        int rc_ = (expr);                \
        if (rc_ != SP3MM_OK) return rc_; \
    } while (0)

// Device scratch owned by one call (freed on scope exit, stream-ordered).
struct Scratch {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit Scratch(cudaStream_t s) : st(s) {}
    ~Scratch() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
    }
    template <typename T> T* get(size_t n) {
        void* p = nullptr;
        if (cudaMallocAsync(&p, sizeof(T) * (n ? n : 1), st) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

}  // namespace
}  // namespace sp3mm

using namespace sp3mm;

extern "C" {

int sp3mm_block_prolongator(sp3mm_ctx* ctx, const sp3mm_dcsr* A, const int32_t* dims, int ndim,
                            int block, double omega, int out_val_type, sp3mm_dcsr* P) {
    if (!ctx || !A || !dims || !P || ndim < 1 || ndim > 3 || block < 1 ||
        (out_val_type != SP3MM_F64 && out_val_type != SP3MM_F32) ||
        (A->val_type != SP3MM_F64 && A->val_type != SP3MM_F32) || !A->row_ptr)
        return fail(ctx, SP3MM_EINVAL, "block_prolongator: invalid arguments");
    const long long nx = dims[0], ny = ndim > 1 ? dims[1] : 1, nz = ndim > 2 ? dims[2] : 1;
    const long long n = nx * ny * nz;
    if (nx < 1 || ny < 1 || nz < 1 || n != A->M || A->M != A->N)
        return fail(ctx, SP3MM_EINVAL, "block_prolongator: grid does not match the operator");
    const long long cn = ((nx + block - 1) / block) * ((ny + block - 1) / block) *
                         ((nz + block - 1) / block);
    cudaStream_t st = static_cast<cudaStream_t>(sp3mm_ctx_stream(ctx));
    Scratch sc(st);
    int* agg = sc.get<int>(n);
    int* rp = sc.get<int>(n + 1);
    int* ci = sc.get<int>(n);
    void* v = A->val_type == SP3MM_F32 ? static_cast<void*>(sc.get<float>(n))
                                       : static_cast<void*>(sc.get<double>(n));
    double* d = sc.get<double>(n);
    unsigned* err = sc.get<unsigned>(1);
    if (!agg || !rp || !ci || !v || !d || !err)
        return fail(ctx, SP3MM_ENOMEM, "block_prolongator: device allocation failed");
    H_CK(cudaMemsetAsync(err, 0, sizeof(unsigned), st));
    k_block_labels<<<grid_of(n), 256, 0, st>>>(n, static_cast<int>(nx), static_cast<int>(ny),
                                                 static_cast<int>(nz), block, agg);
    k_p0<<<grid_of(n + 1), 256, 0, st>>>(n, agg, rp, ci, v, A->val_type);
    k_diag<<<grid_of(n), 256, 0, st>>>(dview(*A), d, err);
    note_launch();
    note_launch();
    note_launch();
    H_CK(cudaGetLastError());
    sp3mm_dcsr P0{};
    P0.M = static_cast<int>(n);
    P0.N = static_cast<int>(cn);
    P0.nnz = n;
    P0.row_ptr = rp;
    P0.col = ci;
    P0.val = v;
    P0.val_type = A->val_type;
    P0.max_row = 1;
    sp3mm_dcsr AP0{};
    if (A->max_row >= 0 && A->max_row <= kAggProductRow)
        H_TRY(agg_product(ctx, *A, agg, static_cast<int>(cn), &AP0));
    else
        H_TRY(sp3mm_spmm(ctx, A, &P0, SP3MM_UB, SP3MM_F64, &AP0));
    void* pv = AP0.val;
    if (out_val_type == SP3MM_F32) {
        if (cudaMallocAsync(&pv, sizeof(float) * std::max<long long>(AP0.nnz, 1), st) !=
            cudaSuccess) {
            cudaGetLastError();
            sp3mm_dcsr_free(ctx, &AP0);
            return fail(ctx, SP3MM_ENOMEM, "block_prolongator: device allocation failed");
        }
    }
    k_jacobi<<<grid_of(n), 256, 0, st>>>(dview(AP0), d, agg, omega, pv, out_val_type);
    note_launch();
    unsigned h_err = 0;
    H_CK(cudaMemcpyAsync(&h_err, err, sizeof h_err, cudaMemcpyDeviceToHost, st));
    H_CK(cudaStreamSynchronize(st));
    if (pv != AP0.val) {
        cudaFreeAsync(AP0.val, st);
        AP0.val = pv;
        AP0.val_type = SP3MM_F32;
    }
    if (h_err) {
        sp3mm_dcsr_free(ctx, &AP0);
        return fail(ctx, SP3MM_EINVAL, "block_prolongator: a row of A has no diagonal entry");
    }
    *P = AP0;
    return SP3MM_OK;
}

int sp3mm_hierarchy_free(sp3mm_ctx* ctx, sp3mm_hierarchy* h) {
    if (!ctx || !h) return SP3MM_EINVAL;
    if (h->owns_arrays) {
        for (size_t l = 0; l < h->P.size(); ++l) {
            sp3mm_dcsr_free(ctx, &h->P[l]);
            sp3mm_dcsr_free(ctx, &h->R[l]);
        }
        for (size_t l = 1; l < h->A.size(); ++l) sp3mm_dcsr_free(ctx, &h->A[l]);
    }
    delete h;   // releases the shared arenas of a batched build
    return SP3MM_OK;
}

int sp3mm_hierarchy_build(sp3mm_ctx* ctx, const sp3mm_dcsr* A0, const int32_t* dims, int ndim,
                          int block, double omega, int64_t min_coarse, int max_levels,
                          int variant, int flavour, int coarse_val_type,
                          sp3mm_hierarchy** out) {
    if (!ctx || !A0 || !dims || !out || ndim < 1 || ndim > 3 || block < 2 || max_levels < 1 ||
        (coarse_val_type != SP3MM_F64 && coarse_val_type != SP3MM_F32))
        return fail(ctx, SP3MM_EINVAL, "hierarchy_build: invalid arguments");
    sp3mm_hierarchy* h = new sp3mm_hierarchy();
    h->ndim = ndim;
    h->block = block;
    h->omega = omega;
    h->min_coarse = min_coarse;
    h->max_levels = max_levels;
    h->coarse_val_type = coarse_val_type;
    h->A.push_back(*A0);
    int nx = dims[0], ny = ndim > 1 ? dims[1] : 1, nz = ndim > 2 ? dims[2] : 1;
    h->nx.push_back(nx);
    h->ny.push_back(ny);
    h->nz.push_back(nz);
    while (static_cast<int>(h->A.size()) < max_levels && h->A.back().M >= min_coarse &&
           h->A.back().M > 1) {
        const sp3mm_dcsr& A = h->A.back();
        const int l = static_cast<int>(h->A.size()) - 1;
        // Level 0 keeps FP64 prolongators; coarse levels use coarse_val_type.
        const int pvt = l == 0 ? A0->val_type : coarse_val_type;
        const int avt = coarse_val_type;
        const int32_t d3[3] = {nx, ny, nz};
        sp3mm_dcsr P{}, R{}, Ac{};
        int rc = sp3mm_block_prolongator(ctx, &A, d3, ndim, block, omega, pvt, &P);
        if (rc == SP3MM_OK) rc = sp3mm_transpose(ctx, &P, &R);
        // The product needs one storage type: R and P follow A's.
        if (rc == SP3MM_OK && P.val_type != A.val_type)
            rc = fail(ctx, SP3MM_EINVAL, "hierarchy_build: level value types differ");
        if (rc == SP3MM_OK) rc = sp3mm_rap(ctx, &R, &A, &P, variant, flavour, avt, &Ac);
        if (rc != SP3MM_OK) {
            sp3mm_dcsr_free(ctx, &P);
            sp3mm_dcsr_free(ctx, &R);
            sp3mm_hierarchy_free(ctx, h);
            return rc;
        }
        h->P.push_back(P);
        h->R.push_back(R);
        h->A.push_back(Ac);
        nx = (nx + block - 1) / block;
        ny = (ny + block - 1) / block;
        nz = (nz + block - 1) / block;
        h->nx.push_back(nx);
        h->ny.push_back(ny);
        h->nz.push_back(nz);
    }
    h->nlev = static_cast<int>(h->A.size());
    *out = h;
    return SP3MM_OK;
}

int sp3mm_hierarchy_levels(const sp3mm_hierarchy* h) { return h ? h->nlev : 0; }

int sp3mm_hierarchy_get(const sp3mm_hierarchy* h, int level, sp3mm_dcsr* A, sp3mm_dcsr* P,
                        sp3mm_dcsr* R) {
    if (!h || level < 0 || level >= h->nlev) return SP3MM_EINVAL;
    if (A) *A = h->A[level];
    const bool has = level < static_cast<int>(h->P.size());
    if (P) *P = has ? h->P[level] : sp3mm_dcsr{};
    if (R) *R = has ? h->R[level] : sp3mm_dcsr{};
    return SP3MM_OK;
}

}  // extern "C"
