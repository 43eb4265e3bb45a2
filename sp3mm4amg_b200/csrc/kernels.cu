// kernels.cu -- bounds, binning, scans, compaction, conversions and
// transpose kernels of the Sp3MM library (sm_100a).  The per-row
// accumulation kernels are in rows.cu.
//
//  * Row binning by upper-bound size replaces the reference's OpenMP 1D / 2D
//    row and column partitions (code/src/Sp3MM_CSR_OMP_UB_Generic.c:85-105,
//    :153-182, :216-302): a bounds kernel gives each output row the number of
//    distinct keys its first table can receive (the reference's upper bound,
//    code/src/include/SpMMUtilsGeneric.h:112-139), and rows are grouped into
//    table-size levels by a count / scatter pair of kernels.
//  * The upper-bound flavour's merge (code/src/include/SpMMUtilsGeneric.h:
//    364-403) becomes a scan of the booked row lengths and a compaction kernel.
#include <cub/device/device_scan.cuh>

#include <atomic>
#include <climits>

#include "kernels.cuh"
#include "sp3mm_internal.cuh"

namespace sp3mm {

static std::atomic<uint64_t> g_launches{0};
uint64_t launch_count() { return g_launches.load(); }
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

__device__ __forceinline__ double load_val(const void* p, int vt, long long i) {
    if (vt == SP3MM_F32) return static_cast<double>(__ldg(static_cast<const float*>(p) + i));
    return __ldg(static_cast<const double*>(p) + i);
}
__device__ __forceinline__ void store_val(void* p, int vt, long long i, double v) {
    if (vt == SP3MM_F32) static_cast<float*>(p)[i] = __double2float_rn(v);
    else static_cast<double*>(p)[i] = v;
}

// ---------------------------------------------------------------------------
// Bounds.

// need[i] = min(flops_i, B.N) with flops_i = sum_{k in A(i)} len(B(k)).
template <int G>
__global__ void __launch_bounds__(256) k_pair_bounds(CsrView A, CsrView B, int* need,
                                                      unsigned long long* total) {
    const Group<G> g;
    const int groups = (gridDim.x * blockDim.x) / G;
    unsigned long long mine = 0;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < A.M; row += groups) {
        const int ab = __ldg(A.rp + row), ae = __ldg(A.rp + row + 1);
        long long f = 0;
        for (int t = ab + g.gl; t < ae; t += G) {
            const int k = __ldg(A.ci + t);
            f += __ldg(B.rp + k + 1) - __ldg(B.rp + k);
        }
        f = g.sum64(f);
        if (g.gl == 0) {
            const long long d = f < B.N ? f : B.N;
            need[row] = static_cast<int>(d < INT_MAX ? d : INT_MAX);
            mine += static_cast<unsigned long long>(f);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(total, mine);
}

// Direct R*A*P: need[i] = min(u1_i, A.N) with u1_i = sum_{k in R(i)} len(A(k))
// (the R*A row's products); total += u1_i * p_max_row, a bound on the C row's
// multiply-adds (each R*A entry forwards one P row of at most p_max_row
// entries).
template <int G>
__global__ void __launch_bounds__(256) k_direct_bounds(CsrView R, CsrView A, int p_max_row,
                                                        int* need, int* need_opt, int d1,
                                                        unsigned long long* total) {
    const Group<G> g;
    const int groups = (gridDim.x * blockDim.x) / G;
    unsigned long long mine = 0;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / G; row < R.M; row += groups) {
        const int rb = __ldg(R.rp + row), re = __ldg(R.rp + row + 1);
        long long u1 = 0;
        for (int t = rb + g.gl; t < re; t += G) {
            const int k = __ldg(R.ci + t);
            u1 += __ldg(A.rp + k + 1) - __ldg(A.rp + k);
        }
        u1 = g.sum64(u1);
        if (g.gl == 0) {
            const long long d = u1 < A.N ? u1 : A.N;
            need[row] = static_cast<int>(d < INT_MAX ? d : INT_MAX);
            if (need_opt) {
                // Optimistic first-table size: the bound >> d1, at most
                // 8 sqrt(products) -- long R*A rows repeat their columns
                // (stencil coarse levels: ~6 sqrt, kNN rows: <= 8.4 sqrt);
                // a row that overflows is recomputed with the bound.  A row
                // with at least as many products as A has columns is taken
                // as dense (the coarsest levels: every column, hundreds of
                // thousands of products) and gets the bound itself, which
                // bins it to the CTA-per-row kernel instead of a warp that
                // overflows and retries alone.
                long long o = d >> d1;
                const long long r =
                    static_cast<long long>(ceil(8.0 * sqrt(static_cast<double>(u1))));
                if (r < o) o = r;
                if (u1 >= A.N) o = d;
                if (d > 0 && o < 1) o = 1;
                need_opt[row] = static_cast<int>(o < INT_MAX ? o : INT_MAX);
            }
            mine += static_cast<unsigned long long>(u1) * static_cast<unsigned long long>(p_max_row);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(total, mine);
}

__global__ void k_need_from_counts(int M, const int* cnt, const int* cnt1, int* need) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    int n = cnt[i];
    if (cnt1 && n > 0) n = max(n, cnt1[i]);
    need[i] = n;
}

// ---------------------------------------------------------------------------
// Binning by table-size level.

__host__ __device__ __forceinline__ int limit_of(long long S, int G) {
    const long long a = S - G - 1, b = (7 * S) / 8;
    return static_cast<int>(a < b ? a : b);
}

__host__ __device__ __forceinline__ int level_of(long long need, int G) {
    if (need <= 0) return -1;
    int L = 0;
    while (L < kLevels - 1 && limit_of(32ll << L, G) < need) ++L;
    return L;
}

int slots_for_need(long long need, int G) {
    const int L = level_of(need < 1 ? 1 : need, G);
    return 32 << L;
}
int level_for_need(long long need, int G) { return level_of(need, G); }

__global__ void __launch_bounds__(256) k_bin_levels(int M, const int* need, const int* est,
                                                     int shift, int G, signed char* level,
                                                     int* counts, int* nmax, int* row_cnt_zero) {
    __shared__ int sc[kLevels + 1];
    __shared__ int smax;
    for (int i = threadIdx.x; i <= kLevels; i += blockDim.x) sc[i] = 0;
    if (threadIdx.x == 0) smax = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
        const int n = need[i];
        int L = -1;
        if (n > 0) {
            const int s = est ? est[i] : n >> shift;
            L = level_of(s > 0 ? s : 1, G);
        }
        level[i] = static_cast<signed char>(L);
        if (L < 0) {
            atomicAdd(&sc[kLevels], 1);
            if (row_cnt_zero) row_cnt_zero[i] = 0;
        } else {
            atomicAdd(&sc[L], 1);
            atomicMax(&smax, n);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= kLevels; i += blockDim.x)
        if (sc[i]) atomicAdd(counts + i, sc[i]);
    if (threadIdx.x == 0 && smax) atomicMax(nmax, smax);
}

// Append every row to its level's list (cursors hold each list's start).
__global__ void __launch_bounds__(256) k_bin_scatter(int M, const signed char* level,
                                                      int* cursors, int* lists) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < M;
    const int L = in ? level[i] : -1;
    // Warp-aggregated append keeps the rows of a warp contiguous and ascending.
    const unsigned act = __ballot_sync(0xffffffffu, in && L >= 0);
    if (!(in && L >= 0)) return;
    const unsigned peers = __match_any_sync(act, L);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cursors + L, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    lists[base + __popc(peers & ((1u << lane) - 1u))] = i;
}

// ---------------------------------------------------------------------------
// Upper-bound flavour: copy of booked rows into exact CSR.  8 lanes per row.
__global__ void __launch_bounds__(256) k_compact(int M, const int* row_cnt,
                                                  const long long* row_off, const int* ub_ci,
                                                  const void* ub_v, const int* c_rp, int* c_ci,
                                                  void* c_v, int vt) {
    const Group<8> g;
    const int groups = (gridDim.x * blockDim.x) / 8;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 8; row < M; row += groups) {
        const int n = row_cnt[row];
        if (!n) continue;
        const long long src = row_off[row];
        const long long dst = c_rp[row];
        for (int i = g.gl; i < n; i += 8) {
            c_ci[dst + i] = ub_ci[src + i];
            if (vt == SP3MM_F32)
                static_cast<float*>(c_v)[dst + i] = static_cast<const float*>(ub_v)[src + i];
            else
                static_cast<double*>(c_v)[dst + i] = static_cast<const double*>(ub_v)[src + i];
        }
    }
}

// ---------------------------------------------------------------------------
// Conversions between the host ABI (64-bit, OFF_F based) and device CSR.

__global__ void k_narrow_rowptr(long long M, long long nnz, const unsigned long long* src,
                                int off, int* dst, unsigned* err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= M;
         i += (long long)gridDim.x * blockDim.x) {
        const long long v = static_cast<long long>(src[i]) - off;
        bool bad = v < 0 || v > nnz;
        if (i == 0) bad |= v != 0;
        if (i == M) bad |= v != nnz;
        if (i > 0) bad |= static_cast<long long>(src[i - 1]) - off > v;
        if (bad) atomicOr(err, kErrInput);
        dst[i] = static_cast<int>(bad ? 0 : v);
    }
}

// Warp per row: narrow columns, check range and strict ascending order.
__global__ void __launch_bounds__(256) k_narrow_cols(long long M, long long N, const int* rp,
                                                      const unsigned long long* src, int off,
                                                      int* dst, int* max_row, unsigned* err) {
    const int lane = threadIdx.x & 31;
    const long long warps = (gridDim.x * (long long)blockDim.x) / 32;
    int my_max = 0;
    for (long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / 32; row < M;
         row += warps) {
        const int b = rp[row], e = rp[row + 1];
        my_max = max(my_max, e - b);
        for (int j = b + lane; j < e; j += 32) {
            const long long c = static_cast<long long>(src[j]) - off;
            bool bad = c < 0 || c >= N;
            if (j > b) bad |= static_cast<long long>(src[j - 1]) - off >= c;
            if (bad) atomicOr(err, kErrInput);
            dst[j] = static_cast<int>(bad ? 0 : c);
        }
    }
    if (lane == 0 && my_max) atomicMax(max_row, my_max);
}

__global__ void k_widen(long long n, const int* src, int off, unsigned long long* dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = static_cast<unsigned long long>(static_cast<long long>(src[i]) + off);
}

__global__ void k_convert_values(long long n, const void* src, int st_, void* dst, int dt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        store_val(dst, dt, i, load_val(src, st_, i));
}

// Validate a device-side int32 CSR: row_ptr monotone from 0, columns in
// range and strictly ascending within rows.
__global__ void __launch_bounds__(256) k_validate_i32(int M, int N, const int* rp,
                                                       const int* ci, int* max_row,
                                                       unsigned* err) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) / 32;
    int my_max = 0;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < M; row += warps) {
        const int b = rp[row], e = rp[row + 1];
        if (e < b || (row == 0 && b != 0)) {
            if (lane == 0) atomicOr(err, kErrInput);
            continue;
        }
        my_max = max(my_max, e - b);
        for (int j = b + lane; j < e; j += 32) {
            const int c = ci[j];
            bool bad = c < 0 || c >= N;
            if (j > b) bad |= ci[j - 1] >= c;
            if (bad) atomicOr(err, kErrInput);
        }
    }
    if (lane == 0 && my_max) atomicMax(max_row, my_max);
}

// ---------------------------------------------------------------------------
// Transpose.

__global__ void k_col_counts(long long nnz, const int* ci, int* counts) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnz;
         i += (long long)gridDim.x * blockDim.x)
        atomicAdd(counts + ci[i], 1);
}

__global__ void __launch_bounds__(256) k_transpose_scatter(CsrView A, const int* t_rp,
                                                            int* cursor, int* t_ci, void* t_v) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) / 32;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < A.M; row += warps) {
        const int b = A.rp[row], e = A.rp[row + 1];
        for (int j = b + lane; j < e; j += 32) {
            const int c = A.ci[j];
            const int pos = t_rp[c] + atomicAdd(cursor + c, 1);
            t_ci[pos] = row;
            if (A.vtype == SP3MM_F32)
                static_cast<float*>(t_v)[pos] = static_cast<const float*>(A.v)[j];
            else
                static_cast<double*>(t_v)[pos] = static_cast<const double*>(A.v)[j];
        }
    }
}

// Rows of more than 32 and at most kSortSmemRow entries: a warp per row
// sorts the row in shared memory with a bitonic network (the coarse levels'
// restrictions hold rows of hundreds of entries; odd-even transposition in
// global memory took 2.8 ms for the 512 rows of 677 entries of 128^3 level
// 3).  Columns within a row are distinct, so the order is unique.
constexpr int kSortSmemRow = 2048;
constexpr int kSortSmemWarps = 4;

__global__ void __launch_bounds__(kSortSmemWarps * 32) k_sort_rows_smem(int M, const int* rp,
                                                                        int* ci, void* v, int vt) {
    extern __shared__ __align__(16) unsigned char sort_smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    double* sv = reinterpret_cast<double*>(sort_smem) + static_cast<size_t>(w) * kSortSmemRow;
    int* sk = reinterpret_cast<int*>(reinterpret_cast<double*>(sort_smem) +
                                     static_cast<size_t>(kSortSmemWarps) * kSortSmemRow) +
              static_cast<size_t>(w) * kSortSmemRow;
    const int warps = (gridDim.x * blockDim.x) / 32;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < M; row += warps) {
        const int b = rp[row], e = rp[row + 1];
        const int n = e - b;
        if (n <= 32 || n > kSortSmemRow) continue;
        int P2 = 64;
        while (P2 < n) P2 <<= 1;
        for (int i = lane; i < P2; i += 32) {
            sk[i] = i < n ? ci[b + i] : INT_MAX;
            sv[i] = i < n ? load_val(v, vt, b + i) : 0.0;
        }
        __syncwarp();
        for (int k = 2; k <= P2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < P2; i += 32) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const int a0 = sk[i], a1 = sk[ixj];
                        if ((a0 > a1) == ((i & k) == 0)) {
                            sk[i] = a1;
                            sk[ixj] = a0;
                            const double x0 = sv[i];
                            sv[i] = sv[ixj];
                            sv[ixj] = x0;
                        }
                    }
                }
                __syncwarp();
            }
        }
        for (int i = lane; i < n; i += 32) {
            ci[b + i] = sk[i];
            store_val(v, vt, b + i, sv[i]);
        }
        __syncwarp();
    }
}

// Sort each row's (col, val) by col.  Warp per row; rows up to 32 entries by
// rank in registers, rows of k_sort_rows_smem's range there, longer rows by
// odd-even transposition in place.
__global__ void __launch_bounds__(256) k_sort_rows(int M, const int* rp, int* ci, void* v,
                                                    int vt) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) / 32;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32; row < M; row += warps) {
        const int b = rp[row], e = rp[row + 1];
        const int n = e - b;
        if (n <= 1) continue;
        if (n <= 32) {
            const bool in = lane < n;
            const int k = in ? ci[b + lane] : INT_MAX;
            const double x = in ? load_val(v, vt, b + lane) : 0.0;
            int r = 0;
            for (int j = 0; j < n; ++j) r += __shfl_sync(0xffffffffu, k, j) < k;
            __syncwarp();
            if (in) {
                ci[b + r] = k;
                store_val(v, vt, b + r, x);
            }
            __syncwarp();
            continue;
        }
        if (n <= kSortSmemRow) continue;   // k_sort_rows_smem
        for (int phase = 0; phase < n; ++phase) {
            for (int i = b + (phase & 1) + 2 * lane; i + 1 < e; i += 64) {
                const int a0 = ci[i], a1 = ci[i + 1];
                if (a0 > a1) {
                    ci[i] = a1;
                    ci[i + 1] = a0;
                    const double x0 = load_val(v, vt, i), x1 = load_val(v, vt, i + 1);
                    store_val(v, vt, i, x1);
                    store_val(v, vt, i + 1, x0);
                }
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// 2D column-partition upper bounds (code/src/include/SpMMUtilsGeneric.h:146-174).
__global__ void k_colparts_ub(CsrView A, int gridCols, const long long* off, long long* out,
                              unsigned long long* total) {
    unsigned long long mine = 0;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         x < static_cast<long long>(A.M) * gridCols; x += (long long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(x / gridCols);
        const int gc = static_cast<int>(x % gridCols);
        long long s = 0;
        for (int jj = A.rp[r]; jj < A.rp[r + 1]; ++jj) {
            const long long id = static_cast<long long>(A.ci[jj]) * gridCols + gc;
            s += off[id + 1] - off[id];
        }
        out[x] = s;
        mine += static_cast<unsigned long long>(s);
    }
    if (mine) atomicAdd(total, mine);
}

// ---------------------------------------------------------------------------
// Host launchers.

static inline int grid_for(long long work, int block, int cap = 148 * 16) {
    long long g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<int>(g);
}

void launch_pair_bounds(const CsrView& A, const CsrView& B, int* need,
                        unsigned long long* total, cudaStream_t st) {
    if (A.M == 0) return;
    k_pair_bounds<8><<<grid_for(static_cast<long long>(A.M) * 8, 256), 256, 0, st>>>(A, B, need,
                                                                                     total);
    note_launch();
}

void launch_direct_bounds(const CsrView& R, const CsrView& A, int p_max_row, int* need,
                          unsigned long long* total, cudaStream_t st, int* need_opt, int d1) {
    if (R.M == 0) return;
    k_direct_bounds<8><<<grid_for(static_cast<long long>(R.M) * 8, 256), 256, 0, st>>>(
        R, A, p_max_row, need, need_opt, d1, total);
    note_launch();
}

__global__ void k_count_max(int M, const int* cnt, const int* rp, int* out,
                            unsigned long long* sum) {
    int m = 0;
    unsigned long long t = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
        const int c = cnt ? cnt[i] : rp[i + 1] - rp[i];
        m = max(m, c);
        t += static_cast<unsigned long long>(c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (m > 0) atomicMax(out, m);
        if (sum && t) atomicAdd(sum, t);
    }
}

void launch_count_max(int M, const int* cnt, const int* rp, int* out, cudaStream_t st,
                      unsigned long long* sum) {
    if (M == 0) return;
    k_count_max<<<grid_for(M, 256), 256, 0, st>>>(M, cnt, rp, out, sum);
    note_launch();
}

void launch_need_from_counts(int M, const int* cnt, const int* cnt1, int* need,
                             cudaStream_t st) {
    if (M == 0) return;
    k_need_from_counts<<<(M + 255) / 256, 256, 0, st>>>(M, cnt, cnt1, need);
    note_launch();
}

void launch_bin_levels(int M, const int* need, int shift, int G, signed char* level,
                       int* counts, int* nmax, int* row_cnt_zero, cudaStream_t st,
                       const int* est) {
    if (M == 0) return;
    k_bin_levels<<<grid_for(M, 256), 256, 0, st>>>(M, need, est, shift, G, level, counts, nmax,
                                                    row_cnt_zero);
    note_launch();
}

void launch_bin_scatter(int M, const signed char* level, int* cursors, int* lists,
                        cudaStream_t st) {
    if (M == 0) return;
    k_bin_scatter<<<(M + 255) / 256, 256, 0, st>>>(M, level, cursors, lists);
    note_launch();
}

void launch_compact(int M, const int* row_cnt, const long long* row_off, const int* ub_ci,
                    const void* ub_v, const int* c_rp, int* c_ci, void* c_v, int vt,
                    cudaStream_t st) {
    if (M == 0) return;
    k_compact<<<grid_for(static_cast<long long>(M) * 8, 256), 256, 0, st>>>(
        M, row_cnt, row_off, ub_ci, ub_v, c_rp, c_ci, c_v, vt);
    note_launch();
}

size_t scan_temp_bytes(int M) {
    size_t bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, bytes, static_cast<const int*>(nullptr),
                                  static_cast<int*>(nullptr), M > 0 ? M : 1);
    return bytes;
}

void launch_scan(int M, const int* cnt, int* row_ptr, void* temp, size_t temp_bytes,
                 cudaStream_t st) {
    cudaMemsetAsync(row_ptr, 0, sizeof(int), st);
    if (M == 0) return;
    cub::DeviceScan::InclusiveSum(temp, temp_bytes, cnt, row_ptr + 1, M, st);
    note_launch();
}

void launch_narrow_rowptr(long long M, long long nnz, const unsigned long long* src, int off,
                          int* dst, unsigned* err, cudaStream_t st) {
    k_narrow_rowptr<<<grid_for(M + 1, 256), 256, 0, st>>>(M, nnz, src, off, dst, err);
    note_launch();
}

void launch_narrow_cols(long long M, long long N, const int* rp, const unsigned long long* src,
                        int off, int* dst, int* max_row, unsigned* err, cudaStream_t st) {
    if (M == 0) return;
    k_narrow_cols<<<grid_for(M * 32, 256), 256, 0, st>>>(M, N, rp, src, off, dst, max_row,
                                                         err);
    note_launch();
}

void launch_widen(long long n, const int* src, int off, unsigned long long* dst,
                  cudaStream_t st) {
    if (n == 0) return;
    k_widen<<<grid_for(n, 256), 256, 0, st>>>(n, src, off, dst);
    note_launch();
}

void launch_convert_values(long long n, const void* src, int src_type, void* dst, int dst_type,
                           cudaStream_t st) {
    if (n == 0) return;
    k_convert_values<<<grid_for(n, 256), 256, 0, st>>>(n, src, src_type, dst, dst_type);
    note_launch();
}

void launch_validate_i32(int M, int N, const int* rp, const int* ci, int* max_row,
                         unsigned* err, cudaStream_t st) {
    if (M == 0) return;
    k_validate_i32<<<grid_for(static_cast<long long>(M) * 32, 256), 256, 0, st>>>(
        M, N, rp, ci, max_row, err);
    note_launch();
}

void launch_col_counts(long long nnz, const int* ci, int* counts, cudaStream_t st) {
    if (nnz == 0) return;
    k_col_counts<<<grid_for(nnz, 256), 256, 0, st>>>(nnz, ci, counts);
    note_launch();
}

void launch_transpose_scatter(const CsrView& A, const int* t_rp, int* cursor, int* t_ci,
                              void* t_v, cudaStream_t st) {
    if (A.M == 0) return;
    k_transpose_scatter<<<grid_for(static_cast<long long>(A.M) * 32, 256), 256, 0, st>>>(
        A, t_rp, cursor, t_ci, t_v);
    note_launch();
}

void launch_sort_rows(int M, const int* rp, int* ci, void* v, int vt, int max_row,
                      cudaStream_t st) {
    if (M == 0 || max_row <= 1) return;
    k_sort_rows<<<grid_for(static_cast<long long>(M) * 32, 256), 256, 0, st>>>(M, rp, ci, v,
                                                                              vt);
    note_launch();
    if (max_row > 32) {
        const int smem = kSortSmemWarps * kSortSmemRow * 12;
        // A failure here surfaces as the launch's error (callers check it).
        cudaFuncSetAttribute(k_sort_rows_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
        k_sort_rows_smem<<<grid_for(static_cast<long long>(M) * 32, kSortSmemWarps * 32),
                           kSortSmemWarps * 32, smem, st>>>(M, rp, ci, v, vt);
        note_launch();
    }
}

void launch_colparts_ub(const CsrView& A, int gridCols, const long long* bColOffsets,
                        long long* out, unsigned long long* total, cudaStream_t st) {
    const long long work = static_cast<long long>(A.M) * gridCols;
    if (work == 0) return;
    k_colparts_ub<<<grid_for(work, 256), 256, 0, st>>>(A, gridCols, bColOffsets, out, total);
    note_launch();
}

}  // namespace sp3mm
