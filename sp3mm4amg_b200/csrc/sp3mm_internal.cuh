// sp3mm_internal.cuh -- shared definitions of the sm_100a Sp3MM kernels.
//
// Device CSR is 0-based int32 row_ptr / col with FP64 (or FP32) values.  All
// accumulation is FP64 with separately rounded multiply and add
// (__dmul_rn / __dadd_rn), never a fused multiply-add: the reference computes
// v[j] += b*a as a rounded product added to the accumulator
// (code/src/include/SpMMUtilsGeneric.h:49), and gcc -O2 on generic x86-64
// forms no FMA.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#define SP3MM_B200_NO_TABLES
#include "sp3mm_b200.h"

namespace sp3mm {

constexpr int kEmpty = -1;          // empty hash slot key
constexpr int kWarp = 32;

// Device error-flag bits (sticky word per context, read by the host after a
// product).
enum : unsigned {
    kErrTable = 1u,      // a hash table ran out of slots at the largest level
    kErrInput = 2u,      // malformed input CSR (row_ptr / col validation)
    kErrCount = 4u,      // numeric row length disagrees with the symbolic one
    kErrBook = 8u,       // upper-bound space booking exceeded its capacity
    kErrSpin = 16u       // a bounded wait gave up
};

// Value load/store in either storage type, accumulated in FP64.
template <typename T> __device__ __forceinline__ double ld_val(const T* p, long long i) {
    return static_cast<double>(__ldg(p + i));
}
template <typename T> __device__ __forceinline__ void st_val(T* p, long long i, double v) {
    p[i] = static_cast<T>(v);
}

// A group of G consecutive lanes of one warp working on one row.
template <int G>
struct Group {
    static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group size");
    unsigned mask;   // this group's lanes
    unsigned below;  // lanes of this group below the calling lane
    int gl;          // lane index inside the group
    __device__ __forceinline__ Group() {
        const int lane = threadIdx.x & 31;
        gl = lane & (G - 1);
        mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
        below = ((1u << lane) - 1u) & mask;
    }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ unsigned ballot(bool p) const { return __ballot_sync(mask, p); }
    template <typename T> __device__ __forceinline__ T bcast(T v, int src) const {
        return __shfl_sync(mask, v, src, G);
    }
    __device__ __forceinline__ int sum(int v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
        return v;
    }
    __device__ __forceinline__ long long sum64(long long v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
        return v;
    }
    __device__ __forceinline__ int max(int v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v = ::max(v, __shfl_xor_sync(mask, v, o, G));
        return v;
    }
};

// Open-addressing table of int keys with linear probing.  `smask` = slots-1
// (slots a power of two), `shift` = 32 - log2(slots).
__device__ __forceinline__ unsigned hash_slot(int key, int shift) {
    return (static_cast<unsigned>(key) * 2654435769u) >> shift;
}

// Find `key` or claim an empty slot for it.  Lanes of one step insert
// distinct keys, so a claimed slot is never contended by an equal key.
// Returns the slot, or -1 after probing every slot (table full).
__device__ __forceinline__ int table_insert(int* keys, unsigned smask, int shift, int key,
                                            bool& is_new) {
    unsigned s = hash_slot(key, shift);
    volatile int* vk = keys;
    for (unsigned probe = 0; probe <= smask; ++probe) {
        const int k = vk[s];
        if (k == key) { is_new = false; return static_cast<int>(s); }
        if (k == kEmpty) {
            const int old = atomicCAS(keys + s, kEmpty, key);
            if (old == kEmpty) { is_new = true; return static_cast<int>(s); }
            if (old == key) { is_new = false; return static_cast<int>(s); }
        }
        s = (s + 1) & smask;
    }
    is_new = false;
    return -1;
}

__device__ __forceinline__ int table_find(const int* keys, unsigned smask, int shift, int key) {
    unsigned s = hash_slot(key, shift);
    for (unsigned probe = 0; probe <= smask; ++probe) {
        const int k = keys[s];
        if (k == key) return static_cast<int>(s);
        if (k == kEmpty) return -1;
        s = (s + 1) & smask;
    }
    return -1;
}

__host__ __device__ __forceinline__ int ilog2_pow2(unsigned v) {
#ifdef __CUDA_ARCH__
    return 31 - __clz(v);
#else
    int r = 0;
    while ((1u << r) < v) ++r;
    return r;
#endif
}

__host__ __device__ __forceinline__ unsigned next_pow2(unsigned v) {
    if (v <= 1) return 1;
#ifdef __CUDA_ARCH__
    return 1u << (32 - __clz(v - 1));
#else
    unsigned p = 1;
    while (p < v) p <<= 1;
    return p;
#endif
}

}  // namespace sp3mm
