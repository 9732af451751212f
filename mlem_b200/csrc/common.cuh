// common.cuh -- device helpers shared by the MLEM kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define MLEM_FULL_MASK 0xffffffffu

namespace mlem {

// Number of SMs of a B200 (2 dies x 74); grids are sized in multiples of it.
constexpr int kB200SMs = 148;

// ---------------------------------------------------------------------------
// Cache-policy loads.  The element stream (8 bytes per matrix element) is
// read once per pass and must not evict the small hot vectors (image,
// correlation, sinogram, norm) from the 126 MB L2, so it is loaded with an
// L2 evict_first policy and without L1 allocation.  Gathers into the hot
// vectors use evict_last.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// 16-byte streaming load of two elements, no L1 allocation.
__device__ __forceinline__ uint4 ld_stream(const uint4* ptr, uint64_t pol) {
    uint4 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(ptr), "l"(pol));
    return r;
}

// 8-byte streaming load of one element.
__device__ __forceinline__ uint2 ld_stream2(const uint2* ptr, uint64_t pol) {
    uint2 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
        : "=r"(r.x), "=r"(r.y)
        : "l"(ptr), "l"(pol));
    return r;
}

__device__ __forceinline__ uint2 ld_keep2(const uint2* ptr, uint64_t pol) {
    uint2 r;
    asm("ld.global.nc.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
        : "=r"(r.x), "=r"(r.y)
        : "l"(ptr), "l"(pol));
    return r;
}

// 16-byte load that allocates in L1 (the fused one-pass kernel re-reads the row).
__device__ __forceinline__ uint4 ld_keep(const uint4* ptr, uint64_t pol) {
    uint4 r;
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(ptr), "l"(pol));
    return r;
}

__device__ __forceinline__ float ld_hot(const float* ptr, uint64_t pol) {
    float r;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(r) : "l"(ptr), "l"(pol));
    return r;
}

__device__ __forceinline__ float4 ld_hot4(const float4* ptr, uint64_t pol) {
    float4 r;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
        : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
        : "l"(ptr), "l"(pol));
    return r;
}

// ---------------------------------------------------------------------------
// Group reductions.  G lanes (a power of two dividing 32) cooperate on one
// row; BT frame accumulators per lane.  After group_reduce_scatter, lane l of
// the group holds the complete sum of frame l / (G/BT) in v[0]
// (recursive halving: log2(BT) exchange steps move half the frames each,
// then log2(G/BT) plain butterfly steps).  Every lane of the warp must call
// it (full-mask shuffles).
// ---------------------------------------------------------------------------
template <int G, int BT>
__device__ __forceinline__ void group_reduce_scatter(float (&v)[BT], int lane) {
    static_assert(BT <= G, "frame tile wider than the lane group");
#pragma unroll
    for (int h = BT / 2, off = G / 2; h >= 1; h >>= 1, off >>= 1) {
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            float send = upper ? v[i] : v[i + h];
            float keep = upper ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(MLEM_FULL_MASK, send, off);
        }
    }
#pragma unroll
    for (int off = G / (2 * BT); off >= 1; off >>= 1)
        v[0] += __shfl_xor_sync(MLEM_FULL_MASK, v[0], off);
}

template <int G>
__device__ __forceinline__ float group_allreduce(float v) {
#pragma unroll
    for (int off = G / 2; off >= 1; off >>= 1) v += __shfl_xor_sync(MLEM_FULL_MASK, v, off);
    return v;
}

// calcCorrel (mlem_seq/seqcsr4mlem.cpp:99): count / projection, 0 where the
// projection is 0.  IEEE division (-prec-div=true).
__device__ __forceinline__ float correl_of(int32_t s, float f) {
    return f != 0.0f ? __int2float_rn(s) / f : 0.0f;
}

// calcUpdate factor (mlem_seq/seqcsr4mlem.cpp:128).
__device__ __forceinline__ float update_factor(float u, float n) {
    return n != 0.0f ? u / n : u;
}

}  // namespace mlem
