// k_order.cu -- the row visiting order of the row kernels.
//
// A grid-stride row kernel runs neighbouring rows at the same time: the 8
// warps of a block take 8 consecutive rows.  The rows of a Siddon matrix
// (LORs) are random lines, so in file order those 8 rays share almost no
// voxels and every image gather misses L1.  Sorting the rows by the Morton
// interleave of (entry voxel, exit voxel) -- the first and last element of
// the row, whose device indices are already a Morton code of the voxel --
// puts rays with nearby endpoints next to each other: nearly coincident rays
// whose gathers hit the same cache lines.  For a matrix without geometry the
// key is still a valid (harmless) permutation.  Results change only by the
// order of the scatter atomics, which is unordered anyway.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace mlem {

namespace {

// Spread the 32 bits of v over the even bits of a 64-bit word.
__device__ __forceinline__ uint64_t spread2(uint32_t v) {
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

__global__ void k_row_keys(SparseView csr, uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < csr.n;
         r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = csr.ptr[r], e = csr.ptr[r + 1];
        uint64_t k = ~0ull;  // empty rows last
        if (e > b) {
            const uint32_t a = el[b].x, z = el[e - 1].x;
            const uint32_t lo = a < z ? a : z, hi = a < z ? z : a;  // direction-free
            k = (spread2(hi) << 1) | spread2(lo);
        }
        key[r] = k;
        idx[r] = (uint32_t)r;
    }
}

__global__ void k_row_ranges(SparseView csr, const uint32_t* __restrict__ order,
                             ulonglong2* __restrict__ vrange) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < csr.n;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = order[k];
        vrange[k] = make_ulonglong2(csr.ptr[r], csr.ptr[r + 1]);
    }
}

// Whether the row at visiting position k has a count in some frame (the
// selection flag, computed as the select reads it).
struct HasCount {
    const uint32_t* order;
    const int32_t* sino;
    uint32_t Bp;
    __host__ __device__ __forceinline__ uint8_t operator()(uint32_t k) const {
        const int32_t* s = sino + (size_t)order[k] * Bp;
        bool any = false;
        for (uint32_t f = 0; f < Bp; ++f) any |= (s[f] != 0);
        return any ? 1 : 0;
    }
};
using PosIt = thrust::counting_iterator<uint32_t>;
using FlagIt = thrust::transform_iterator<HasCount, PosIt, uint8_t>;

// The selected visiting positions (in act_order) become the rows and their
// ranges, in place; *z += their elements (one atomic per warp).
__global__ void k_active_gather(const uint32_t* __restrict__ order,
                                const ulonglong2* __restrict__ vrange,
                                const uint32_t* __restrict__ n_act, uint32_t* __restrict__ act_order,
                                ulonglong2* __restrict__ act_ranges, unsigned long long* __restrict__ z) {
    const uint64_t n = *n_act;
    unsigned long long mine = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = act_order[i];
        const ulonglong2 q = vrange[k];
        act_order[i] = order[k];
        act_ranges[i] = q;
        mine += q.y - q.x;
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(MLEM_FULL_MASK, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(z, mine);
}

// Bit k & 31 of keep[k >> 5]: whether the ray at visiting position k has a
// count in some frame (one ballot per 32 positions; whole warps, so the
// grid stride stays a multiple of 32).
__global__ void k_pos_keep(HasCount has, uint32_t n, uint32_t* __restrict__ keep) {
    const uint64_t n32 = ((uint64_t)n + 31) & ~31ull;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n32;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const bool f = k < n && has((uint32_t)k);
        const unsigned w = __ballot_sync(MLEM_FULL_MASK, f);
        if ((threadIdx.x & 31) == 0) keep[k >> 5] = w;
    }
}

// A warp per column: the column's entries whose rays are kept, in their order,
// from the start of the column's span; len[col] = their number.  Each step
// takes kSteps batches of 32 entries, their loads and flag gathers in flight
// together.
__global__ void __launch_bounds__(256) k_csc_active(const uint64_t* __restrict__ ptr,
                                                    const uint2* __restrict__ src, uint32_t C,
                                                    const uint32_t* __restrict__ keep,
                                                    uint2* __restrict__ dst,
                                                    uint32_t* __restrict__ len) {
    constexpr int kSteps = 4;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t ps = l2_evict_first();
    for (uint64_t col = warp; col < C; col += nwarps) {
        const uint64_t b = ptr[col], e = ptr[col + 1];
        uint32_t n = 0;
        for (uint64_t k0 = b; k0 < e; k0 += 32 * kSteps) {
            uint2 q[kSteps];
            bool f[kSteps];
#pragma unroll
            for (int u = 0; u < kSteps; ++u) {
                const uint64_t k = k0 + 32 * u + lane;
                q[u] = k < e ? ld_stream2(src + k, ps) : make_uint2(0u, 0u);
            }
#pragma unroll
            for (int u = 0; u < kSteps; ++u)
                f[u] = k0 + 32 * u + lane < e && ((keep[q[u].x >> 5] >> (q[u].x & 31)) & 1u);
#pragma unroll
            for (int u = 0; u < kSteps; ++u) {
                const unsigned m = __ballot_sync(MLEM_FULL_MASK, f[u]);
                if (f[u]) dst[b + n + __popc(m & below)] = q[u];
                n += __popc(m);
            }
        }
        if (lane == 0) len[col] = n;
    }
}

}  // namespace

cudaError_t csc_active_build(const SparseView& csr, const int32_t* sino, uint32_t Bp,
                             const SparseView& csc_vis, uint32_t* keep, uint2* dst, uint32_t* len,
                             cudaStream_t st) {
    if (!csr.order || Bp == 0) return cudaErrorInvalidValue;
    if (csr.n) {  // blocks of 256 threads: whole warps for the ballot
        const int grid = (int)std::min<uint64_t>((csr.n + 255) / 256, 148ull * 16);
        k_pos_keep<<<grid, 256, 0, st>>>(HasCount{csr.order, sino, Bp}, csr.n, keep);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (csc_vis.n == 0) return cudaSuccess;
    const int grid = (int)std::min<uint64_t>(((uint64_t)csc_vis.n + 7) / 8, 148ull * 16);
    k_csc_active<<<grid, 256, 0, st>>>(csc_vis.ptr, reinterpret_cast<const uint2*>(csc_vis.pairs),
                                       csc_vis.n, keep, dst, len);
    return cudaGetLastError();
}

size_t active_rows_tmp_bytes(uint32_t n) {
    size_t a = 0;
    cub::DeviceSelect::Flagged(nullptr, a, PosIt(0), FlagIt(PosIt(0), HasCount{nullptr, nullptr, 1}),
                               static_cast<uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                               (int)n);
    return std::max<size_t>(a, 16);
}

// Two passes: the select of the visiting positions whose rows have counts
// (flags computed on the fly from the order and the sinograms), then the
// gather of those rows and ranges; the list keeps the visiting order.
cudaError_t active_rows_build(const SparseView& csr, const int32_t* sino, uint32_t Bp,
                              void* tmp, size_t tmp_bytes, uint32_t* act_order,
                              ulonglong2* act_ranges, uint32_t* act_n, unsigned long long* act_z,
                              cudaStream_t st) {
    if (!csr.order || !csr.vrange || csr.n > 0x7fffffffu || Bp == 0) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(act_z, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(act_n, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess || csr.n == 0) return e;
    size_t tb = tmp_bytes;
    e = cub::DeviceSelect::Flagged(tmp, tb, PosIt(0), FlagIt(PosIt(0), HasCount{csr.order, sino, Bp}),
                                   act_order, act_n, (int)csr.n, st);
    if (e != cudaSuccess) return e;
    const int grid = (int)std::min<uint64_t>((csr.n + 255) / 256, 148ull * 16);
    k_active_gather<<<grid, 256, 0, st>>>(csr.order, csr.vrange, act_n, act_order, act_ranges, act_z);
    return cudaGetLastError();
}

cudaError_t row_ranges_build(const SparseView& csr, const uint32_t* order, ulonglong2* vrange,
                             cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    const int grid = (int)std::min<uint64_t>((csr.n + 255) / 256, 148ull * 16);
    k_row_ranges<<<grid, 256, 0, st>>>(csr, order, vrange);
    return cudaGetLastError();
}

cudaError_t row_order_build(const SparseView& csr, uint32_t C, uint32_t* order, cudaStream_t st) {
    const uint64_t n = csr.n;
    if (n == 0) return cudaSuccess;
    int bits = 1;
    while (bits < 32 && (1ull << bits) < (uint64_t)C) ++bits;
    const int end_bit = std::min(64, 2 * bits);
    uint64_t *key = nullptr, *key_sorted = nullptr;
    uint32_t* idx = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = cudaMalloc(&key, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&key_sorted, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&idx, n * 4);
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key_sorted, idx, order,
                                            (int64_t)n, 0, end_bit, st);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 256));
    if (e == cudaSuccess) {
        const int grid = (int)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
        k_row_keys<<<grid, 256, 0, st>>>(csr, key, idx);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key_sorted, idx, order,
                                            (int64_t)n, 0, end_bit, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) cudaGetLastError();
    cudaFree(key);
    cudaFree(key_sorted);
    cudaFree(idx);
    cudaFree(tmp);
    return e;
}

}  // namespace mlem
