// k_batch.cu -- one kernel per iteration for reconstructions over several
// matrices of uneven size (different scanners, different frame counts).
//
// Each matrix keeps its own context (CSR, image, sinograms, update vector).
// Two schedules run the one-pass per-row work (fused_row_range, row_dev.cuh)
// over the rows of all matrices in one launch, so a small matrix fills the
// tail of a large one instead of running in a launch of its own:
//   items       -- the rows are cut into work items of about equal cost
//                  (rows x elements per row x frames) that a persistent grid
//                  pulls from a global counter, heaviest first;
//   interleaved -- one virtual row space over all matrices, walked in
//                  grid-stride order.
//
// BT is one template parameter for the whole batch: dispatching several tile
// widths inside one kernel makes the compiler allocate their registers side
// by side (72-80 registers for one width, 167 for five), which would halve
// the resident warps of a latency-bound gather kernel.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "row_dev.cuh"
#include "staged_dev.cuh"

namespace mlem {

namespace {

constexpr int kBatchThreads = 256;

template <int BT, bool SORTED>
__global__ void __launch_bounds__(kBatchThreads, 4) k_batch_fused(const BatchTable t,
                                                                   const BatchItem* __restrict__ items,
                                                                   uint32_t n_items,
                                                                   unsigned int* __restrict__ counter) {
    __shared__ BatchItem s_item;
    const uint64_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t it = atomicAdd(counter, 1u);
            s_item = it < n_items ? items[it] : BatchItem{0u, 0u, 0u, 1u};
        }
        __syncthreads();
        const BatchItem item = s_item;
        __syncthreads();                 // s_item is rewritten by the next grab
        if (item.pad) return;            // block-uniform: no items left
        const BatchMat& m = t.mats[item.mat];
        const uint32_t Bp = m.Bp;
#pragma unroll 1
        for (uint32_t f0 = 0; f0 < Bp; f0 += BT)
            fused_row_range<32, BT, SORTED>(m.csr, m.x, Bp, f0, m.sino, m.u, item.row0, item.row1,
                                            warp, nwarps);
    }
}

// Items schedule with the staged row walk (staged_dev.cuh): the warps of a
// CTA pipeline their rows of the item through shared-memory stages.  Sorted
// visiting order only (the walk reads csr.vrange / csr.order).
template <int BT>
__global__ void __launch_bounds__(kBatchThreads, 4) k_batch_staged(const BatchTable t,
                                                                    const BatchItem* __restrict__ items,
                                                                    uint32_t n_items,
                                                                    unsigned int* __restrict__ counter) {
    extern __shared__ uint4 s_stage[];
    __shared__ BatchItem s_item;
    const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint2* stages = reinterpret_cast<const uint2*>(s_stage) + (size_t)warp * kStages * kStageCap;
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(stages);
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t it = atomicAdd(counter, 1u);
            s_item = it < n_items ? items[it] : BatchItem{0u, 0u, 0u, 1u};
        }
        __syncthreads();
        const BatchItem item = s_item;
        __syncthreads();                 // s_item is rewritten by the next grab
        if (item.pad) return;            // block-uniform: no items left
        const BatchMat& m = t.mats[item.mat];
        const uint32_t Bp = m.Bp;
#pragma unroll 1
        for (uint32_t f0 = 0; f0 < Bp; f0 += BT)
            staged_walk<BT, kStages>(m.csr, m.x, Bp, f0, m.sino, m.u, item.row0 + warp, item.row1,
                                     nwarps, stages, sa);
    }
}

template <int BT>
cudaError_t launch_batch_staged(const BatchTable& t, const BatchItem* items, uint32_t n_items,
                                unsigned int* counter, int grid, cudaStream_t st) {
    const size_t smem = staged_smem_bytes(kBatchThreads);
    cudaError_t e = cudaFuncSetAttribute(k_batch_staged<BT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_batch_staged<BT><<<grid, kBatchThreads, smem, st>>>(t, items, n_items, counter);
    return cudaGetLastError();
}

// Interleaved schedule: the rows of all matrices form one virtual row space
// (matrix i owns [row_base[i], row_base[i+1])), and global warp w takes
// virtual rows w, w + W, w + 2W, ... -- the grid-stride order of k_fused_row,
// so at any moment the whole grid works on one window of neighbouring rows,
// and a warp that finishes one matrix's rows goes straight on to the next
// matrix's.  Each row does all its frame tiles back to back.  The table is a
// kernel parameter: it lives in the constant bank like k_fused_row's
// arguments instead of taking registers.
template <int BT, bool SORTED>
__global__ void __launch_bounds__(kBatchThreads, 4) k_batch_interleaved(const BatchTable t) {
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t total = t.row_base[t.n];
    uint32_t mi = 0;
    for (; v < total; v += nw) {
        while (v >= t.row_base[mi + 1]) ++mi;  // warp-uniform, monotone
        const uint64_t r = v - t.row_base[mi];
        const uint32_t Bp = t.mats[mi].Bp;
#pragma unroll 1
        for (uint32_t f0 = 0; f0 < Bp; f0 += BT)
            fused_row_range<32, BT, SORTED>(t.mats[mi].csr, t.mats[mi].x, Bp, f0, t.mats[mi].sino,
                                    t.mats[mi].u, r, r + 1, 0, 1);
    }
}

// One matrix in dynamically scheduled chunks of consecutive visiting
// positions (the items schedule with uniform items and no item list).
template <int BT>
__global__ void __launch_bounds__(1024, 1) k_fused_chunked(SparseView csr,
                                                                     const float* __restrict__ x,
                                                                     uint32_t B,
                                                                     const int32_t* __restrict__ sino,
                                                                     float* __restrict__ u,
                                                                     uint32_t chunk,
                                                                     unsigned int* __restrict__ counter) {
    __shared__ uint32_t s_chunk;
    const uint64_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(counter, 1u);
        __syncthreads();
        const uint64_t ci = s_chunk;
        __syncthreads();  // s_chunk is rewritten by the next grab
        // re-read per chunk (a cached load) rather than held in a register
        const uint64_t n = visit_count(csr);
        if (ci >= (n + chunk - 1) / chunk) return;  // block-uniform
        const uint64_t r0 = ci * chunk, r1 = r0 + chunk < n ? r0 + chunk : n;
#pragma unroll 1
        for (uint32_t f0 = 0; f0 < B; f0 += BT)
            fused_row_range<32, BT, true>(csr, x, B, f0, sino, u, r0, r1, warp, nwarps);
    }
}

}  // namespace

cudaError_t fused_chunked(const SparseView& csr, const float* x, uint32_t B, int frame_tile,
                          const int32_t* sino, float* u, uint32_t chunk_rows, int ctas_per_sm,
                          unsigned int* counter, int sm_count, cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    if (chunk_rows == 0 || ((uint64_t)csr.n + chunk_rows - 1) / chunk_rows > 0xffffffffull)
        return cudaErrorInvalidValue;
    if (ctas_per_sm != 1 && ctas_per_sm != 2 && ctas_per_sm != 4) return cudaErrorInvalidValue;
    if (!csr.order || !csr.vrange) return cudaErrorInvalidValue;  // a sorted visit
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    // the resident CTAs: 64 registers x 1024 threads per SM, in 1, 2 or 4 CTAs
    const int grid = std::max(1, sm_count * ctas_per_sm), threads = 1024 / ctas_per_sm;
    switch (frame_tile) {
        case 1: k_fused_chunked<1><<<grid, threads, 0, st>>>(csr, x, B, sino, u, chunk_rows, counter); break;
        case 2: k_fused_chunked<2><<<grid, threads, 0, st>>>(csr, x, B, sino, u, chunk_rows, counter); break;
        case 4: k_fused_chunked<4><<<grid, threads, 0, st>>>(csr, x, B, sino, u, chunk_rows, counter); break;
        case 8: k_fused_chunked<8><<<grid, threads, 0, st>>>(csr, x, B, sino, u, chunk_rows, counter); break;
        case 16: k_fused_chunked<16><<<grid, threads, 0, st>>>(csr, x, B, sino, u, chunk_rows, counter); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

#define MLEM_BATCH_TILES(KERNEL, ...)                                                \
    switch (frame_tile) {                                                            \
        case 1: (sorted ? KERNEL<1, true> : KERNEL<1, false>)<<<__VA_ARGS__; break;  \
        case 2: (sorted ? KERNEL<2, true> : KERNEL<2, false>)<<<__VA_ARGS__; break;  \
        case 4: (sorted ? KERNEL<4, true> : KERNEL<4, false>)<<<__VA_ARGS__; break;  \
        case 8: (sorted ? KERNEL<8, true> : KERNEL<8, false>)<<<__VA_ARGS__; break;  \
        case 16: (sorted ? KERNEL<16, true> : KERNEL<16, false>)<<<__VA_ARGS__; break; \
        default: return cudaErrorInvalidValue;                                       \
    }

cudaError_t batch_interleaved(const BatchTable& t, int frame_tile, bool sorted, int sm_count,
                              int blocks_per_sm, cudaStream_t st) {
    if (t.n == 0 || t.n > kBatchTableMax) return cudaErrorInvalidValue;
    const int grid = std::max(1, sm_count * blocks_per_sm);
    MLEM_BATCH_TILES(k_batch_interleaved, grid, kBatchThreads, 0, st>>>(t))
    return cudaGetLastError();
}

cudaError_t batch_fused(const BatchTable& t, const BatchItem* items, uint32_t n_items,
                        unsigned int* counter, int frame_tile, bool sorted, int sm_count,
                        int blocks_per_sm, cudaStream_t st) {
    if (n_items == 0) return cudaSuccess;
    if (t.n == 0 || t.n > kBatchTableMax) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    const int grid = std::max(1, std::min<int>((int)std::min<uint32_t>(n_items, 1u << 30),
                                               sm_count * blocks_per_sm));
    MLEM_BATCH_TILES(k_batch_fused, grid, kBatchThreads, 0, st>>>(t, items, n_items, counter))
    return cudaGetLastError();
}

cudaError_t batch_staged(const BatchTable& t, const BatchItem* items, uint32_t n_items,
                         unsigned int* counter, int frame_tile, int sm_count, int blocks_per_sm,
                         cudaStream_t st) {
    if (n_items == 0) return cudaSuccess;
    if (t.n == 0 || t.n > kBatchTableMax) return cudaErrorInvalidValue;
    for (uint32_t i = 0; i < t.n; ++i)
        if (!t.mats[i].csr.order || !t.mats[i].csr.vrange) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    // at most 4 resident CTAs: each holds 32 KiB of stages
    const int grid = std::max(1, std::min<int>((int)std::min<uint32_t>(n_items, 1u << 30),
                                               sm_count * std::min(blocks_per_sm, 4)));
    switch (frame_tile) {
        case 1: return launch_batch_staged<1>(t, items, n_items, counter, grid, st);
        case 2: return launch_batch_staged<2>(t, items, n_items, counter, grid, st);
        case 4: return launch_batch_staged<4>(t, items, n_items, counter, grid, st);
        case 8: return launch_batch_staged<8>(t, items, n_items, counter, grid, st);
        case 16: return launch_batch_staged<16>(t, items, n_items, counter, grid, st);
        default: return cudaErrorInvalidValue;
    }
}
#undef MLEM_BATCH_TILES

}  // namespace mlem
