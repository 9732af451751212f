// k_staged.cu -- one-pass MLEM row kernel with the element stream staged
// through shared memory by asynchronous copies (MLEM_VISIT_SORTED_STAGED;
// the per-warp pipeline is staged_walk in staged_dev.cuh).
//
// Rows are visited in the sorted order (csr.order / csr.vrange), in chunks of
// neighbouring visiting positions that CTAs take from a counter, as in
// k_fused_chunked; within a chunk warp w takes positions w, w + W, ... (W the
// warps of the CTA), so the rays a CTA has in flight are near each other and
// share image lines in L1.
//
// Measured on the plain-full matrix (4,194,304 rows, 7.8e8 elements) against
// k_fused_chunked: 16 frames in one tile 10.1-10.2 vs 11.7 ms, 8-frame tiles
// 14.7 vs 15.8 ms, one frame 2.55 vs 2.46 ms and 4-frame tiles 4.6-4.8 vs
// 4.3-4.5 ms (the stages take L1 capacity from the image gathers, which is
// what a narrow row mostly waits on).  A third stage (two rows in flight) was
// slower at every width: 2.90 ms at one frame, 10.5 ms at sixteen.
#include <algorithm>

#include "staged_dev.cuh"

namespace mlem {

namespace {

constexpr int kStagedThreads = 256;

template <int BT>
__global__ void __launch_bounds__(kStagedThreads, 4) k_fused_staged(SparseView csr,
                                                                    const float* __restrict__ x,
                                                                    uint32_t B,
                                                                    const int32_t* __restrict__ sino,
                                                                    float* __restrict__ u,
                                                                    uint32_t chunk,
                                                                    unsigned int* __restrict__ counter) {
    extern __shared__ uint4 s_stage[];
    __shared__ uint32_t s_chunk;
    const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint2* stages = reinterpret_cast<const uint2*>(s_stage) + (size_t)warp * kStages * kStageCap;
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(stages);
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
            staged_walk<BT, kStages>(csr, x, B, f0, sino, u, r0 + warp, r1, nwarps, stages, sa);
    }
}

template <int BT>
cudaError_t launch_staged(const SparseView& csr, const float* x, uint32_t B, const int32_t* sino,
                          float* u, uint32_t chunk_rows, int grid, unsigned int* counter,
                          cudaStream_t st) {
    // the stages plus the static chunk slot may pass the 48 KiB default
    const size_t smem = staged_smem_bytes(kStagedThreads);
    cudaError_t e = cudaFuncSetAttribute(k_fused_staged<BT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_fused_staged<BT><<<grid, kStagedThreads, smem, st>>>(csr, x, B, sino, u, chunk_rows, counter);
    return cudaGetLastError();
}

}  // namespace

cudaError_t fused_staged(const SparseView& csr, const float* x, uint32_t B, int frame_tile,
                         const int32_t* sino, float* u, uint32_t chunk_rows, int ctas_per_sm,
                         unsigned int* counter, int sm_count, cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    if (chunk_rows == 0 || ((uint64_t)csr.n + chunk_rows - 1) / chunk_rows > 0xffffffffull)
        return cudaErrorInvalidValue;
    if (ctas_per_sm < 1 || ctas_per_sm > 4) return cudaErrorInvalidValue;
    if (!csr.order || !csr.vrange) return cudaErrorInvalidValue;  // a sorted visit
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    const int grid = std::max(1, sm_count * ctas_per_sm);
    switch (frame_tile) {
        case 1: return launch_staged<1>(csr, x, B, sino, u, chunk_rows, grid, counter, st);
        case 2: return launch_staged<2>(csr, x, B, sino, u, chunk_rows, grid, counter, st);
        case 4: return launch_staged<4>(csr, x, B, sino, u, chunk_rows, grid, counter, st);
        case 8: return launch_staged<8>(csr, x, B, sino, u, chunk_rows, grid, counter, st);
        case 16: return launch_staged<16>(csr, x, B, sino, u, chunk_rows, grid, counter, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mlem
