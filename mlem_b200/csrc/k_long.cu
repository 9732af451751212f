// k_long.cu -- rows too long for one warp: the nnz split of the one-pass method.
//
// The one-pass kernels give a row to one warp (or lane group).  A skewed
// matrix with a few rows of 1e4..1e6 elements then waits for the warps that
// walk those rows alone.  Rows longer than kLongRowElems are therefore left
// out of the one-pass launch (the view's long_len makes them empty there) and
// cut into segments of at most kLongSegElems elements, which warps take in a
// grid-stride walk:
//   k_long_dot     -- each segment's partial forward projection, added into
//                     the row's sum f_long[slot][frame] by float atomics;
//   k_long_scatter -- after it, each segment's elements scatter value x
//                     calcCorrel(count, f) into the update, like a one-pass row.
// A long row's forward sum is thus a sum of segment partials in the order the
// atomics land: like the scatter, within float rounding of the sequential
// sum of calcFwProj (mlem_seq/seqcsr4mlem.cpp:76-90).
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "row_dev.cuh"

namespace mlem {

namespace {

constexpr int kLongThreads = 256;

template <int BT>
__global__ void __launch_bounds__(kLongThreads) k_long_dot(const uint2* __restrict__ el,
                                                           const LongSeg* __restrict__ segs,
                                                           uint32_t n_seg,
                                                           const float* __restrict__ x, uint32_t B,
                                                           float* __restrict__ f_long) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL, EPS = 32 / FL;
    constexpr int kDepth = VW == 4 ? 4 : 8;
    const int lane = threadIdx.x & 31, slot = lane / FL, sub = lane % FL;
    const uint64_t ph = l2_evict_last();
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_seg; w += nw) {
        const LongSeg sg = segs[w];
        for (uint32_t f0 = 0; f0 < B; f0 += BT) {
            const uint32_t off = f0 + sub * VW;
            float acc[VW];
#pragma unroll
            for (int i = 0; i < VW; ++i) acc[i] = 0.0f;
            for (uint64_t k0 = sg.b + slot; k0 < sg.e; k0 += (uint64_t)kDepth * EPS) {
                uint2 q[kDepth];
                float xv[kDepth][VW];
#pragma unroll
                for (int t = 0; t < kDepth; ++t) {
                    const uint64_t k = k0 + (uint64_t)t * EPS;
                    q[t] = k < sg.e ? el[k] : make_uint2(0u, 0u);
                }
#pragma unroll
                for (int t = 0; t < kDepth; ++t) ld_vec<VW>(x + off + (size_t)q[t].x * B, xv[t], ph);
#pragma unroll
                for (int t = 0; t < kDepth; ++t) {
                    const float v = __uint_as_float(q[t].y);  // 0 beyond the segment
#pragma unroll
                    for (int i = 0; i < VW; ++i) acc[i] = fmaf(v, xv[t][i], acc[i]);
                }
            }
            slot_allreduce<32, BT>(acc);
            if (slot == 0) {
#pragma unroll
                for (int i = 0; i < VW; ++i) atomicAdd(f_long + (size_t)sg.slot * B + off + i, acc[i]);
            }
        }
    }
}

template <int BT>
__global__ void __launch_bounds__(kLongThreads) k_long_scatter(const uint2* __restrict__ el,
                                                               const LongSeg* __restrict__ segs,
                                                               uint32_t n_seg,
                                                               const int32_t* __restrict__ sino,
                                                               const float* __restrict__ f_long,
                                                               uint32_t B, float* __restrict__ u) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL, EPS = 32 / FL;
    const int lane = threadIdx.x & 31, slot = lane / FL, sub = lane % FL;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_seg; w += nw) {
        const LongSeg sg = segs[w];
        for (uint32_t f0 = 0; f0 < B; f0 += BT) {
            const uint32_t off = f0 + sub * VW;
            int32_t s[VW];
            ld_counts<VW>(sino + (size_t)sg.row * B + off, s);
            float cv[VW];
            bool any = false;
#pragma unroll
            for (int i = 0; i < VW; ++i) {
                cv[i] = correl_of(s[i], f_long[(size_t)sg.slot * B + off + i]);
                any |= cv[i] != 0.0f;
            }
            if (!any) continue;  // no shuffles below: lanes may skip on their own
            for (uint64_t k = sg.b + slot; k < sg.e; k += EPS) {
                const uint2 q = el[k];
                red_vec<VW>(u + off + (size_t)q.x * B, __uint_as_float(q.y), cv);
            }
        }
    }
}

template <int BT>
cudaError_t launch_long(const SparseView& csr, const LongSeg* segs, uint32_t n_seg, const float* x,
                        uint32_t B, const int32_t* sino, float* f_long, float* u, int grid,
                        cudaStream_t st) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    k_long_dot<BT><<<grid, kLongThreads, 0, st>>>(el, segs, n_seg, x, B, f_long);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_long_scatter<BT><<<grid, kLongThreads, 0, st>>>(el, segs, n_seg, sino, f_long, B, u);
    return cudaGetLastError();
}

}  // namespace

cudaError_t long_rows_pass(const SparseView& csr, const LongSeg* segs, uint32_t n_seg,
                           uint32_t n_long, const float* x, uint32_t B, int frame_tile,
                           const int32_t* sino, float* f_long, float* u, int sm_count,
                           cudaStream_t st) {
    if (n_seg == 0) return cudaSuccess;
    if (B % (uint32_t)frame_tile) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(f_long, 0, (size_t)n_long * B * sizeof(float), st);
    if (e != cudaSuccess) return e;
    const uint64_t warps = n_seg;
    const int grid = (int)std::max<uint64_t>(
        1, std::min<uint64_t>((warps * 32 + kLongThreads - 1) / kLongThreads, (uint64_t)sm_count * 8));
    switch (frame_tile) {
        case 1: return launch_long<1>(csr, segs, n_seg, x, B, sino, f_long, u, grid, st);
        case 2: return launch_long<2>(csr, segs, n_seg, x, B, sino, f_long, u, grid, st);
        case 4: return launch_long<4>(csr, segs, n_seg, x, B, sino, f_long, u, grid, st);
        case 8: return launch_long<8>(csr, segs, n_seg, x, B, sino, f_long, u, grid, st);
        case 16: return launch_long<16>(csr, segs, n_seg, x, B, sino, f_long, u, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mlem
