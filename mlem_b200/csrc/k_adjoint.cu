// k_adjoint.cu -- one-pass kernels of the differentiable MLEM's backward pass.
//
// The unrolled MLEM of mlem_b200/torch_ext.py recomputes, for every iteration
// k of its backward pass, the projection f = A x_k, the update ratio
// A^T calcCorrel(s, A x_k), and then propagates the adjoint du through
// calcCorrel and both projections: A^T df with df = -(A du) s / f^2 where the
// row has a count and a nonzero projection.  Done with separate projections
// that is four passes over the matrix; these two kernels do it in two:
//   RATIO  : one pass computes A x, calcCorrel and the scatter of the ratio's
//            numerator (as the one-pass iteration) and also stores the row
//            sums f = A x;
//   ADJOINT: one pass computes A du per row, df from it and the stored f, and
//            scatters A^T df.
// A row whose count is zero has calcCorrel 0 and df 0 whatever its
// projection, so both walks skip it before loading any element (RATIO stores
// 0 as its f, which ADJOINT then also treats as "no gradient").  One frame,
// a warp per row, the sorted rows in chunks taken from a counter (or file
// order without a row order); the scatter's float atomics make the summation
// order vary from run to run.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "row_dev.cuh"

namespace mlem {

namespace {

template <int OP, bool SORTED>
__device__ __forceinline__ void adjoint_row_range(const SparseView& csr, const float* __restrict__ x,
                                                  const int32_t* __restrict__ sino,
                                                  float* __restrict__ rows, float* __restrict__ u,
                                                  uint64_t r_begin, uint64_t r_end, uint64_t warp,
                                                  uint64_t nwarps) {
    constexpr int kBatch = batch_depth<32>();
    const int lane = threadIdx.x & 31;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t v = r_begin + warp; v < r_end; v += nwarps) {
        uint64_t r, b, e;
        if constexpr (SORTED) {
            const ulonglong2 q = csr.vrange[v];
            r = csr.order[v];
            b = q.x;
            e = q.y;
        } else {
            r = v;
            b = csr.ptr[r];
            e = csr.ptr[r + 1];
        }
        const int32_t s = sino[r];
        if (s == 0) {  // calcCorrel 0 and no gradient: nothing to gather or scatter
            if (OP == kOpRatio && lane == 0) rows[r] = 0.0f;
            continue;
        }
        float acc[1];
        uint2 kept[kBatch];
        const bool in_regs = row_dot<32, 1, true>(el, b, e, lane, x, 1, 0, acc, ps, ph, kept);
        slot_allreduce<32, 1>(acc);
        float h;
        if constexpr (OP == kOpRatio) {
            h = correl_of(s, acc[0]);
            if (lane == 0) rows[r] = acc[0];
        } else {
            // d/df of calcCorrel(s, f) = s / f, applied to A du: -(A du) (s / f) / f
            const float f = rows[r];
            h = f != 0.0f ? -(acc[0] * (__int2float_rn(s) / f)) / f : 0.0f;
        }
        if (h == 0.0f) continue;
        if (in_regs) {
#pragma unroll
            for (int q = 0; q < kBatch; ++q)
                if (b + lane + (uint64_t)q * 32 < e) atomicAdd(u + kept[q].x, __uint_as_float(kept[q].y) * h);
        } else {
            for (uint64_t k = b + lane; k < e; k += 32) {
                const uint2 q = ld_keep2(el + k, ps);
                atomicAdd(u + q.x, __uint_as_float(q.y) * h);
            }
        }
    }
}

template <int OP, bool SORTED>
__global__ void __launch_bounds__(256) k_adjoint_chunked(SparseView csr, const float* __restrict__ x,
                                                         const int32_t* __restrict__ sino,
                                                         float* __restrict__ rows,
                                                         float* __restrict__ u, uint32_t chunk,
                                                         unsigned int* __restrict__ counter) {
    __shared__ uint32_t s_chunk;
    const uint64_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint64_t n = csr.n;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(counter, 1u);
        __syncthreads();
        const uint64_t ci = s_chunk;
        __syncthreads();  // s_chunk is rewritten by the next grab
        if (ci >= (n + chunk - 1) / chunk) return;  // block-uniform
        const uint64_t r0 = ci * chunk, r1 = r0 + chunk < n ? r0 + chunk : n;
        adjoint_row_range<OP, SORTED>(csr, x, sino, rows, u, r0, r1, warp, nwarps);
    }
}

}  // namespace

cudaError_t adjoint_pass(int op, const SparseView& csr, const float* x, const int32_t* sino,
                         float* rows, float* u, unsigned int* counter, int sm_count,
                         cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    if (op != kOpRatio && op != kOpAdjoint) return cudaErrorInvalidValue;
    const bool sorted = csr.order && csr.vrange;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    // 4 CTAs of 256 threads per SM; about 16 chunks per CTA, at least 32 rows each
    const int grid = std::max(1, sm_count * 4);
    const uint64_t chunk64 = std::max<uint64_t>(32, ((uint64_t)csr.n + (uint64_t)grid * 16 - 1) /
                                                        ((uint64_t)grid * 16));
    const uint32_t chunk = (uint32_t)std::min<uint64_t>(chunk64, 0xffffffffull);
    if (op == kOpRatio) {
        if (sorted) k_adjoint_chunked<kOpRatio, true><<<grid, 256, 0, st>>>(csr, x, sino, rows, u, chunk, counter);
        else k_adjoint_chunked<kOpRatio, false><<<grid, 256, 0, st>>>(csr, x, sino, rows, u, chunk, counter);
    } else {
        if (sorted) k_adjoint_chunked<kOpAdjoint, true><<<grid, 256, 0, st>>>(csr, x, sino, rows, u, chunk, counter);
        else k_adjoint_chunked<kOpAdjoint, false><<<grid, 256, 0, st>>>(csr, x, sino, rows, u, chunk, counter);
    }
    return cudaGetLastError();
}

}  // namespace mlem
