// k_project.cu -- the per-iteration MLEM kernels (sm_100a).
//
// Forward projection fused with calcCorrel, back projection over the CSC copy
// fused with calcUpdate, the atomic-scatter back projection, the one-pass
// per-row kernel, and the bit-exact variants.  Reference functions:
// calcFwProj/calcCorrel/calcBkProj/calcUpdate, mlem_seq/seqcsr4mlem.cpp:69-134.
//
// Work decomposition: G lanes (4..32) own one row (or column); a warp owns
// 32/G rows; warps stride over rows (grid = blocks_per_sm x SMs, persistent
// style).  Each lane reads whole 16-byte element pairs, so a warp issues
// fully coalesced 512-byte reads of the element stream.  A row that starts
// on an odd element shares its first pair with the previous row: the lane
// masks the element that is not its own.  Frames (B sinograms reconstructed
// together) are interleaved in the vectors, and a kernel instance processes a
// tile of BT frames per pass over the matrix, gathering BT contiguous floats
// per element with 16-byte loads.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace mlem {

namespace {

template <int BT>
__device__ __forceinline__ void gather(const float* __restrict__ p, float (&v)[BT], uint64_t pol) {
    if constexpr (BT % 4 == 0) {
#pragma unroll
        for (int i = 0; i < BT / 4; ++i) {
            float4 t = ld_hot4(reinterpret_cast<const float4*>(p) + i, pol);
            v[4 * i + 0] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < BT; ++i) v[i] = ld_hot(p + i, pol);
    }
}

template <int BT>
__device__ __forceinline__ void scatter_add(float* __restrict__ p, float w, const float (&c)[BT]) {
    if constexpr (BT % 4 == 0) {
#pragma unroll
        for (int i = 0; i < BT / 4; ++i)
            atomicAdd(reinterpret_cast<float4*>(p) + i,
                      make_float4(w * c[4 * i], w * c[4 * i + 1], w * c[4 * i + 2], w * c[4 * i + 3]));
    } else {
#pragma unroll
        for (int i = 0; i < BT; ++i) atomicAdd(p + i, w * c[i]);
    }
}

// acc += v * vec[idx][f0 .. f0+BT) for the two elements of pair q, masking
// elements outside [b, e).  k0 = global index of the pair's first element.
// With p in [b>>1, (e+1)>>1): k0 < e and k0 + 1 >= b always hold.
template <int BT>
__device__ __forceinline__ void accum_pair(const uint4& q, uint64_t k0, uint64_t b, uint64_t e,
                                           const float* __restrict__ vec, uint32_t B,
                                           uint32_t f0, float (&acc)[BT], uint64_t pol) {
    if (k0 >= b) {
        float xv[BT];
        gather<BT>(vec + (size_t)q.x * B + f0, xv, pol);
        const float v = __uint_as_float(q.y);
#pragma unroll
        for (int i = 0; i < BT; ++i) acc[i] = fmaf(v, xv[i], acc[i]);
    }
    if (k0 + 1 < e) {
        float xv[BT];
        gather<BT>(vec + (size_t)q.z * B + f0, xv, pol);
        const float v = __uint_as_float(q.w);
#pragma unroll
        for (int i = 0; i < BT; ++i) acc[i] = fmaf(v, xv[i], acc[i]);
    }
}

// Dot products of one row (or column) against BT frames of `vec`.
template <int G, int BT, bool KEEP>
__device__ __forceinline__ void row_dot(const uint4* __restrict__ pairs, uint64_t b, uint64_t e,
                                        int lane, const float* __restrict__ vec, uint32_t B,
                                        uint32_t f0, float (&acc)[BT], uint64_t ps,
                                        uint64_t ph) {
#pragma unroll
    for (int i = 0; i < BT; ++i) acc[i] = 0.0f;
    const uint64_t pend = (e + 1) >> 1;
    uint64_t p = (b >> 1) + lane;
    for (; p + 3 * G < pend; p += 4 * G) {
        uint4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            q[u] = KEEP ? ld_keep(pairs + p + u * G, ps) : ld_stream(pairs + p + u * G, ps);
#pragma unroll
        for (int u = 0; u < 4; ++u) accum_pair<BT>(q[u], 2 * (p + u * G), b, e, vec, B, f0, acc, ph);
    }
    for (; p < pend; p += G) {
        uint4 q = KEEP ? ld_keep(pairs + p, ps) : ld_stream(pairs + p, ps);
        accum_pair<BT>(q, 2 * p, b, e, vec, B, f0, acc, ph);
    }
}

// ---------------------------------------------------------------------------
// Forward projection (+ calcCorrel).
// ---------------------------------------------------------------------------
template <int G, int BT>
__global__ void __launch_bounds__(256) k_fwproj(SparseView csr, const float* __restrict__ x,
                                                uint32_t B, uint32_t f0,
                                                const int32_t* __restrict__ sino,
                                                float* __restrict__ c, float* __restrict__ y) {
    constexpr int RPW = 32 / G;
    constexpr int SPAN = G / BT;
    const int lw = threadIdx.x & 31;
    const int lane = lw & (G - 1);
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    for (uint64_t base = warp * RPW; base < csr.n; base += nwarps * RPW) {
        const uint64_t r = base + lw / G;
        const bool active = r < csr.n;
        uint64_t b = 0, e = 0;
        if (active) { b = csr.ptr[r]; e = csr.ptr[r + 1]; }
        float acc[BT];
        row_dot<G, BT, false>(csr.pairs, b, e, lane, x, B, f0, acc, ps, ph);
        group_reduce_scatter<G, BT>(acc, lane);
        if (active && (lane % SPAN) == 0) {
            const uint64_t idx = r * B + f0 + lane / SPAN;
            if (y) y[idx] = acc[0];
            if (c) c[idx] = correl_of(sino[idx], acc[0]);
        }
    }
}

// ---------------------------------------------------------------------------
// Back projection over the CSC copy (+ calcUpdate).
// ---------------------------------------------------------------------------
template <int G, int BT>
__global__ void __launch_bounds__(256) k_bkproj_csc(SparseView csc, const float* __restrict__ c,
                                                    uint32_t B, uint32_t f0,
                                                    const float* __restrict__ norm,
                                                    float* __restrict__ x, float* __restrict__ u) {
    constexpr int RPW = 32 / G;
    constexpr int SPAN = G / BT;
    const int lw = threadIdx.x & 31;
    const int lane = lw & (G - 1);
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    for (uint64_t base = warp * RPW; base < csc.n; base += nwarps * RPW) {
        const uint64_t col = base + lw / G;
        const bool active = col < csc.n;
        uint64_t b = 0, e = 0;
        if (active) { b = csc.ptr[col]; e = csc.ptr[col + 1]; }
        float acc[BT];
        row_dot<G, BT, false>(csc.pairs, b, e, lane, c, B, f0, acc, ps, ph);
        group_reduce_scatter<G, BT>(acc, lane);
        if (active && (lane % SPAN) == 0) {
            const uint64_t idx = col * B + f0 + lane / SPAN;
            if (norm) x[idx] *= update_factor(acc[0], norm[col]);
            else u[idx] = acc[0];
        }
    }
}

// ---------------------------------------------------------------------------
// Back projection by atomic scatter over the CSR (the reference GPU drivers'
// approach, mlem_cuda/helper_files/cudaKernels.cu:155-178, kept for
// comparison and chosen by the autotuner where it wins).
// ---------------------------------------------------------------------------
template <int G, int BT>
__global__ void __launch_bounds__(256) k_bkproj_scatter(SparseView csr,
                                                        const float* __restrict__ c, uint32_t B,
                                                        uint32_t f0, float* __restrict__ u) {
    constexpr int RPW = 32 / G;
    const int lw = threadIdx.x & 31;
    const int lane = lw & (G - 1);
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    for (uint64_t base = warp * RPW; base < csr.n; base += nwarps * RPW) {
        const uint64_t r = base + lw / G;
        if (r >= csr.n) continue;  // no shuffles in this kernel
        const uint64_t b = csr.ptr[r], e = csr.ptr[r + 1];
        float cv[BT];
        gather<BT>(c + r * B + f0, cv, ph);
        bool any = false;
#pragma unroll
        for (int i = 0; i < BT; ++i) any |= (cv[i] != 0.0f);
        if (!any) continue;  // adding +0 changes no update entry
        const uint64_t pend = (e + 1) >> 1;
        for (uint64_t p = (b >> 1) + lane; p < pend; p += G) {
            const uint4 q = ld_stream(csr.pairs + p, ps);
            if (2 * p >= b) scatter_add<BT>(u + (size_t)q.x * B + f0, __uint_as_float(q.y), cv);
            if (2 * p + 1 < e) scatter_add<BT>(u + (size_t)q.z * B + f0, __uint_as_float(q.w), cv);
        }
    }
}

// ---------------------------------------------------------------------------
// One pass per row: forward projection, calcCorrel, and the back-projection
// scatter of the same row while its elements are still on chip (the row is
// re-read from L1).  The matrix streams from HBM once per iteration.
// ---------------------------------------------------------------------------
template <int G, int BT>
__global__ void __launch_bounds__(256) k_fused_row(SparseView csr, const float* __restrict__ x,
                                                   uint32_t B, uint32_t f0,
                                                   const int32_t* __restrict__ sino,
                                                   float* __restrict__ u) {
    constexpr int RPW = 32 / G;
    constexpr int SPAN = G / BT;
    const int lw = threadIdx.x & 31;
    const int lane = lw & (G - 1);
    const int gbase = lw & ~(G - 1);
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    for (uint64_t base = warp * RPW; base < csr.n; base += nwarps * RPW) {
        const uint64_t r = base + lw / G;
        const bool active = r < csr.n;
        uint64_t b = 0, e = 0;
        if (active) { b = csr.ptr[r]; e = csr.ptr[r + 1]; }
        float acc[BT];
        row_dot<G, BT, true>(csr.pairs, b, e, lane, x, B, f0, acc, ps, ph);
        group_reduce_scatter<G, BT>(acc, lane);
        float mine = 0.0f;
        if (active && (lane % SPAN) == 0) mine = correl_of(sino[r * B + f0 + lane / SPAN], acc[0]);
        float cv[BT];
        bool any = false;
#pragma unroll
        for (int i = 0; i < BT; ++i) {
            cv[i] = __shfl_sync(MLEM_FULL_MASK, mine, gbase + i * SPAN);
            any |= (cv[i] != 0.0f);
        }
        if (!any) continue;
        const uint64_t pend = (e + 1) >> 1;
        for (uint64_t p = (b >> 1) + lane; p < pend; p += G) {
            const uint4 q = ld_keep(csr.pairs + p, ps);
            if (2 * p >= b) scatter_add<BT>(u + (size_t)q.x * B + f0, __uint_as_float(q.y), cv);
            if (2 * p + 1 < e) scatter_add<BT>(u + (size_t)q.z * B + f0, __uint_as_float(q.w), cv);
        }
    }
}

template <bool ONE_FRAME>
__global__ void k_apply_update(float* __restrict__ x, float* __restrict__ u,
                               const float* __restrict__ norm, uint64_t n, uint32_t B,
                               bool zero_u) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t col = ONE_FRAME ? i : i / B;
        x[i] *= update_factor(u[i], norm[col]);
        if (zero_u) u[i] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Bit-exact kernels.  One warp per row (column); the 32 lanes load and
// multiply 32 consecutive elements in parallel (__fmul_rn: no contraction),
// then every lane adds the 32 products into its running sum in element order
// (__fadd_rn), which is exactly the sequential float order of the reference
// loops.  Used for calcColumnSums always, and for the whole iteration when a
// context is created with MLEM_FLAG_EXACT.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fwproj_exact(SparseView csr, const float* __restrict__ x,
                                                      uint32_t B, const int32_t* __restrict__ sino,
                                                      float* __restrict__ c,
                                                      float* __restrict__ y) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < csr.n; r += nwarps) {
        const uint64_t b = csr.ptr[r], e = csr.ptr[r + 1];
        for (uint32_t f = 0; f < B; ++f) {
            float s = 0.0f;
            for (uint64_t base = b; base < e; base += 32) {
                float prod = 0.0f;
                if (base + lane < e) {
                    const uint2 q = el[base + lane];
                    prod = __fmul_rn(__uint_as_float(q.y), x[(size_t)q.x * B + f]);
                }
                const int cnt = (int)min((uint64_t)32, e - base);
                for (int j = 0; j < cnt; ++j) s = __fadd_rn(s, __shfl_sync(MLEM_FULL_MASK, prod, j));
            }
            if (lane == 0) {
                if (y) y[r * B + f] = s;
                if (c) c[r * B + f] = correl_of(sino[r * B + f], s);
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_bkproj_exact(SparseView csc, const float* __restrict__ c,
                                                      uint32_t B, const float* __restrict__ norm,
                                                      float* __restrict__ x, float* __restrict__ u) {
    const uint2* el = reinterpret_cast<const uint2*>(csc.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t col = warp; col < csc.n; col += nwarps) {
        const uint64_t b = csc.ptr[col], e = csc.ptr[col + 1];
        for (uint32_t f = 0; f < B; ++f) {
            float s = 0.0f;
            for (uint64_t base = b; base < e; base += 32) {
                float prod = 0.0f;
                if (base + lane < e) {
                    const uint2 q = el[base + lane];
                    prod = __fmul_rn(__uint_as_float(q.y), c[(size_t)q.x * B + f]);
                }
                const int cnt = (int)min((uint64_t)32, e - base);
                for (int j = 0; j < cnt; ++j) s = __fadd_rn(s, __shfl_sync(MLEM_FULL_MASK, prod, j));
            }
            if (lane == 0) {
                if (norm) x[col * B + f] = __fmul_rn(x[col * B + f], update_factor(s, norm[col]));
                else u[col * B + f] = s;
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_colsum_exact(SparseView csc, float* __restrict__ norm) {
    const uint2* el = reinterpret_cast<const uint2*>(csc.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t col = warp; col < csc.n; col += nwarps) {
        const uint64_t b = csc.ptr[col], e = csc.ptr[col + 1];
        float s = 0.0f;
        for (uint64_t base = b; base < e; base += 32) {
            float v = 0.0f;
            if (base + lane < e) v = __uint_as_float(el[base + lane].y);
            const int cnt = (int)min((uint64_t)32, e - base);
            for (int j = 0; j < cnt; ++j) s = __fadd_rn(s, __shfl_sync(MLEM_FULL_MASK, v, j));
        }
        if (lane == 0) norm[col] = s;
    }
}

__global__ void k_colsum_atomic(SparseView csr, float* __restrict__ norm) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < csr.nnz;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint2 q = el[k];
        atomicAdd(norm + q.x, __uint_as_float(q.y));
    }
}

inline int grid_for(const LaunchCfg& cfg) { return cfg.blocks_per_sm * cfg.sm_count; }

// (G, BT) dispatch.  Only BT <= G instances exist.
template <template <int, int> class K, typename... Args>
cudaError_t dispatch(const LaunchCfg& cfg, cudaStream_t st, Args... args);

#define MLEM_KERNEL_FUNCTOR(NAME, KERNEL)                                              \
    template <int G, int BT>                                                           \
    struct NAME {                                                                      \
        template <typename... A>                                                       \
        static void run(int grid, cudaStream_t st, A... a) {                           \
            KERNEL<G, BT><<<grid, 256, 0, st>>>(a...);                                 \
        }                                                                              \
    };
MLEM_KERNEL_FUNCTOR(FwprojK, k_fwproj)
MLEM_KERNEL_FUNCTOR(BkprojCscK, k_bkproj_csc)
MLEM_KERNEL_FUNCTOR(ScatterK, k_bkproj_scatter)
MLEM_KERNEL_FUNCTOR(FusedK, k_fused_row)
#undef MLEM_KERNEL_FUNCTOR

template <template <int, int> class K, int G, typename... Args>
cudaError_t dispatch_bt(const LaunchCfg& cfg, cudaStream_t st, Args... args) {
    const int grid = grid_for(cfg);
    switch (cfg.frame_tile) {
        case 1: K<G, 1>::run(grid, st, args...); break;
        case 2: if constexpr (G >= 2) { K<G, 2>::run(grid, st, args...); break; } else return cudaErrorInvalidValue;
        case 4: if constexpr (G >= 4) { K<G, 4>::run(grid, st, args...); break; } else return cudaErrorInvalidValue;
        case 8: if constexpr (G >= 8) { K<G, 8>::run(grid, st, args...); break; } else return cudaErrorInvalidValue;
        case 16: if constexpr (G >= 16) { K<G, 16>::run(grid, st, args...); break; } else return cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <template <int, int> class K, typename... Args>
cudaError_t dispatch(const LaunchCfg& cfg, cudaStream_t st, Args... args) {
    switch (cfg.group) {
        case 4: return dispatch_bt<K, 4>(cfg, st, args...);
        case 8: return dispatch_bt<K, 8>(cfg, st, args...);
        case 16: return dispatch_bt<K, 16>(cfg, st, args...);
        case 32: return dispatch_bt<K, 32>(cfg, st, args...);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

bool cfg_valid(const LaunchCfg& c) {
    const bool g = c.group == 4 || c.group == 8 || c.group == 16 || c.group == 32;
    const bool t = c.frame_tile == 1 || c.frame_tile == 2 || c.frame_tile == 4 ||
                   c.frame_tile == 8 || c.frame_tile == 16;
    return g && t && c.frame_tile <= c.group && c.blocks_per_sm >= 1 && c.blocks_per_sm <= 8 &&
           c.sm_count >= 1;
}

cudaError_t fwproj(const SparseView& csr, const float* x, uint32_t B, uint32_t f0,
                   const int32_t* sino, float* c, float* y, const LaunchCfg& cfg,
                   cudaStream_t st) {
    if (!cfg_valid(cfg) || (B % cfg.frame_tile) || (f0 % cfg.frame_tile)) return cudaErrorInvalidValue;
    if (csr.n == 0) return cudaSuccess;
    return dispatch<FwprojK>(cfg, st, csr, x, B, f0, sino, c, y);
}

cudaError_t bkproj_csc(const SparseView& csc, const float* c, uint32_t B, uint32_t f0,
                       const float* norm, float* x, float* u, const LaunchCfg& cfg,
                       cudaStream_t st) {
    if (!cfg_valid(cfg) || (B % cfg.frame_tile) || (f0 % cfg.frame_tile)) return cudaErrorInvalidValue;
    if (csc.n == 0) return cudaSuccess;
    return dispatch<BkprojCscK>(cfg, st, csc, c, B, f0, norm, x, u);
}

cudaError_t bkproj_scatter(const SparseView& csr, const float* c, uint32_t B, uint32_t f0,
                           float* u, const LaunchCfg& cfg, cudaStream_t st) {
    if (!cfg_valid(cfg) || (B % cfg.frame_tile) || (f0 % cfg.frame_tile)) return cudaErrorInvalidValue;
    if (csr.n == 0) return cudaSuccess;
    return dispatch<ScatterK>(cfg, st, csr, c, B, f0, u);
}

cudaError_t fused_row(const SparseView& csr, const float* x, uint32_t B, uint32_t f0,
                      const int32_t* sino, float* u, const LaunchCfg& cfg, cudaStream_t st) {
    if (!cfg_valid(cfg) || (B % cfg.frame_tile) || (f0 % cfg.frame_tile)) return cudaErrorInvalidValue;
    if (csr.n == 0) return cudaSuccess;
    return dispatch<FusedK>(cfg, st, csr, x, B, f0, sino, u);
}

cudaError_t apply_update(float* x, float* u, const float* norm, uint32_t C, uint32_t B,
                         bool zero_u, cudaStream_t st) {
    const uint64_t n = (uint64_t)C * B;
    if (n == 0) return cudaSuccess;
    const int grid = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)kB200SMs * 16);
    if (B == 1) k_apply_update<true><<<grid, 256, 0, st>>>(x, u, norm, n, B, zero_u);
    else k_apply_update<false><<<grid, 256, 0, st>>>(x, u, norm, n, B, zero_u);
    return cudaGetLastError();
}

cudaError_t fwproj_exact(const SparseView& csr, const float* x, uint32_t B, const int32_t* sino,
                         float* c, float* y, cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    k_fwproj_exact<<<kB200SMs * 8, 256, 0, st>>>(csr, x, B, sino, c, y);
    return cudaGetLastError();
}

cudaError_t bkproj_exact(const SparseView& csc, const float* c, uint32_t B, const float* norm,
                         float* x, float* u, cudaStream_t st) {
    if (csc.n == 0) return cudaSuccess;
    k_bkproj_exact<<<kB200SMs * 8, 256, 0, st>>>(csc, c, B, norm, x, u);
    return cudaGetLastError();
}

cudaError_t column_sums_exact(const SparseView& csc, float* norm, cudaStream_t st) {
    if (csc.n == 0) return cudaSuccess;
    k_colsum_exact<<<kB200SMs * 8, 256, 0, st>>>(csc, norm);
    return cudaGetLastError();
}

cudaError_t column_sums_atomic(const SparseView& csr, uint32_t C, float* norm, cudaStream_t st) {
    cudaError_t err = cudaMemsetAsync(norm, 0, (size_t)C * sizeof(float), st);
    if (err != cudaSuccess || csr.nnz == 0) return err;
    k_colsum_atomic<<<kB200SMs * 8, 256, 0, st>>>(csr, norm);
    return cudaGetLastError();
}

}  // namespace mlem
