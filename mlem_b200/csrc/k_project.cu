// k_project.cu -- the per-iteration MLEM kernels (sm_100a).
//
// Forward projection fused with calcCorrel, back projection over the CSC copy
// fused with calcUpdate, the atomic-scatter back projection, the one-pass
// per-row kernel, and the bit-exact variants.  Reference functions:
// calcFwProj/calcCorrel/calcBkProj/calcUpdate, mlem_seq/seqcsr4mlem.cpp:69-134.
//
// Work decomposition.  G lanes (4..32) own one row (or column); a warp owns
// 32/G rows; warps stride over rows (grid = blocks_per_sm x SMs, persistent
// style).  A kernel instance handles a tile of BT frames of the B frames that
// are interleaved in the vectors (x[col][B], c[row][B], ...).  Each element's
// BT floats are split over FL = BT/VW lanes of VW <= 4 floats, so the G lanes
// work on EPS = G/FL consecutive elements at a time: lane (slot, sub) takes
// element b + slot + j*EPS and frames [sub*VW, sub*VW + VW) of the tile.
// One gather instruction therefore reads, per element, one contiguous
// 4..64-byte block of the vector, and with one frame the 32 lanes hold 32
// consecutive voxels of a ray (packed into few sectors by the brick layout).
// Element loads are 8 bytes per lane with an L2 evict_first policy (the
// matrix is streamed once per pass); vector gathers use evict_last.  The
// per-row sums are combined by a butterfly over the slot bits of the lane.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "row_dev.cuh"

namespace mlem {

namespace {

#define MLEM_WARP_LOOP_SETUP                                                     \
    constexpr int RPW = 32 / G;                                                  \
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL;                        \
    const int lw = threadIdx.x & 31;                                             \
    const int lane = lw & (G - 1);                                               \
    const int sub = lane % FL;                                                   \
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; \
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;            \
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();                  \
    (void)VW;

// ---------------------------------------------------------------------------
// Forward projection (+ calcCorrel).
// ---------------------------------------------------------------------------
template <int G, int BT>
__global__ void __launch_bounds__(256) k_fwproj(SparseView csr, const float* __restrict__ x,
                                                uint32_t B, uint32_t f0,
                                                const int32_t* __restrict__ sino,
                                                float* __restrict__ c, float* __restrict__ y) {
    MLEM_WARP_LOOP_SETUP
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    // Only the correlation wanted: a row whose counts are zero in the tile's
    // frames has calcCorrel 0 whatever its projection, so its elements are
    // not read (the counts are loaded beside the row range).
    const bool skip_empty = c != nullptr && y == nullptr;
    // the visiting positions: a device-built list (the rows with counts) or all n
    const uint64_t nv = visit_count(csr);
    for (uint64_t base = warp * RPW; base < nv; base += nwarps * RPW) {
        const uint64_t v = base + lw / G;
        const bool active = v < nv;
        uint64_t r = 0, b = 0, e = 0;
        int32_t s[VW];
#pragma unroll
        for (int i = 0; i < VW; ++i) s[i] = 0;
        if (active) {
            if (csr.vrange) {  // a sorted visit: the row's range in one load
                const ulonglong2 q = csr.vrange[v];
                r = csr.order[v];
                b = q.x;
                e = q.y;
            } else {
                r = row_at(csr, v);
                b = csr.ptr[r];
                e = csr.ptr[r + 1];
            }
            if (c) ld_counts<VW>(sino + r * B + f0 + sub * VW, s);
        }
        if (skip_empty) {
            bool any = false;
#pragma unroll
            for (int i = 0; i < VW; ++i) any |= s[i] != 0;
            // the group's frames are split over its FL lanes: all of them decide
#pragma unroll
            for (int o = 1; o < FL; o <<= 1) any |= __shfl_xor_sync(MLEM_FULL_MASK, any, o) != 0;
            if (!any) e = b;  // an empty walk: the sum is 0, calcCorrel 0
        }
        float acc[VW];
        row_dot<G, BT, false>(el, b, e, lane, x, B, f0 + sub * VW, acc, ps, ph);
        slot_allreduce<G, BT>(acc);
        if (active && lane < FL) {
            const uint64_t pos = csr.out_pos ? (uint64_t)csr.out_pos[r] : v;
            const uint64_t oidx = (csr.out_by_visit ? pos : r) * B + f0 + sub * VW;
            if (y) st_vec<VW>(y + oidx, acc);
            if (c) {
                float o[VW];
#pragma unroll
                for (int i = 0; i < VW; ++i) o[i] = correl_of(s[i], acc[i]);
                st_vec<VW>(c + oidx, o);
            }
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
    MLEM_WARP_LOOP_SETUP
    const uint2* el = reinterpret_cast<const uint2*>(csc.pairs);
    for (uint64_t base = warp * RPW; base < csc.n; base += nwarps * RPW) {
        const uint64_t col = base + lw / G;
        const bool active = col < csc.n;
        uint64_t b = 0, e = 0;
        if (active) span_of(csc, col, b, e);
        float acc[VW];
        row_dot<G, BT, false>(el, b, e, lane, c, B, f0 + sub * VW, acc, ps, ph);
        slot_allreduce<G, BT>(acc);
        if (active && lane < FL) {
            const uint64_t idx = col * B + f0 + sub * VW;
            if (norm) {
                const float n = norm[col];
                float xv[VW];
                ld_plain<VW>(x + idx, xv);
#pragma unroll
                for (int i = 0; i < VW; ++i) xv[i] *= update_factor(acc[i], n);
                st_vec<VW>(x + idx, xv);
            } else {
                st_vec<VW>(u + idx, acc);
            }
        }
    }
}

// The same back projection at one frame per pass and 32 lanes per column,
// with each warp's batches of 256 elements pipelined in registers across its
// columns: the element loads of the next batch (of this column or of the
// warp's next column) go out before the current batch's correlation gathers,
// so a batch costs about one memory round trip instead of two.  The lanes add
// their elements in the order of k_bkproj_csc<32, 1> and the same butterfly
// combines them: the results are those of that kernel, bit for bit.
__global__ void __launch_bounds__(256) k_bkproj_csc_pipe(SparseView csc, const float* __restrict__ c,
                                                         uint32_t B, uint32_t f0,
                                                         const float* __restrict__ norm,
                                                         float* __restrict__ x) {
    constexpr int kBatch = 8;
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    const uint2* el = reinterpret_cast<const uint2*>(csc.pairs);
    const uint64_t n = csc.n;
    uint64_t col = warp;
    if (col >= n) return;
    uint64_t k0 = 0, e = 0;
    span_of(csc, col, k0, e);
    uint2 q[kBatch];
#pragma unroll
    for (int t = 0; t < kBatch; ++t) {
        const uint64_t k = k0 + lane + 32 * t;
        q[t] = k < e ? ld_stream2(el + k, ps) : make_uint2(0u, 0u);
    }
    float acc = 0.0f;
    for (;;) {
        // the next batch: the rest of this column, else the warp's next column
        uint64_t ncol = col, nk0 = k0 + 32 * kBatch, ne = e;
        if (nk0 >= e) {
            ncol = col + nwarps;
            nk0 = ne = 0;
            if (ncol < n) span_of(csc, ncol, nk0, ne);
        }
        uint2 qn[kBatch];
#pragma unroll
        for (int t = 0; t < kBatch; ++t) {
            const uint64_t k = nk0 + lane + 32 * t;
            qn[t] = k < ne ? ld_stream2(el + k, ps) : make_uint2(0u, 0u);
        }
        float xv[kBatch];
#pragma unroll
        for (int t = 0; t < kBatch; ++t)
            xv[t] = k0 + lane + 32 * t < e ? ld_hot(c + (size_t)q[t].x * B + f0, ph) : 0.0f;
#pragma unroll
        for (int t = 0; t < kBatch; ++t) acc = fmaf(__uint_as_float(q[t].y), xv[t], acc);
        if (ncol != col) {  // the column is complete: k_bkproj_csc's butterfly and epilogue
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) acc += __shfl_xor_sync(MLEM_FULL_MASK, acc, o);
            if (lane == 0) {
                const uint64_t idx = col * B + f0;
                x[idx] *= update_factor(acc, norm[col]);
            }
            acc = 0.0f;
            if (ncol >= n) break;
        }
        col = ncol;
        k0 = nk0;
        e = ne;
#pragma unroll
        for (int t = 0; t < kBatch; ++t) q[t] = qn[t];
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
    MLEM_WARP_LOOP_SETUP
    constexpr int EPS = G / FL;
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t base = warp * RPW; base < csr.n; base += nwarps * RPW) {
        const uint64_t v = base + lw / G;
        if (v >= csr.n) continue;  // no shuffles in this kernel
        const uint64_t r = row_at(csr, v);
        const uint64_t b = csr.ptr[r], e = csr.ptr[r + 1];
        float cv[VW];
        ld_vec<VW>(c + r * B + f0 + sub * VW, cv, ph);
        bool any = false;
#pragma unroll
        for (int i = 0; i < VW; ++i) any |= (cv[i] != 0.0f);
        if (!any) continue;  // adding +0 changes no update entry
        float* ub = u + f0 + sub * VW;
        for (uint64_t k = b + lane / FL; k < e; k += EPS) {
            const uint2 q = ld_stream2(el + k, ps);
            red_vec<VW>(ub + (size_t)q.x * B, __uint_as_float(q.y), cv);
        }
    }
}

// ---------------------------------------------------------------------------
// One pass per row: forward projection, calcCorrel, and the back-projection
// scatter of the same row while its elements are still on chip (in
// registers when the row fits one load batch, else re-read from L1).  The
// matrix streams from HBM once per iteration.  The per-row work is in
// fused_row_range (row_dev.cuh), shared with the multi-matrix kernel.
// ---------------------------------------------------------------------------
template <int G, int BT, bool SORTED>
__global__ void __launch_bounds__(256) k_fused_row(SparseView csr, const float* __restrict__ x,
                                                   uint32_t B, uint32_t f0,
                                                   const int32_t* __restrict__ sino,
                                                   float* __restrict__ u) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    fused_row_range<G, BT, SORTED>(csr, x, B, f0, sino, u, 0, visit_count(csr), warp, nwarps);
}


#undef MLEM_WARP_LOOP_SETUP

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

// Column sums of the rows of subset s (row % S == s), in ascending row order:
// the elements of other subsets enter the sequential sum as +0, which leaves
// a non-negative float sum unchanged, so the result is calcColumnSums over the
// subset's rows bit for bit.
__global__ void __launch_bounds__(256) k_colsum_subset_exact(SparseView csc, uint32_t S, uint32_t s,
                                                             float* __restrict__ norm) {
    const uint2* el = reinterpret_cast<const uint2*>(csc.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t col = warp; col < csc.n; col += nwarps) {
        const uint64_t b = csc.ptr[col], e = csc.ptr[col + 1];
        float acc = 0.0f;
        for (uint64_t base = b; base < e; base += 32) {
            float v = 0.0f;
            if (base + lane < e) {
                const uint2 q = el[base + lane];
                if (q.x % S == s) v = __uint_as_float(q.y);
            }
            const int cnt = (int)min((uint64_t)32, e - base);
            for (int j = 0; j < cnt; ++j) acc = __fadd_rn(acc, __shfl_sync(MLEM_FULL_MASK, v, j));
        }
        if (lane == 0) norm[col] = acc;
    }
}

// Column sums of every subset at once by atomics (no CSC): norm[(r % S) * C + col].
__global__ void k_colsum_subset_atomic(SparseView csr, uint32_t S, uint64_t C,
                                       float* __restrict__ norm) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < csr.n; r += nwarps) {
        float* ns = norm + (r % S) * C;
        for (uint64_t k = csr.ptr[r] + lane; k < csr.ptr[r + 1]; k += 32) {
            const uint2 q = el[k];
            atomicAdd(ns + q.x, __uint_as_float(q.y));
        }
    }
}

// The ordered-subsets update: x *= norm_s != 0 ? u / norm_s : (norm != 0 ? 1 : u),
// u = 0 afterwards.  A voxel the subset does not see keeps its value; with one
// subset (norm_s == norm) this is calcUpdate.
template <bool ONE_FRAME>
__global__ void k_apply_update_subset(float* __restrict__ x, float* __restrict__ u,
                                      const float* __restrict__ norm_s,
                                      const float* __restrict__ norm, uint64_t n, uint32_t B) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t col = ONE_FRAME ? i : i / B;
        const float ns = norm_s[col];
        const float f = ns != 0.0f ? u[i] / ns : (norm[col] != 0.0f ? 1.0f : u[i]);
        x[i] *= f;
        u[i] = 0.0f;
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
template <int G, int BT>
struct FusedK {  // file order
    template <typename... A>
    static void run(int grid, cudaStream_t st, A... a) {
        k_fused_row<G, BT, false><<<grid, 256, 0, st>>>(a...);
    }
};
template <int G, int BT>
struct FusedSortedK {  // sorted visiting order (csr.order + csr.vrange)
    template <typename... A>
    static void run(int grid, cudaStream_t st, A... a) {
        k_fused_row<G, BT, true><<<grid, 256, 0, st>>>(a...);
    }
};
#undef MLEM_KERNEL_FUNCTOR

template <template <int, int> class K, int G, typename... Args>
cudaError_t dispatch_bt(const LaunchCfg& cfg, cudaStream_t st, Args... args) {
    const int grid = grid_for(cfg);
    switch (cfg.frame_tile) {
        case 1: K<G, 1>::run(grid, st, args...); break;
        case 2: K<G, 2>::run(grid, st, args...); break;
        case 4: K<G, 4>::run(grid, st, args...); break;
        case 8: K<G, 8>::run(grid, st, args...); break;
        case 16: K<G, 16>::run(grid, st, args...); break;
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
    // lanes per element (frame_tile / min(frame_tile, 4)) never exceed the group
    return g && t && c.blocks_per_sm >= 1 && c.blocks_per_sm <= 8 && c.sm_count >= 1;
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
    if (cfg.group == 32 && cfg.frame_tile == 1 && norm) {
        // the pipelined kernel (same results); 8 CTAs per SM measured best for
        // it whatever the configuration's blocks per SM (plain-full: 1.40 ms
        // against 1.66 for k_bkproj_csc<32, 1> at 4, the CSC method's choice)
        k_bkproj_csc_pipe<<<8 * cfg.sm_count, 256, 0, st>>>(csc, c, B, f0, norm, x);
        return cudaGetLastError();
    }
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
    if (csr.order && !csr.vrange) return cudaErrorInvalidValue;  // sorted visits carry vrange
    if (csr.vrange) return dispatch<FusedSortedK>(cfg, st, csr, x, B, f0, sino, u);
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

cudaError_t apply_update_subset(float* x, float* u, const float* norm_s, const float* norm,
                                uint32_t C, uint32_t B, cudaStream_t st) {
    const uint64_t n = (uint64_t)C * B;
    if (n == 0) return cudaSuccess;
    const int grid = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)kB200SMs * 16);
    if (B == 1) k_apply_update_subset<true><<<grid, 256, 0, st>>>(x, u, norm_s, norm, n, B);
    else k_apply_update_subset<false><<<grid, 256, 0, st>>>(x, u, norm_s, norm, n, B);
    return cudaGetLastError();
}

cudaError_t subset_column_sums_exact(const SparseView& csc, uint32_t S, uint32_t s, float* norm,
                                     cudaStream_t st) {
    if (S == 0 || s >= S) return cudaErrorInvalidValue;
    if (csc.n == 0) return cudaSuccess;
    k_colsum_subset_exact<<<kB200SMs * 8, 256, 0, st>>>(csc, S, s, norm);
    return cudaGetLastError();
}

cudaError_t subset_column_sums_atomic(const SparseView& csr, uint32_t S, uint32_t C, float* norm,
                                      cudaStream_t st) {
    if (S == 0) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(norm, 0, (size_t)S * C * 4, st);
    if (e != cudaSuccess || csr.n == 0) return e;
    k_colsum_subset_atomic<<<kB200SMs * 8, 256, 0, st>>>(csr, S, C, norm);
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
