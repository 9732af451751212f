// k_mirror.cu -- projections of a symmetry-compressed matrix with the mirrors
// applied inside the kernels (contexts made with MLEM_FLAG_MIRROR_KERNELS).
//
// A compressed matrix stores the elements of some LOR x voxel pairs; the full
// matrix (what k_sym.cu builds at creation) adds, for every mirror s of the
// header flags, element (lor(r, s), vox(v, s), a) for every stored (r, v, a)
// (csr4matrix.cpp:62-65; regeneration as visualizematrix/dispcsr4spy.cpp:
// 123-140 with the tables of symhandler.cpp:33-114).  Here the device keeps
// only the stored elements; each kernel reads a stored row once and works it
// for every mirror in turn (the identity first), so the matrix streams about
// 1/|mirrors| of the full matrix's bytes while the image gathers and update
// reductions stay those of the full matrix.
//
// Because a full row collects elements from several stored rows, the
// iteration takes two passes: the forward pass adds each (stored row,
// mirror) partial sum into f[lor(r, s)] (float atomics), then the backward
// pass scatters value * calcCorrel(sino[t], f[t]) -- or value * y[t] for a
// plain transposed product -- to the mirrored voxels.
//
// Voxel maps: the device voxel order is a Morton code; when every grid
// dimension is a power of two that code is the bit interleave itself, and a
// mirror (x -> nx-1-x and so on) complements that axis's bits: an XOR with a
// mask.  Otherwise the map is a table of C entries per mirror.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "row_dev.cuh"

namespace mlem {

namespace {

constexpr int kMirrorThreads = 256;
constexpr int kMirrorCtasPerSm = 3;
// 3 blocks of 256 threads per SM (at most 85 registers): the mirror groups
// below hold more loads in flight than 64 registers allow, and unbounded
// they take 100-110 registers and too few warps (measured on the plain-full
// matrix with three mirrors: 30.7 ms per iteration bounded, 33.3 unbounded,
// 31.8 with one mirror at a time).
constexpr int kMirrorBatch = 8;  // elements per lane held across the mirrors

// Mirrors worked on together, so that their loads go out back to back: the
// forward pass gathers for FW mirrors at once (one at wide frame tiles, whose
// gathers already fill the registers), the backward pass loads the row sums
// and counts of BK mirrors at once.
template <int BT>
constexpr int fw_group() { return Lanes<BT>::VW == 1 ? 2 : 1; }
template <int BT>
constexpr int bk_group() { return Lanes<BT>::VW == 1 ? 8 : Lanes<BT>::VW == 2 ? 4 : 2; }

// Full rows of stored row r = d1 * n_crystals + d2 under mirrors j0 .. j0+MG-1
// (symhandler.hpp transformLor: both detectors mapped, the smaller first;
// mirror 0 is the row itself).  Entries past the last mirror are left as r.
template <int MG>
__device__ __forceinline__ void mirror_rows(uint32_t r, uint32_t d1, uint32_t d2, uint32_t j0,
                                            const MirrorView& mv, uint32_t (&t)[MG]) {
    uint32_t a[MG], c[MG];
#pragma unroll
    for (int p = 0; p < MG; ++p) {
        const uint32_t j = j0 + p;
        const bool mapped = j != 0 && j < mv.n;
        const uint32_t* lut = mv.lut + (size_t)(mapped ? j : 0) * mv.n_crystals;
        a[p] = mapped ? __ldg(lut + d1) : 0u;
        c[p] = mapped ? __ldg(lut + d2) : 0u;
    }
#pragma unroll
    for (int p = 0; p < MG; ++p) {
        const uint32_t j = j0 + p;
        t[p] = (j == 0 || j >= mv.n) ? r
               : a[p] < c[p] ? a[p] * mv.n_crystals + c[p] : c[p] * mv.n_crystals + a[p];
    }
}

struct VoxMap {
    const uint32_t* table;  // null: XOR with mask (or the identity)
    uint32_t mask;
    __device__ __forceinline__ uint32_t operator()(uint32_t v) const {
        return table ? __ldg(table + v) : (v ^ mask);
    }
};

// Mirror j's voxel map (j past the last mirror: the identity, never used).
__device__ __forceinline__ VoxMap vox_map(uint32_t j, const MirrorView& mv) {
    if (j == 0 || j >= mv.n) return VoxMap{nullptr, 0u};
    if (!mv.vox) return VoxMap{nullptr, mv.xor_mask[j]};
    return VoxMap{mv.vox + (size_t)j * mv.C, 0u};
}

// acc[p][0..VW) += sum over the loaded elements q[] of value *
// vec[map_p(col) * B + ...] for the MG mirrors of a group (nm of them real).
template <int BT, int MG>
__device__ __forceinline__ void mirrored_dot(const uint2 (&q)[kMirrorBatch],
                                             const bool (&live)[kMirrorBatch],
                                             const VoxMap (&map)[MG], int nm,
                                             const float* __restrict__ base, uint32_t B,
                                             float (&acc)[MG][Lanes<BT>::VW], uint64_t ph) {
    constexpr int VW = Lanes<BT>::VW;
    uint32_t m[MG][kMirrorBatch];
#pragma unroll
    for (int p = 0; p < MG; ++p)
#pragma unroll
        for (int u = 0; u < kMirrorBatch; ++u) m[p][u] = (p < nm && live[u]) ? map[p](q[u].x) : 0u;
    float xv[MG][kMirrorBatch][VW];
#pragma unroll
    for (int p = 0; p < MG; ++p)
#pragma unroll
        for (int u = 0; u < kMirrorBatch; ++u) {
            if (p < nm && live[u]) {
                ld_vec<VW>(base + (size_t)m[p][u] * B, xv[p][u], ph);
            } else {
#pragma unroll
                for (int i = 0; i < VW; ++i) xv[p][u][i] = 0.0f;
            }
        }
#pragma unroll
    for (int p = 0; p < MG; ++p)
#pragma unroll
        for (int u = 0; u < kMirrorBatch; ++u) {
            const float v = __uint_as_float(q[u].y);
#pragma unroll
            for (int i = 0; i < VW; ++i) acc[p][i] = fmaf(v, xv[p][u][i], acc[p][i]);
        }
}

// Element range of the warp's row at visiting position v.
template <bool SORTED>
__device__ __forceinline__ void row_at(const SparseView& csr, uint64_t v, uint32_t& r, uint64_t& b,
                                       uint64_t& e) {
    if constexpr (SORTED) {
        const ulonglong2 q = csr.vrange[v];
        r = csr.order[v];
        b = q.x;
        e = q.y;
    } else {
        r = (uint32_t)v;
        b = csr.ptr[v];
        e = csr.ptr[v + 1];
    }
}

// Loads batch k0 (lane offsets k0 + lane/FL + u*EPS) of the row [b, b+n).
template <int BT>
__device__ __forceinline__ void load_batch(const uint2* __restrict__ el, uint64_t b, uint64_t n,
                                           uint64_t k0, int lane, uint2 (&q)[kMirrorBatch],
                                           bool (&live)[kMirrorBatch], uint64_t ps) {
    constexpr int FL = Lanes<BT>::FL, EPS = 32 / FL;
#pragma unroll
    for (int u = 0; u < kMirrorBatch; ++u) {
        const uint64_t k = k0 + (uint64_t)(lane / FL) + (uint64_t)u * EPS;
        live[u] = k < n;
        q[u] = live[u] ? ld_keep2(el + b + k, ps) : make_uint2(0u, 0u);
    }
}

// Forward pass: f[lor(r, j) * B + f0 + ...] += the partial sum of stored row
// r under mirror j, for frames [f0, f0 + BT).
template <int BT, bool SORTED>
__global__ void __launch_bounds__(kMirrorThreads, kMirrorCtasPerSm) k_mirror_fw(SparseView csr, MirrorView mv,
                                                              const float* __restrict__ x, uint32_t B,
                                                              uint32_t f0, float* __restrict__ f) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL, EPS = 32 / FL, MG = fw_group<BT>();
    constexpr uint64_t kSpan = (uint64_t)kMirrorBatch * EPS;
    const int lane = threadIdx.x & 31, sub = lane % FL;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const float* xb = x + f0 + sub * VW;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < csr.n; v += nw) {
        uint32_t r;
        uint64_t b, e;
        row_at<SORTED>(csr, v, r, b, e);
        const uint64_t n = e - b;
        if (n == 0) continue;  // warp-uniform
        const uint32_t d1 = r / mv.n_crystals, d2 = r - d1 * mv.n_crystals;
        uint2 q0[kMirrorBatch];
        bool l0[kMirrorBatch];
        load_batch<BT>(el, b, n, 0, lane, q0, l0, ps);
        for (uint32_t j0 = 0; j0 < mv.n; j0 += MG) {
            const int nm = (int)min((uint32_t)MG, mv.n - j0);
            uint32_t t[MG];
            mirror_rows<MG>(r, d1, d2, j0, mv, t);  // off the gathers' path
            VoxMap map[MG];
#pragma unroll
            for (int p = 0; p < MG; ++p) map[p] = vox_map(j0 + p, mv);
            float acc[MG][VW];
#pragma unroll
            for (int p = 0; p < MG; ++p)
#pragma unroll
                for (int i = 0; i < VW; ++i) acc[p][i] = 0.0f;
            mirrored_dot<BT, MG>(q0, l0, map, nm, xb, B, acc, ph);
            for (uint64_t k0 = kSpan; k0 < n; k0 += kSpan) {  // rows longer than one batch
                uint2 q[kMirrorBatch];
                bool l[kMirrorBatch];
                load_batch<BT>(el, b, n, k0, lane, q, l, ps);
                mirrored_dot<BT, MG>(q, l, map, nm, xb, B, acc, ph);
            }
#pragma unroll
            for (int p = 0; p < MG; ++p) {
                slot_allreduce<32, BT>(acc[p]);
                if (p < nm && lane < FL) red_vec<VW>(f + (size_t)t[p] * B + f0 + sub * VW, 1.0f, acc[p]);
            }
        }
    }
}

// Backward pass: u[vox(v, j) * B + f0 + ...] += value * c, with c =
// calcCorrel(sino[t], y[t]) when sino is non-null, else y[t] (t = lor(r, j)).
template <int BT, bool SORTED>
__global__ void __launch_bounds__(kMirrorThreads, kMirrorCtasPerSm) k_mirror_bk(SparseView csr, MirrorView mv,
                                                              const float* __restrict__ y,
                                                              const int32_t* __restrict__ sino,
                                                              uint32_t B, uint32_t f0,
                                                              float* __restrict__ u) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL, EPS = 32 / FL, MG = bk_group<BT>();
    constexpr uint64_t kSpan = (uint64_t)kMirrorBatch * EPS;
    const int lane = threadIdx.x & 31, sub = lane % FL;
    const uint64_t ps = l2_evict_first();
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    float* ub = u + f0 + sub * VW;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < csr.n; v += nw) {
        uint32_t r;
        uint64_t b, e;
        row_at<SORTED>(csr, v, r, b, e);
        const uint64_t n = e - b;
        if (n == 0) continue;  // warp-uniform
        const uint32_t d1 = r / mv.n_crystals, d2 = r - d1 * mv.n_crystals;
        uint2 q0[kMirrorBatch];
        bool l0[kMirrorBatch];
        load_batch<BT>(el, b, n, 0, lane, q0, l0, ps);
        for (uint32_t j0 = 0; j0 < mv.n; j0 += MG) {
            uint32_t t[MG];
            mirror_rows<MG>(r, d1, d2, j0, mv, t);
            // the group's row sums and counts, all loads in flight together
            float cv[MG][VW];
            int32_t s[MG][VW];
#pragma unroll
            for (int p = 0; p < MG; ++p) {
                const size_t idx = (size_t)t[p] * B + f0 + sub * VW;
                ld_plain<VW>(y + idx, cv[p]);
                if (sino) ld_counts<VW>(sino + idx, s[p]);
            }
#pragma unroll
            for (int p = 0; p < MG; ++p) {
                if (j0 + p >= mv.n) break;  // warp-uniform
                bool any = false;
#pragma unroll
                for (int i = 0; i < VW; ++i) {
                    if (sino) cv[p][i] = correl_of(s[p][i], cv[p][i]);
                    any |= (cv[p][i] != 0.0f);
                }
                if (!__any_sync(MLEM_FULL_MASK, any)) continue;
                const VoxMap map = vox_map(j0 + p, mv);
#pragma unroll
                for (int w = 0; w < kMirrorBatch; ++w)
                    if (l0[w] && any)
                        red_vec<VW>(ub + (size_t)map(q0[w].x) * B, __uint_as_float(q0[w].y), cv[p]);
                for (uint64_t k = kSpan + (uint64_t)(lane / FL); k < n; k += EPS) {
                    const uint2 qe = ld_keep2(el + b + k, ps);
                    if (any) red_vec<VW>(ub + (size_t)map(qe.x) * B, __uint_as_float(qe.y), cv[p]);
                }
            }
        }
    }
}

// norm_full[w] = sum over the mirrors j (identity first) of norm_stored[vox(w, j)]:
// every mirror is its own inverse, so the stored elements that land on w
// under mirror j are those of column vox(w, j).
__global__ void k_mirror_norm(const float* __restrict__ norm, MirrorView mv, float* __restrict__ out) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < mv.C;
         w += (uint64_t)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (uint32_t j = 0; j < mv.n; ++j) s += norm[vox_map(j, mv)((uint32_t)w)];
        out[w] = s;
    }
}

// blocks_per_sm x SMs blocks (at most one warp per row).  More blocks than
// are resident (kMirrorCtasPerSm per SM) measured faster than one resident
// wave: 30.7 against 33.2 ms per iteration on the plain-full matrix with
// three mirrors at blocks_per_sm 8.
int mirror_grid(const SparseView& csr, int sm_count, int blocks_per_sm) {
    const uint64_t warps = csr.n;
    const uint64_t want = (warps * 32 + kMirrorThreads - 1) / kMirrorThreads;
    return (int)std::max<uint64_t>(
        1, std::min<uint64_t>(want, (uint64_t)sm_count * (uint64_t)std::max(1, blocks_per_sm)));
}

#define MLEM_MIRROR_TILES(KERNEL, SORTED, ...)                                           \
    switch (frame_tile) {                                                               \
        case 1: (SORTED ? KERNEL<1, true> : KERNEL<1, false>)<<<__VA_ARGS__; break;    \
        case 2: (SORTED ? KERNEL<2, true> : KERNEL<2, false>)<<<__VA_ARGS__; break;    \
        case 4: (SORTED ? KERNEL<4, true> : KERNEL<4, false>)<<<__VA_ARGS__; break;    \
        case 8: (SORTED ? KERNEL<8, true> : KERNEL<8, false>)<<<__VA_ARGS__; break;    \
        case 16: (SORTED ? KERNEL<16, true> : KERNEL<16, false>)<<<__VA_ARGS__; break; \
        default: return cudaErrorInvalidValue;                                          \
    }

}  // namespace

cudaError_t mirror_fwproj(const SparseView& csr, const MirrorView& mv, const float* x, uint32_t B,
                          uint32_t f0, int frame_tile, float* f, int sm_count, int blocks_per_sm,
                          cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    if (mv.n < 1 || mv.n > 8 || B % (uint32_t)frame_tile || f0 % (uint32_t)frame_tile)
        return cudaErrorInvalidValue;
    const bool sorted = csr.order && csr.vrange;
    const int grid = mirror_grid(csr, sm_count, blocks_per_sm);
    MLEM_MIRROR_TILES(k_mirror_fw, sorted, grid, kMirrorThreads, 0, st>>>(csr, mv, x, B, f0, f))
    return cudaGetLastError();
}

cudaError_t mirror_bkproj(const SparseView& csr, const MirrorView& mv, const float* y,
                          const int32_t* sino, uint32_t B, uint32_t f0, int frame_tile, float* u,
                          int sm_count, int blocks_per_sm, cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    if (mv.n < 1 || mv.n > 8 || B % (uint32_t)frame_tile || f0 % (uint32_t)frame_tile)
        return cudaErrorInvalidValue;
    const bool sorted = csr.order && csr.vrange;
    const int grid = mirror_grid(csr, sm_count, blocks_per_sm);
    MLEM_MIRROR_TILES(k_mirror_bk, sorted, grid, kMirrorThreads, 0,
                      st>>>(csr, mv, y, sino, B, f0, u))
    return cudaGetLastError();
}

cudaError_t mirror_norm(const float* norm_stored, const MirrorView& mv, float* norm_full,
                        cudaStream_t st) {
    if (mv.C == 0) return cudaSuccess;
    const int grid = (int)std::min<uint64_t>((mv.C + 255) / 256, (uint64_t)kB200SMs * 16);
    k_mirror_norm<<<grid, 256, 0, st>>>(norm_stored, mv, norm_full);
    return cudaGetLastError();
}

}  // namespace mlem
