// k_region.cu -- the region-blocked method (shared-memory tiles per region).
//
// With B frames the image gathers and update scatters of the row-wise
// kernels move 8*B bytes per element through L2 -- for 16 frames about 100 GB
// per iteration on the plain-full matrix, far more than the matrix itself.
// This method stores the matrix twice more, grouped by region: the device
// voxel order is a Morton curve, so every aligned block of RS = 2^rlog voxels
// is a compact box of the grid, and each row (a ray) is cut into segments,
// one per region it crosses.  Segments are ordered by region; each element
// becomes {word, value} with word = (segment index inside its region << rlog)
// | voxel index inside the region.  One CTA owns one region per launch:
//
//   forward : loads the region's image tile (RS x BT floats) into shared
//             memory once; lane groups walk fixed spans of the segment-major
//             copy, accumulate in registers and add each finished segment
//             partial into its row's projection with one vector atomic;
//   correl  : c = calcCorrel(s, f), elementwise, in place;
//   backward: the region's segments form blocks of SB; for each block the
//             correlations of its SB rows are staged in shared memory and the
//             block's voxel-major copy is walked in spans, accumulating each
//             voxel run in registers and adding it into the shared update tile
//             when the voxel changes; finally calcUpdate is applied to the
//             region's voxels of the image (the update vector never leaves
//             the SM).
//
// Per element the vectors cost two shared-memory reads and a fraction of a
// shared-memory atomic instead of two L2 round trips; the matrix is read
// twice per iteration (one copy per pass).  The atomics make the summation
// order vary from run to run (like the atomic methods); results stay within
// the parity tolerance.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "row_dev.cuh"

namespace mlem {

namespace {

__host__ __device__ inline uint64_t cdiv(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// --- build -------------------------------------------------------------------
// Warp per row; flags mark the first element of every run of one region.
__global__ void k_seg_count(SparseView csr, int rlog, uint64_t* __restrict__ nseg) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < csr.n; r += nwarps) {
        const uint64_t b = csr.ptr[r], e = csr.ptr[r + 1];
        uint32_t cnt = 0, carry = 0xffffffffu;
        for (uint64_t base = b; base < e; base += 32) {
            const uint64_t k = base + lane;
            const uint32_t g = k < e ? (el[k].x >> rlog) : 0xfffffffeu;
            uint32_t prev = __shfl_up_sync(MLEM_FULL_MASK, g, 1);
            if (lane == 0) prev = carry;
            const unsigned m = __ballot_sync(MLEM_FULL_MASK, k < e && g != prev);
            cnt += __popc(m);
            carry = __shfl_sync(MLEM_FULL_MASK, g, 31);
        }
        if (lane == 0) nseg[r] = cnt;
    }
}

__global__ void k_seg_emit(SparseView csr, int rlog, const uint64_t* __restrict__ seg_ptr,
                           uint64_t* __restrict__ seg_start, uint32_t* __restrict__ seg_row,
                           uint32_t* __restrict__ seg_region) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < csr.n; r += nwarps) {
        const uint64_t b = csr.ptr[r], e = csr.ptr[r + 1];
        uint64_t s = seg_ptr[r];
        uint32_t carry = 0xffffffffu;
        for (uint64_t base = b; base < e; base += 32) {
            const uint64_t k = base + lane;
            const uint32_t g = k < e ? (el[k].x >> rlog) : 0xfffffffeu;
            uint32_t prev = __shfl_up_sync(MLEM_FULL_MASK, g, 1);
            if (lane == 0) prev = carry;
            const bool flag = k < e && g != prev;
            const unsigned m = __ballot_sync(MLEM_FULL_MASK, flag);
            if (flag) {
                const uint64_t idx = s + __popc(m & ((1u << lane) - 1u));
                seg_start[idx] = k;
                seg_row[idx] = (uint32_t)r;
                seg_region[idx] = g;
            }
            s += __popc(m);
            carry = __shfl_sync(MLEM_FULL_MASK, g, 31);
        }
    }
}

// Segment length: up to the next segment of the same row, or the row's end.
__global__ void k_seg_len(SparseView csr, uint64_t S, const uint64_t* __restrict__ seg_start,
                          const uint32_t* __restrict__ seg_row, uint32_t* __restrict__ seg_len) {
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < S;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = seg_row[s];
        const uint64_t end = (s + 1 < S && seg_row[s + 1] == r) ? seg_start[s + 1] : csr.ptr[r + 1];
        seg_len[s] = (uint32_t)(end - seg_start[s]);
    }
}

__global__ void k_iota(uint32_t* __restrict__ v, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        v[i] = (uint32_t)i;
}

// Gather the lengths in region order (for the element-offset scan).
__global__ void k_seg_gather_len(uint64_t S, const uint32_t* __restrict__ order,
                                 const uint32_t* __restrict__ len, uint64_t* __restrict__ len_sorted) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < S;
         p += (uint64_t)gridDim.x * blockDim.x)
        len_sorted[p] = len[order[p]];
}

__global__ void k_region_count(uint64_t S, const uint32_t* __restrict__ region_sorted,
                               unsigned long long* __restrict__ cnt) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < S;
         p += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + region_sorted[p], 1ull);
}

// Elements per span (one lane group walks one span) and the position of
// linear element i of a block in the span-interleaved copies: a tile of gpw
// spans stores element k of all its spans side by side, so a warp step over
// its gpw lane groups is one coalesced load.  Blocks are padded to whole tiles.
constexpr uint32_t kSpan = 16;

__host__ __device__ __forceinline__ uint64_t span_pos(uint64_t i, uint32_t gpw) {
    const uint64_t tile = (uint64_t)gpw * kSpan;
    const uint64_t t = i / tile, w = i - t * tile;
    return t * tile + (w % kSpan) * gpw + w / kSpan;
}

// Blocks of every region: raw element start (el_off of the block's first
// segment; blk_raw[nblk] = all elements) and length padded to whole tiles.
__global__ void k_block_lens(uint32_t nreg, int sblog, uint64_t tile,
                             const uint64_t* __restrict__ reg_seg_ptr,
                             const uint32_t* __restrict__ reg_blk_ptr,
                             const uint64_t* __restrict__ el_off, uint64_t* __restrict__ blk_raw,
                             uint64_t* __restrict__ blk_plen) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g <= nreg;
         g += (uint64_t)gridDim.x * blockDim.x) {
        if (g == nreg) {
            blk_raw[reg_blk_ptr[nreg]] = el_off[reg_seg_ptr[nreg]];
            continue;
        }
        const uint64_t s0 = reg_seg_ptr[g], s1 = reg_seg_ptr[g + 1];
        for (uint32_t b = reg_blk_ptr[g]; b < reg_blk_ptr[g + 1]; ++b) {
            const uint64_t bs = s0 + ((uint64_t)(b - reg_blk_ptr[g]) << sblog);
            const uint64_t be = min(bs + ((uint64_t)1 << sblog), s1);
            blk_raw[b] = el_off[bs];
            blk_plen[b] = cdiv(el_off[be] - el_off[bs], tile) * tile;
        }
    }
}

__global__ void k_reg_el_ptr(uint32_t nreg, const uint32_t* __restrict__ reg_blk_ptr,
                             const uint64_t* __restrict__ blk_el_ptr, uint64_t* __restrict__ reg_el_ptr) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g <= nreg;
         g += (uint64_t)gridDim.x * blockDim.x)
        reg_el_ptr[g] = blk_el_ptr[reg_blk_ptr[g]];
}

// Segment-major copy: warp per sorted segment p (region g, segment index
// p - reg_seg_ptr[g] inside it), its elements in row order.
__global__ void k_fill_fw(SparseView csr, int rlog, int sblog, uint32_t gpw, uint64_t S,
                          const uint32_t* __restrict__ order, const uint32_t* __restrict__ region_sorted,
                          const uint64_t* __restrict__ seg_start, const uint32_t* __restrict__ seg_row,
                          const uint32_t* __restrict__ seg_len, const uint64_t* __restrict__ el_off,
                          const uint64_t* __restrict__ reg_seg_ptr,
                          const uint32_t* __restrict__ reg_blk_ptr, const uint64_t* __restrict__ blk_raw,
                          const uint64_t* __restrict__ blk_el_ptr, uint32_t* __restrict__ row_sorted,
                          uint2* __restrict__ el_fw) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t mask = (1u << rlog) - 1u;
    for (uint64_t p = warp; p < S; p += nwarps) {
        const uint32_t s = order[p];
        const uint32_t g = region_sorted[p];
        const uint32_t local = (uint32_t)(p - reg_seg_ptr[g]);
        const uint32_t b = reg_blk_ptr[g] + (local >> sblog);
        const uint64_t i0 = el_off[p] - blk_raw[b], dst = blk_el_ptr[b], src = seg_start[s];
        const uint32_t len = seg_len[s];
        if (lane == 0) row_sorted[p] = seg_row[s];
        for (uint32_t k = lane; k < len; k += 32) {
            const uint2 q = el[src + k];
            el_fw[dst + span_pos(i0 + k, gpw)] = make_uint2((local << rlog) | (q.x & mask), q.y);
        }
    }
}

// Padding of every block to whole tiles: copies of the block's last element
// (in the copy's own order) with value 0 -- they add 0 to a segment / voxel
// the span already holds.
__global__ void k_pad(uint32_t nblk, uint32_t gpw, const uint64_t* __restrict__ blk_raw,
                      const uint64_t* __restrict__ blk_el_ptr, uint2* __restrict__ el) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t b = warp; b < nblk; b += nwarps) {
        const uint64_t len = blk_raw[b + 1] - blk_raw[b], plen = blk_el_ptr[b + 1] - blk_el_ptr[b];
        if (len == 0 || len >= plen) continue;
        uint2* base = el + blk_el_ptr[b];
        const uint32_t w = base[span_pos(len - 1, gpw)].x;
        for (uint64_t i = len + lane; i < plen; i += 32) base[span_pos(i, gpw)] = make_uint2(w, 0u);
    }
}

// Voxel-major copy of every block: CTA per block, counting sort of its
// elements by voxel (shared-memory histogram, run placement, scatter).  The
// order inside one voxel's run is whatever the scatter atomics give.  The
// spans of the copy hold whole runs: a run of at most kSpan elements that
// would cross a span boundary starts the next span instead (the gap is
// padded with value-0 elements of the run before it), and a longer run
// starts a span of its own and pads its last one, so a span holds either
// whole runs or one piece of a single run.  The back projection then adds a
// run into the shared update tile with a plain read-modify-write, and uses
// atomics only for a span of one voxel (which may be such a piece).  A pad
// element's word carries segment 0 of its block (it adds 0 x that segment's
// correlation).  COUNT: the padded length of every block, whole tiles;
// otherwise the copy.
template <bool COUNT>
__global__ void __launch_bounds__(512) k_bk_layout(int rlog, uint32_t gpw,
                                                   const uint64_t* __restrict__ blk_raw,
                                                   const uint64_t* __restrict__ blk_el_ptr,
                                                   const uint2* __restrict__ el_fw,
                                                   uint64_t* __restrict__ bk_plen,
                                                   const uint64_t* __restrict__ bk_el_ptr,
                                                   uint2* __restrict__ el_bk) {
    extern __shared__ uint32_t hist[];  // RS counters, then the run starts
    const uint32_t RS = 1u << rlog, mask = RS - 1u;
    const uint64_t tile = (uint64_t)gpw * kSpan;
    const uint64_t len = blk_raw[blockIdx.x + 1] - blk_raw[blockIdx.x];
    const uint2* src = el_fw + blk_el_ptr[blockIdx.x];
    uint2* dst = COUNT ? nullptr : el_bk + bk_el_ptr[blockIdx.x];
    for (uint32_t i = threadIdx.x; i < RS; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint64_t i = threadIdx.x; i < len; i += blockDim.x)
        atomicAdd(hist + (src[span_pos(i, gpw)].x & mask), 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t pos = 0;
        uint32_t last = 0;
        auto pad_to = [&](uint64_t end, uint32_t word) {
            if (!COUNT)
                for (uint64_t p = pos; p < end; ++p) dst[span_pos(p, gpw)] = make_uint2(word, 0u);
            pos = end;
        };
        for (uint32_t v = 0; v < RS; ++v) {
            const uint32_t c = hist[v];
            if (c == 0) continue;
            const uint64_t up = cdiv(pos, kSpan) * kSpan;  // the next span boundary
            if (c <= kSpan) {
                if ((pos % kSpan) + c > kSpan) pad_to(up, last);
            } else if (pos % kSpan) {
                pad_to(up, last);
            }
            if (!COUNT) hist[v] = (uint32_t)pos;  // the run's first position
            pos += c;
            if (c > kSpan) {  // the long run's last span holds nothing else
                const uint64_t end = cdiv(pos, kSpan) * kSpan;
                if (!COUNT)
                    for (uint64_t p = pos; p < end; ++p) dst[span_pos(p, gpw)] = make_uint2(v, 0u);
                pos = end;
            }
            last = v;
        }
        const uint64_t plen = cdiv(pos, tile) * tile;
        pad_to(plen, last);
        if (COUNT) bk_plen[blockIdx.x] = plen;
    }
    __syncthreads();
    if (!COUNT)
        for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) {
            const uint2 q = src[span_pos(i, gpw)];
            const uint32_t p = atomicAdd(hist + (q.x & mask), 1u);
            dst[span_pos(p, gpw)] = q;
        }
}

// --- iteration kernels ---------------------------------------------------------
constexpr int kRbThreads = 512;

template <int BT>
struct RLanes2 {
    static constexpr int VW = BT < 4 ? BT : 4;  // frames per lane
    static constexpr int FL = BT / VW;          // lanes per element (one lane group)
};

template <int VW>
__device__ __forceinline__ void sts_vec(float* p, const float (&v)[VW]) {
    if constexpr (VW == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else if constexpr (VW == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else *p = v[0];
}

template <int VW>
__device__ __forceinline__ void lds_vec(const float* p, float (&v)[VW]) {
    if constexpr (VW == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (VW == 2) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = *p;
    }
}

// Forward projection of one frame tile: fw[row][f0 .. f0+BT) += partials.
template <int BT>
__global__ void __launch_bounds__(kRbThreads) k_rb_fwproj(RegionView rv, const float* __restrict__ x,
                                                          uint32_t B, uint32_t f0, uint32_t C,
                                                          float* __restrict__ fw) {
    extern __shared__ float tile[];  // RS x BT
    constexpr int VW = RLanes2<BT>::VW, FL = RLanes2<BT>::FL;
    const uint32_t g = rv.reg_order[blockIdx.x];
    const uint32_t RS = 1u << rv.rlog, mask = RS - 1u;
    const uint64_t v0 = (uint64_t)g * RS;
    for (uint32_t i = threadIdx.x; i < RS * BT; i += blockDim.x) {
        const uint32_t v = i / BT, f = i - v * BT;
        tile[i] = (v0 + v < C) ? x[(v0 + v) * B + f0 + f] : 0.0f;
    }
    __syncthreads();
    const uint64_t E0 = rv.reg_el_ptr[g], E1 = rv.reg_el_ptr[g + 1];  // whole tiles
    const uint32_t* __restrict__ srow = rv.seg_row + rv.reg_seg_ptr[g];
    constexpr uint32_t GPW = 32 / FL, TILE = GPW * kSpan;
    const int lane = threadIdx.x & 31, sub = lane % FL, grp = lane / FL;
    const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint64_t t0 = E0 + (uint64_t)warp * TILE; t0 < E1; t0 += (uint64_t)nwarps * TILE) {
        const uint2* __restrict__ sp = rv.el_fw + t0 + grp;  // element k of the span: sp[k * GPW]
        uint32_t cur = 0xffffffffu;
        uint32_t row = 0;  // srow[cur], loaded when the segment starts (used at its flush)
        float acc[VW];
#pragma unroll
        for (int i = 0; i < VW; ++i) acc[i] = 0.0f;
#pragma unroll 1
        for (uint32_t k0 = 0; k0 < kSpan; k0 += 8) {
            uint2 q[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) q[j] = sp[(k0 + j) * GPW];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t seg = q[j].x >> rv.rlog;
                if (seg != cur) {
                    if (cur != 0xffffffffu)
                        red_vec<VW>(fw + (uint64_t)row * B + f0 + sub * VW, 1.0f, acc);
                    cur = seg;
                    row = srow[seg];
#pragma unroll
                    for (int i = 0; i < VW; ++i) acc[i] = 0.0f;
                }
                float t[VW];
                lds_vec<VW>(tile + (q[j].x & mask) * BT + sub * VW, t);
                const float w = __uint_as_float(q[j].y);
#pragma unroll
                for (int i = 0; i < VW; ++i) acc[i] += w * t[i];
            }
        }
        red_vec<VW>(fw + (uint64_t)row * B + f0 + sub * VW, 1.0f, acc);
    }
}

// Back projection + calcUpdate of one frame tile: x[v][f0 .. f0+BT) of the
// region's voxels *= factor(A^T c, norm).
template <int BT>
__global__ void __launch_bounds__(kRbThreads, 2) k_rb_bkproj(RegionView rv, const float* __restrict__ c,
                                                          uint32_t B, uint32_t f0, uint32_t C,
                                                          const float* __restrict__ norm,
                                                          float* __restrict__ x) {
    extern __shared__ float sm[];  // update tile RS x BT, then the block's correlations SB x BT
    constexpr int VW = RLanes2<BT>::VW, FL = RLanes2<BT>::FL;
    const uint32_t g = rv.reg_order[blockIdx.x];
    const uint32_t RS = 1u << rv.rlog, mask = RS - 1u, SB = 1u << rv.sblog;
    float* ut = sm;
    float* cs = sm + (size_t)RS * BT;
    for (uint32_t i = threadIdx.x; i < RS * BT; i += blockDim.x) ut[i] = 0.0f;
    const uint64_t seg0 = rv.reg_seg_ptr[g], nseg = rv.reg_seg_ptr[g + 1] - seg0;
    constexpr uint32_t GPW = 32 / FL, TILE = GPW * kSpan;
    const int lane = threadIdx.x & 31, sub = lane % FL, grp = lane / FL;
    const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t b0 = rv.reg_blk_ptr[g], b1 = rv.reg_blk_ptr[g + 1];
    for (uint32_t b = b0; b < b1; ++b) {
        const uint64_t bs = seg0 + ((uint64_t)(b - b0) << rv.sblog);
        const uint32_t bn = (uint32_t)min((uint64_t)SB, seg0 + nseg - bs);
        __syncthreads();  // the previous block is done with cs (and ut is zeroed)
        // thread per segment: one row lookup, then the row's BT correlations as
        // independent vector loads (a strided float-by-float copy would chain a
        // row lookup and a gather per float)
        for (uint32_t sl = threadIdx.x; sl < bn; sl += blockDim.x) {
            const float* src = c + (uint64_t)rv.seg_row[bs + sl] * B + f0;
            float* dst = cs + sl * BT;
            if constexpr (BT >= 4) {
                float4 v[BT / 4];
#pragma unroll
                for (int i = 0; i < BT / 4; ++i) v[i] = reinterpret_cast<const float4*>(src)[i];
#pragma unroll
                for (int i = 0; i < BT / 4; ++i) reinterpret_cast<float4*>(dst)[i] = v[i];
            } else {
#pragma unroll
                for (int i = 0; i < BT; ++i) dst[i] = src[i];
            }
        }
        __syncthreads();
        const uint64_t E0 = rv.bk_el_ptr[b], E1 = rv.bk_el_ptr[b + 1];  // whole tiles
        for (uint64_t t0 = E0 + (uint64_t)warp * TILE; t0 < E1; t0 += (uint64_t)nwarps * TILE) {
            const uint2* __restrict__ sp = rv.el_bk + t0 + grp;
            uint32_t cur = 0xffffffffu;
            bool first = true;  // the current run is the span's first
            float acc[VW];
#pragma unroll
            for (int i = 0; i < VW; ++i) acc[i] = 0.0f;
#pragma unroll 1
            for (uint32_t k0 = 0; k0 < kSpan; k0 += 8) {
                uint2 q[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) q[j] = sp[(k0 + j) * GPW];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t vox = q[j].x & mask;
                    if (vox != cur) {
                        if (cur != 0xffffffffu) {
                            // The spans hold whole runs (k_bk_layout): a run that
                            // ends inside the span is in no other span, and this
                            // lane group adds it with a plain read-modify-write.
                            float* dst = ut + cur * BT + sub * VW;
                            float t[VW];
                            lds_vec<VW>(dst, t);
#pragma unroll
                            for (int i = 0; i < VW; ++i) t[i] += acc[i];
                            sts_vec<VW>(dst, t);
                            first = false;
                        }
                        cur = vox;
#pragma unroll
                        for (int i = 0; i < VW; ++i) acc[i] = 0.0f;
                    }
                    float cv[VW];
                    lds_vec<VW>(cs + ((q[j].x >> rv.rlog) & (SB - 1u)) * BT + sub * VW, cv);
                    const float w = __uint_as_float(q[j].y);
#pragma unroll
                    for (int i = 0; i < VW; ++i) acc[i] += w * cv[i];
                }
            }
            // the span's last run: whole (plain), unless the span holds one voxel
            // only, which may be a piece of a run longer than a span (atomics)
            float* dst = ut + cur * BT + sub * VW;
            if (first) {
#pragma unroll
                for (int i = 0; i < VW; ++i) atomicAdd(dst + i, acc[i]);
            } else {
                float t[VW];
                lds_vec<VW>(dst, t);
#pragma unroll
                for (int i = 0; i < VW; ++i) t[i] += acc[i];
                sts_vec<VW>(dst, t);
            }
        }
    }
    __syncthreads();
    const uint64_t v0 = (uint64_t)g * RS;
    for (uint32_t i = threadIdx.x; i < RS * BT; i += blockDim.x) {
        const uint32_t v = i / BT, f = i - v * BT;
        if (v0 + v < C) {
            float* px = x + (v0 + v) * B + f0 + f;
            *px *= update_factor(ut[i], norm[v0 + v]);
        }
    }
}

__global__ void k_correl_inplace(float* __restrict__ f, const int32_t* __restrict__ s, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        f[i] = correl_of(s[i], f[i]);
}

template <typename F>
cudaError_t set_smem_all(F f, size_t smem) {
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

size_t fw_smem(int rlog, int bt) { return ((size_t)1 << rlog) * bt * 4; }
size_t bk_smem(int rlog, int sblog, int bt) {
    return ((size_t)1 << rlog) * bt * 4 + ((size_t)1 << sblog) * bt * 4;
}
size_t fill_smem(int rlog) { return ((size_t)1 << rlog) * 4 + 512 * 4; }

}  // namespace

void region_params(int frame_tile, uint32_t C, int* rlog_out, int* sblog_out, uint32_t* gpw_out) {
    // image / update tile: RS x BT floats <= 64 KiB; at least ~4 regions per
    // SM so that one-region CTAs fill the GPU; correlation stage SB x BT
    // floats = 32 KiB
    int lt = 0;
    while ((1 << (lt + 1)) <= frame_tile) ++lt;
    int rlog = 14 - lt;
    while (rlog > 3 && ((uint64_t)kB200SMs * 4 << rlog) > C) --rlog;
    *rlog_out = rlog;
    *sblog_out = 13 - lt;
    // lane groups per warp: 32 / (lanes per element), lanes take <= 4 frames
    *gpw_out = 32u / (uint32_t)(frame_tile > 4 ? frame_tile / 4 : 1);
}
static_assert(kRegionTileBytes == (1u << 14) * 4, "region_params keeps RS x BT x 4 <= 64 KiB");

// Opt the kernels into the largest dynamic shared memory any build can ask
// for.  The attribute belongs to the kernel, not to a context, so it must not
// follow one build's sizes: region_params bounds every footprint (image /
// update tile RS x BT floats <= 64 KiB, correlation stage SB x BT floats =
// 32 KiB), and a launch may always ask for less than the attribute.
static cudaError_t raise_smem() {
    cudaError_t e = cudaSuccess;
    constexpr size_t kTile = 64u << 10, kStage = 32u << 10;
#define MLEM_RAISE(BT)                                                            \
    if (e == cudaSuccess) e = set_smem_all(k_rb_fwproj<BT>, kTile);              \
    if (e == cudaSuccess) e = set_smem_all(k_rb_bkproj<BT>, kTile + kStage);
    MLEM_RAISE(1) MLEM_RAISE(2) MLEM_RAISE(4) MLEM_RAISE(8) MLEM_RAISE(16)
#undef MLEM_RAISE
    return e;
}

cudaError_t region_build(const SparseView& csr, uint32_t C, int rlog, int sblog, uint32_t gpw,
                         RegionBlocks* out, size_t* bytes_out, int* failed_line, cudaStream_t st) {
    *out = RegionBlocks{};
    out->rlog = rlog;
    out->sblog = sblog;
    out->gpw = gpw;
    out->nreg = (uint32_t)cdiv(C, 1ull << rlog);
    const uint64_t R = csr.n;
    const uint32_t nreg = out->nreg;
    std::vector<void*> tmp;
    size_t bytes = 0;
    auto alloc = [&](void** p, size_t b) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, b ? b : 256);
        if (e == cudaSuccess) tmp.push_back(*p);
        return e;
    };
    auto keep = [&](void** p, size_t b) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, b ? b : 256);
        if (e == cudaSuccess) bytes += b ? b : 256;
        return e;
    };
    auto release = [&]() { for (void* p : tmp) cudaFree(p); tmp.clear(); };
    cudaError_t e;
#define MLEM_TRY(x)                                                  \
    do {                                                             \
        if ((e = (x)) != cudaSuccess) {                              \
            if (failed_line) *failed_line = __LINE__;                \
            release();                                               \
            region_free(out);                                        \
            return e;                                                \
        }                                                            \
    } while (0)
    const int grid = kB200SMs * 8;
    uint64_t* nseg = nullptr;
    uint64_t* seg_ptr = nullptr;
    void* scan_tmp = nullptr;
    MLEM_TRY(alloc((void**)&nseg, (R + 1) * 8));
    MLEM_TRY(alloc((void**)&seg_ptr, (R + 1) * 8));
    const size_t scan_bytes = scan_scratch_bytes(std::max<uint64_t>(R, nreg) + 1);
    MLEM_TRY(alloc(&scan_tmp, scan_bytes));
    if (R) {
        k_seg_count<<<grid, 256, 0, st>>>(csr, rlog, nseg);
        MLEM_TRY(cudaGetLastError());
    }
    MLEM_TRY(exclusive_scan_u64(nseg, seg_ptr, R, scan_tmp, scan_bytes, st));
    uint64_t S = 0;
    MLEM_TRY(cudaMemcpyAsync(&S, seg_ptr + R, 8, cudaMemcpyDeviceToHost, st));
    MLEM_TRY(cudaStreamSynchronize(st));
    // segment indices are 32-bit and the sort takes an int item count
    if (S > 0x7fffffffull) MLEM_TRY(cudaErrorInvalidValue);
    uint64_t *seg_start = nullptr, *len_sorted = nullptr, *el_off = nullptr, *reg_cnt = nullptr;
    uint32_t *seg_row = nullptr, *seg_region = nullptr, *seg_len = nullptr, *order_in = nullptr,
             *order = nullptr, *region_sorted = nullptr;
    MLEM_TRY(alloc((void**)&seg_start, S * 8));
    MLEM_TRY(alloc((void**)&seg_row, S * 4));
    MLEM_TRY(alloc((void**)&seg_region, S * 4));
    MLEM_TRY(alloc((void**)&seg_len, S * 4));
    MLEM_TRY(alloc((void**)&order_in, S * 4));
    MLEM_TRY(alloc((void**)&order, S * 4));
    MLEM_TRY(alloc((void**)&region_sorted, S * 4));
    MLEM_TRY(alloc((void**)&len_sorted, (S + 1) * 8));
    MLEM_TRY(alloc((void**)&el_off, (S + 1) * 8));
    MLEM_TRY(alloc((void**)&reg_cnt, ((uint64_t)nreg + 1) * 8));
    MLEM_TRY(keep((void**)&out->reg_seg_ptr, ((uint64_t)nreg + 1) * 8));
    if (S) {
        k_seg_emit<<<grid, 256, 0, st>>>(csr, rlog, seg_ptr, seg_start, seg_row, seg_region);
        MLEM_TRY(cudaGetLastError());
        k_seg_len<<<grid, 256, 0, st>>>(csr, S, seg_start, seg_row, seg_len);
        MLEM_TRY(cudaGetLastError());
        k_iota<<<grid, 256, 0, st>>>(order_in, S);
        MLEM_TRY(cudaGetLastError());
        int bits = 1;
        while ((1ull << bits) < nreg) ++bits;
        size_t sort_bytes = 0;
        MLEM_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, seg_region, region_sorted,
                                                 order_in, order, (int)S, 0, bits, st));
        void* sort_tmp = nullptr;
        MLEM_TRY(alloc(&sort_tmp, sort_bytes));
        MLEM_TRY(cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, seg_region, region_sorted,
                                                 order_in, order, (int)S, 0, bits, st));
        k_seg_gather_len<<<grid, 256, 0, st>>>(S, order, seg_len, len_sorted);
        MLEM_TRY(cudaGetLastError());
    }
    // element offsets in region order (the scan has S items: own scratch)
    void* scan_tmp_s = nullptr;
    const size_t scan_bytes_s = scan_scratch_bytes(S + 1);
    MLEM_TRY(alloc(&scan_tmp_s, scan_bytes_s));
    MLEM_TRY(exclusive_scan_u64(len_sorted, el_off, S, scan_tmp_s, scan_bytes_s, st));
    // segments per region
    MLEM_TRY(cudaMemsetAsync(reg_cnt, 0, ((uint64_t)nreg + 1) * 8, st));
    if (S) {
        k_region_count<<<grid, 256, 0, st>>>(S, region_sorted, reinterpret_cast<unsigned long long*>(reg_cnt));
        MLEM_TRY(cudaGetLastError());
    }
    MLEM_TRY(exclusive_scan_u64(reg_cnt, out->reg_seg_ptr, nreg, scan_tmp, scan_bytes, st));
    // blocks of SB segments per region (host: nreg is small); the segment
    // index inside a region must fit the word's 32 - rlog high bits
    std::vector<uint64_t> h_seg_ptr((size_t)nreg + 1);
    MLEM_TRY(cudaMemcpyAsync(h_seg_ptr.data(), out->reg_seg_ptr, ((size_t)nreg + 1) * 8,
                             cudaMemcpyDeviceToHost, st));
    MLEM_TRY(cudaStreamSynchronize(st));
    std::vector<uint32_t> h_blk_ptr((size_t)nreg + 1, 0);
    for (uint32_t g = 0; g < nreg; ++g) {
        const uint64_t n = h_seg_ptr[g + 1] - h_seg_ptr[g];
        if (n >= (1ull << (32 - rlog))) MLEM_TRY(cudaErrorInvalidValue);
        h_blk_ptr[g + 1] = h_blk_ptr[g] + (uint32_t)cdiv(n, 1ull << sblog);
    }
    const uint32_t nblk = h_blk_ptr[nreg];
    out->nblk = nblk;
    MLEM_TRY(keep((void**)&out->reg_blk_ptr, ((size_t)nreg + 1) * 4));
    MLEM_TRY(cudaMemcpyAsync(out->reg_blk_ptr, h_blk_ptr.data(), ((size_t)nreg + 1) * 4,
                             cudaMemcpyHostToDevice, st));
    // block element ranges, padded to whole span tiles
    const uint64_t tile = (uint64_t)gpw * kSpan;
    uint64_t *blk_raw = nullptr, *blk_plen = nullptr;
    MLEM_TRY(alloc((void**)&blk_raw, ((uint64_t)nblk + 1) * 8));
    MLEM_TRY(alloc((void**)&blk_plen, ((uint64_t)nblk + 1) * 8));
    k_block_lens<<<(unsigned)cdiv((uint64_t)nreg + 1, 256), 256, 0, st>>>(
        nreg, sblog, tile, out->reg_seg_ptr, out->reg_blk_ptr, el_off, blk_raw, blk_plen);
    MLEM_TRY(cudaGetLastError());
    MLEM_TRY(keep((void**)&out->blk_el_ptr, ((uint64_t)nblk + 1) * 8));
    void* scan_tmp_b = nullptr;
    const size_t scan_bytes_b = scan_scratch_bytes((uint64_t)nblk + 1);
    MLEM_TRY(alloc(&scan_tmp_b, scan_bytes_b));
    MLEM_TRY(exclusive_scan_u64(blk_plen, out->blk_el_ptr, nblk, scan_tmp_b, scan_bytes_b, st));
    MLEM_TRY(keep((void**)&out->reg_el_ptr, ((uint64_t)nreg + 1) * 8));
    k_reg_el_ptr<<<(unsigned)cdiv((uint64_t)nreg + 1, 256), 256, 0, st>>>(nreg, out->reg_blk_ptr,
                                                                         out->blk_el_ptr, out->reg_el_ptr);
    MLEM_TRY(cudaGetLastError());
    // regions with the most elements first (one CTA per region)
    std::vector<uint64_t> h_el_ptr((size_t)nreg + 1);
    MLEM_TRY(cudaMemcpyAsync(h_el_ptr.data(), out->reg_el_ptr, ((size_t)nreg + 1) * 8,
                             cudaMemcpyDeviceToHost, st));
    MLEM_TRY(cudaStreamSynchronize(st));
    std::vector<uint32_t> h_order(nreg);
    for (uint32_t g = 0; g < nreg; ++g) h_order[g] = g;
    std::stable_sort(h_order.begin(), h_order.end(), [&](uint32_t a, uint32_t b) {
        return h_el_ptr[a + 1] - h_el_ptr[a] > h_el_ptr[b + 1] - h_el_ptr[b];
    });
    MLEM_TRY(keep((void**)&out->reg_order, (size_t)nreg * 4));
    MLEM_TRY(cudaMemcpyAsync(out->reg_order, h_order.data(), (size_t)nreg * 4,
                             cudaMemcpyHostToDevice, st));
    // the two element copies (span-interleaved, padded)
    const uint64_t Z = h_el_ptr[nreg];
    MLEM_TRY(keep((void**)&out->seg_row, S * 4));
    MLEM_TRY(keep((void**)&out->el_fw, Z * 8));
    if (S) {
        k_fill_fw<<<grid, 256, 0, st>>>(csr, rlog, sblog, gpw, S, order, region_sorted, seg_start,
                                        seg_row, seg_len, el_off, out->reg_seg_ptr, out->reg_blk_ptr,
                                        blk_raw, out->blk_el_ptr, out->seg_row, out->el_fw);
        MLEM_TRY(cudaGetLastError());
    }
    // the voxel-major copy: its block lengths (run-aligned spans), offsets, then the copy
    MLEM_TRY(keep((void**)&out->bk_el_ptr, ((uint64_t)nblk + 1) * 8));
    uint64_t Zb = 0;
    if (nblk) {
        k_pad<<<grid, 256, 0, st>>>(nblk, gpw, blk_raw, out->blk_el_ptr, out->el_fw);
        MLEM_TRY(cudaGetLastError());
        // the largest region any build uses
        MLEM_TRY(set_smem_all(k_bk_layout<true>, fill_smem(14)));
        MLEM_TRY(set_smem_all(k_bk_layout<false>, fill_smem(14)));
        k_bk_layout<true><<<nblk, 512, fill_smem(rlog), st>>>(rlog, gpw, blk_raw, out->blk_el_ptr,
                                                            out->el_fw, blk_plen, nullptr, nullptr);
        MLEM_TRY(cudaGetLastError());
        MLEM_TRY(exclusive_scan_u64(blk_plen, out->bk_el_ptr, nblk, scan_tmp_b, scan_bytes_b, st));
        MLEM_TRY(cudaMemcpyAsync(&Zb, out->bk_el_ptr + nblk, 8, cudaMemcpyDeviceToHost, st));
        MLEM_TRY(cudaStreamSynchronize(st));
    } else {
        MLEM_TRY(cudaMemsetAsync(out->bk_el_ptr, 0, 8, st));
    }
    MLEM_TRY(keep((void**)&out->el_bk, Zb * 8));
    if (nblk) {
        k_bk_layout<false><<<nblk, 512, fill_smem(rlog), st>>>(rlog, gpw, blk_raw, out->blk_el_ptr,
                                                             out->el_fw, nullptr, out->bk_el_ptr,
                                                             out->el_bk);
        MLEM_TRY(cudaGetLastError());
    }
    MLEM_TRY(cudaStreamSynchronize(st));
    MLEM_TRY(raise_smem());
    release();
#undef MLEM_TRY
    out->nseg = S;
    out->nel = Z;
    out->nel_bk = Zb;
    *bytes_out = bytes;
    return cudaSuccess;
}

void region_free(RegionBlocks* rb) {
    for (void* p : {(void*)rb->reg_order, (void*)rb->reg_seg_ptr, (void*)rb->reg_el_ptr,
                    (void*)rb->reg_blk_ptr, (void*)rb->blk_el_ptr, (void*)rb->bk_el_ptr,
                    (void*)rb->seg_row,
                    (void*)rb->el_fw, (void*)rb->el_bk})
        if (p) cudaFree(p);
    *rb = RegionBlocks{};
}

template <template <int> class K, typename... A>
static cudaError_t rb_dispatch(int bt, int grid, size_t smem, cudaStream_t st, A... a) {
    switch (bt) {
        case 1: K<1>::run(grid, smem, st, a...); break;
        case 2: K<2>::run(grid, smem, st, a...); break;
        case 4: K<4>::run(grid, smem, st, a...); break;
        case 8: K<8>::run(grid, smem, st, a...); break;
        case 16: K<16>::run(grid, smem, st, a...); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int BT>
struct RbFw {
    static void run(int grid, size_t smem, cudaStream_t st, RegionView rv, const float* x,
                    uint32_t B, uint32_t f0, uint32_t C, float* fw) {
        k_rb_fwproj<BT><<<grid, kRbThreads, smem, st>>>(rv, x, B, f0, C, fw);
    }
};

template <int BT>
struct RbBk {
    static void run(int grid, size_t smem, cudaStream_t st, RegionView rv, const float* c,
                    uint32_t B, uint32_t f0, uint32_t C, const float* norm, float* x) {
        k_rb_bkproj<BT><<<grid, kRbThreads, smem, st>>>(rv, c, B, f0, C, norm, x);
    }
};

static bool region_fits(const RegionBlocks& rb, int frame_tile, uint32_t C) {
    int rlog = 0, sblog = 0;
    uint32_t gpw = 0;
    region_params(frame_tile, C, &rlog, &sblog, &gpw);
    return rb.el_fw && rb.rlog == rlog && rb.sblog == sblog && rb.gpw == gpw;
}

cudaError_t region_fwproj(const RegionBlocks& rb, const float* x, uint32_t B, uint32_t f0,
                          uint32_t C, float* fw, const LaunchCfg& cfg, cudaStream_t st) {
    if (!region_fits(rb, cfg.frame_tile, C)) return cudaErrorInvalidValue;
    if (rb.nreg == 0 || rb.nel == 0) return cudaSuccess;
    return rb_dispatch<RbFw>(cfg.frame_tile, (int)rb.nreg, fw_smem(rb.rlog, cfg.frame_tile), st,
                             rb.view(), x, B, f0, C, fw);
}

cudaError_t region_bkproj_update(const RegionBlocks& rb, const float* c, uint32_t B, uint32_t f0,
                                 uint32_t C, const float* norm, float* x, const LaunchCfg& cfg,
                                 cudaStream_t st) {
    if (!region_fits(rb, cfg.frame_tile, C)) return cudaErrorInvalidValue;
    if (rb.nreg == 0) return cudaSuccess;
    return rb_dispatch<RbBk>(cfg.frame_tile, (int)rb.nreg,
                             bk_smem(rb.rlog, rb.sblog, cfg.frame_tile), st, rb.view(), c, B, f0,
                             C, norm, x);
}

cudaError_t correl_inplace(float* f, const int32_t* s, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(cdiv(n, 256), kB200SMs * 16));
    k_correl_inplace<<<grid, 256, 0, st>>>(f, s, n);
    return cudaGetLastError();
}

}  // namespace mlem
