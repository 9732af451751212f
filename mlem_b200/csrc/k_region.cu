// k_region.cu -- the region-blocked method (one shared-memory tile per region).
//
// With B frames the image gathers and update scatters of the row-wise
// kernels move 8*B bytes per element through L2 -- for 16 frames about 100 GB
// per iteration on the plain-full matrix, far more than the matrix itself.
// This method stores the matrix a second time, grouped by region: the device
// voxel order is a Morton curve, so every aligned block of RS = 2^rlog voxels
// is a compact box of the grid, and each row (a ray) is cut into segments,
// one per region it crosses.  A CTA then owns one region at a time:
//
//   forward : loads the region's image tile (RS x BT floats) into shared
//             memory once, computes every segment's partial projection from
//             shared memory, and adds it into the row's projection with one
//             vector atomic per segment (rows are complete after the pass);
//   correl  : c = calcCorrel(s, f), elementwise, in place;
//   backward: accumulates the region's update tile in shared memory from
//             every segment, then adds the tile into the update vector.
//
// Work is split evenly: the region-major element array (each region padded
// to whole 32-element chunks) is cut into equal contiguous chunk ranges, one
// per CTA; a CTA loads a region's tile once for the part of the region its
// range covers.  A warp takes one 32-element chunk at a time: the first
// element of every segment carries a head flag (bit 31 of its index word),
// chunk_seg[] gives the segment of each chunk's first element, so every lane
// knows its segment (and row) from a ballot; a segmented shuffle scan adds
// the products of a segment and its last lane adds the sum into the row's
// projection with one vector atomic.  The back projection accumulates each
// region's update tile with shared-memory atomics and flushes it to the
// global update vector once per (CTA, region); calcUpdate then runs as for
// the atomic methods.  Element traffic is two passes over the matrix, vector
// traffic is about one partial per segment instead of one gather per
// element.  The atomics make the summation order vary from run to run (like
// the atomic methods); results stay within the parity tolerance.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace mlem {

namespace {

__host__ __device__ inline uint64_t cdiv(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

template <int BT>
struct RLanes {
    static constexpr int VW = BT < 4 ? BT : 4;
    static constexpr int FL = BT / VW;
};

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

// Whole 32-element chunks per region (its elements rounded up).
__global__ void k_region_chunks(uint32_t nreg, const uint64_t* __restrict__ reg_seg_ptr,
                                const uint64_t* __restrict__ el_off, uint64_t* __restrict__ nchunks) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < nreg;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t len = el_off[reg_seg_ptr[g + 1]] - el_off[reg_seg_ptr[g]];
        nchunks[g] = cdiv(len, 32);
    }
}

// Warp per sorted segment: the segment's row, its elements (region-local
// index, head flag on the first), and the segment of every chunk that starts
// inside it.
__global__ void k_seg_fill(SparseView csr, int rlog, uint64_t S, const uint32_t* __restrict__ order,
                           const uint32_t* __restrict__ region_sorted,
                           const uint64_t* __restrict__ seg_start, const uint32_t* __restrict__ seg_row,
                           const uint32_t* __restrict__ seg_len, const uint64_t* __restrict__ el_off,
                           const uint64_t* __restrict__ reg_seg_ptr,
                           const uint64_t* __restrict__ reg_chunk_ptr,
                           uint32_t* __restrict__ row_sorted, uint32_t* __restrict__ chunk_seg,
                           uint2* __restrict__ rb_el) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t mask = (1u << rlog) - 1u;
    for (uint64_t p = warp; p < S; p += nwarps) {
        const uint32_t s = order[p];
        const uint32_t g = region_sorted[p];
        const uint64_t dst = reg_chunk_ptr[g] * 32 + (el_off[p] - el_off[reg_seg_ptr[g]]);
        const uint64_t src = seg_start[s];
        const uint32_t len = seg_len[s];
        if (lane == 0) row_sorted[p] = seg_row[s];
        for (uint32_t k = lane; k < len; k += 32) {
            const uint2 q = el[src + k];
            rb_el[dst + k] = make_uint2((q.x & mask) | (k == 0 ? 0x80000000u : 0u), q.y);
        }
        const uint64_t c_lo = cdiv(dst, 32), c_hi = (dst + len - 1) / 32;
        for (uint64_t c = c_lo + lane; c <= c_hi; c += 32) chunk_seg[c] = (uint32_t)p;
    }
}

// --- iteration kernels ---------------------------------------------------------
constexpr int kRbThreads = 512;

// The lanes of the warp that hold slot `slot` (lane = slot*FL + sub): the
// segment index of every lane's element, from the head flags.
template <int FL>
__device__ __forceinline__ uint32_t lane_segment(unsigned heads_sub0, int slot, uint32_t seg_prev) {
    const int bit = slot * FL;
    const unsigned upto = bit >= 31 ? 0xffffffffu : ((2u << bit) - 1u);
    return seg_prev + __popc(heads_sub0 & upto);
}

// Range of chunks of this CTA, and the region containing its first chunk.
__device__ __forceinline__ bool cta_range(const RegionView& rv, uint64_t& c0, uint64_t& c1,
                                          uint32_t& g) {
    const uint64_t per = cdiv(rv.nchunks, gridDim.x);
    c0 = (uint64_t)blockIdx.x * per;
    c1 = min(rv.nchunks, c0 + per);
    if (c0 >= c1) return false;
    uint32_t lo = 0, hi = rv.nreg;  // largest g with reg_chunk_ptr[g] <= c0
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (rv.reg_chunk_ptr[mid] <= c0) lo = mid; else hi = mid;
    }
    g = lo;
    return true;
}

template <int BT>
__global__ void __launch_bounds__(kRbThreads) k_rb_fwproj(RegionView rv, const float* __restrict__ x,
                                                          uint32_t B, uint32_t f0, uint32_t C,
                                                          float* __restrict__ fw) {
    extern __shared__ float tile[];  // RS x BT
    constexpr int VW = RLanes<BT>::VW, FL = RLanes<BT>::FL, EPS = 32 / FL;
    const uint32_t RS = 1u << rv.rlog;
    const int lane = threadIdx.x & 31, sub = lane % FL, slot = lane / FL;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint64_t pol = l2_evict_first();
    uint64_t c0, c1;
    uint32_t g;
    if (!cta_range(rv, c0, c1, g)) return;
    while (c0 < c1) {
        const uint64_t cend = min(c1, rv.reg_chunk_ptr[g + 1]);
        if (cend > c0) {
            const uint64_t v0 = (uint64_t)g * RS;
            for (uint32_t i = threadIdx.x; i < RS * BT; i += blockDim.x) {
                const uint32_t v = i / BT, f = i - v * BT;
                tile[i] = (v0 + v < C) ? x[(v0 + v) * B + f0 + f] : 0.0f;
            }
            __syncthreads();
            for (uint64_t cc = c0 + warp; cc < cend; cc += nwarps) {
                uint32_t seg_prev = 0;
#pragma unroll
                for (int pass = 0; pass < FL; ++pass) {
                    const uint2 q = ld_stream2(rv.el + cc * 32 + pass * EPS + slot, pol);
                    const bool head = (q.x >> 31) != 0;
                    const unsigned hb = __ballot_sync(MLEM_FULL_MASK, head && sub == 0);
                    if (pass == 0) seg_prev = rv.chunk_seg[cc] - (hb & 1u);
                    const uint32_t seg = lane_segment<FL>(hb, slot, seg_prev);
                    const float v = __uint_as_float(q.y);
                    const float* t = tile + (q.x & 0x7fffffffu) * BT + sub * VW;
                    float p[VW];
#pragma unroll
                    for (int i = 0; i < VW; ++i) p[i] = v * t[i];
#pragma unroll
                    for (int d = 1; d < EPS; d <<= 1) {
                        const uint32_t so = __shfl_up_sync(MLEM_FULL_MASK, seg, d * FL);
#pragma unroll
                        for (int i = 0; i < VW; ++i) {
                            const float po = __shfl_up_sync(MLEM_FULL_MASK, p[i], d * FL);
                            if (slot >= d && so == seg) p[i] += po;
                        }
                    }
                    const uint32_t sn = __shfl_down_sync(MLEM_FULL_MASK, seg, FL);
                    if (slot == EPS - 1 || sn != seg) {
                        float* dst = fw + (uint64_t)rv.seg_row[seg] * B + f0 + sub * VW;
                        if constexpr (VW == 4) atomicAdd(reinterpret_cast<float4*>(dst), make_float4(p[0], p[1], p[2], p[3]));
                        else if constexpr (VW == 2) atomicAdd(reinterpret_cast<float2*>(dst), make_float2(p[0], p[1]));
                        else atomicAdd(dst, p[0]);
                    }
                    seg_prev = __shfl_sync(MLEM_FULL_MASK, seg, (EPS - 1) * FL);
                }
            }
            __syncthreads();
        }
        c0 = cend;
        ++g;
    }
}

// Back projection: one frame per lane (FL = BT lanes per element), so each
// lane issues one shared-memory atomic per element, the BT lanes of an
// element hit BT consecutive banks, and the correlation of a segment's row
// is one coalesced BT-float read.
template <int BT>
__global__ void __launch_bounds__(kRbThreads) k_rb_bkproj(RegionView rv, const float* __restrict__ c,
                                                          uint32_t B, uint32_t f0, uint32_t C,
                                                          float* __restrict__ u) {
    extern __shared__ float tile[];  // RS x BT update accumulators
    constexpr int FL = BT, EPS = 32 / FL;
    const uint32_t RS = 1u << rv.rlog;
    const int lane = threadIdx.x & 31, sub = lane % FL, slot = lane / FL;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint64_t pol = l2_evict_first(), ph = l2_evict_last();
    uint64_t c0, c1;
    uint32_t g;
    if (!cta_range(rv, c0, c1, g)) return;
    while (c0 < c1) {
        const uint64_t cend = min(c1, rv.reg_chunk_ptr[g + 1]);
        if (cend > c0) {
            for (uint32_t i = threadIdx.x; i < RS * BT; i += blockDim.x) tile[i] = 0.0f;
            __syncthreads();
            for (uint64_t cc = c0 + warp; cc < cend; cc += nwarps) {
                uint32_t seg_prev = 0;
#pragma unroll 4
                for (int pass = 0; pass < FL; ++pass) {
                    const uint2 q = ld_stream2(rv.el + cc * 32 + pass * EPS + slot, pol);
                    const bool head = (q.x >> 31) != 0;
                    const unsigned hb = __ballot_sync(MLEM_FULL_MASK, head && sub == 0);
                    if (pass == 0) seg_prev = rv.chunk_seg[cc] - (hb & 1u);
                    const uint32_t seg = lane_segment<FL>(hb, slot, seg_prev);
                    seg_prev = __shfl_sync(MLEM_FULL_MASK, seg, (EPS - 1) * FL);
                    const float v = __uint_as_float(q.y);
                    if (v == 0.0f) continue;  // padding
                    const float cv = ld_hot(c + (uint64_t)rv.seg_row[seg] * B + f0 + sub, ph);
                    if (cv != 0.0f) atomicAdd(tile + (q.x & 0x7fffffffu) * BT + sub, v * cv);
                }
            }
            __syncthreads();
            const uint64_t v0 = (uint64_t)g * RS;
            for (uint32_t i = threadIdx.x; i < RS * BT; i += blockDim.x) {
                const uint32_t v = i / BT, f = i - v * BT;
                const float t = tile[i];
                if (t != 0.0f && v0 + v < C) atomicAdd(u + (v0 + v) * B + f0 + f, t);
            }
            __syncthreads();
        }
        c0 = cend;
        ++g;
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

}  // namespace

int region_rlog(int frame_tile, uint32_t C) {
    // one 64 KiB tile per CTA: RS * BT * 4 bytes (the work split keeps every
    // SM busy whatever the number of regions)
    int rlog = 14;
    for (int bt = frame_tile; bt > 1; bt >>= 1) --rlog;
    while (rlog > 3 && ((uint64_t)1 << rlog) > C) --rlog;
    return rlog;
}
static_assert(kRegionTileBytes == (1 << 14) * 4, "tile size and region_rlog disagree");

static int region_grid(const RegionBlocks& rb, int frame_tile, int sm_count) {
    const size_t tile = ((size_t)1 << rb.rlog) * frame_tile * 4;
    const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(4, (200u << 10) / std::max<size_t>(tile, 1)));
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(rb.nchunks, (uint64_t)sm_count * per_sm));
}

static cudaError_t raise_smem(size_t smem) {
    cudaError_t e = cudaSuccess;
#define MLEM_RAISE(BT)                                                       \
    if (e == cudaSuccess) e = set_smem_all(k_rb_fwproj<BT>, smem);           \
    if (e == cudaSuccess) e = set_smem_all(k_rb_bkproj<BT>, smem);
    MLEM_RAISE(1) MLEM_RAISE(2) MLEM_RAISE(4) MLEM_RAISE(8) MLEM_RAISE(16)
#undef MLEM_RAISE
    return e;
}

cudaError_t region_build(const SparseView& csr, uint32_t C, int rlog, RegionBlocks* out,
                         size_t* bytes_out, int* failed_line, cudaStream_t st) {
    *out = RegionBlocks{};
    out->rlog = rlog;
    out->nreg = (uint32_t)cdiv(C, 1ull << rlog);
    const uint64_t R = csr.n;
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
    const size_t scan_bytes = scan_scratch_bytes(std::max<uint64_t>(R, out->nreg) + 1);
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
    uint64_t *seg_start = nullptr, *len_sorted = nullptr, *el_off = nullptr, *reg_cnt = nullptr,
             *reg_seg_ptr = nullptr, *reg_nch = nullptr;
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
    MLEM_TRY(alloc((void**)&reg_cnt, ((uint64_t)out->nreg + 1) * 8));
    MLEM_TRY(alloc((void**)&reg_seg_ptr, ((uint64_t)out->nreg + 1) * 8));
    MLEM_TRY(alloc((void**)&reg_nch, ((uint64_t)out->nreg + 1) * 8));
    if (S) {
        k_seg_emit<<<grid, 256, 0, st>>>(csr, rlog, seg_ptr, seg_start, seg_row, seg_region);
        MLEM_TRY(cudaGetLastError());
        k_seg_len<<<grid, 256, 0, st>>>(csr, S, seg_start, seg_row, seg_len);
        MLEM_TRY(cudaGetLastError());
        k_iota<<<grid, 256, 0, st>>>(order_in, S);
        MLEM_TRY(cudaGetLastError());
        int bits = 1;
        while ((1ull << bits) < out->nreg) ++bits;
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
    // segments per region, chunks per region
    MLEM_TRY(cudaMemsetAsync(reg_cnt, 0, ((uint64_t)out->nreg + 1) * 8, st));
    if (S) {
        k_region_count<<<grid, 256, 0, st>>>(S, region_sorted, reinterpret_cast<unsigned long long*>(reg_cnt));
        MLEM_TRY(cudaGetLastError());
    }
    MLEM_TRY(exclusive_scan_u64(reg_cnt, reg_seg_ptr, out->nreg, scan_tmp, scan_bytes, st));
    k_region_chunks<<<(unsigned)cdiv(out->nreg, 256), 256, 0, st>>>(out->nreg, reg_seg_ptr, el_off, reg_nch);
    MLEM_TRY(cudaGetLastError());
    MLEM_TRY(keep((void**)&out->reg_chunk_ptr, ((uint64_t)out->nreg + 1) * 8));
    MLEM_TRY(exclusive_scan_u64(reg_nch, out->reg_chunk_ptr, out->nreg, scan_tmp, scan_bytes, st));
    uint64_t NC = 0;
    MLEM_TRY(cudaMemcpyAsync(&NC, out->reg_chunk_ptr + out->nreg, 8, cudaMemcpyDeviceToHost, st));
    MLEM_TRY(cudaStreamSynchronize(st));
    out->nchunks = NC;
    MLEM_TRY(keep((void**)&out->el, NC * 32 * 8));
    MLEM_TRY(keep((void**)&out->seg_row, S * 4));
    MLEM_TRY(keep((void**)&out->chunk_seg, NC * 4));
    MLEM_TRY(cudaMemsetAsync(out->el, 0, NC * 32 * 8, st));  // padding: value 0, no head
    if (S) {
        k_seg_fill<<<grid, 256, 0, st>>>(csr, rlog, S, order, region_sorted, seg_start, seg_row,
                                         seg_len, el_off, reg_seg_ptr, out->reg_chunk_ptr,
                                         out->seg_row, out->chunk_seg, out->el);
        MLEM_TRY(cudaGetLastError());
    }
    MLEM_TRY(cudaStreamSynchronize(st));
    MLEM_TRY(raise_smem(kRegionTileBytes));
    release();
#undef MLEM_TRY
    out->nseg = S;
    *bytes_out = bytes;
    return cudaSuccess;
}

void region_free(RegionBlocks* rb) {
    for (void* p : {(void*)rb->reg_chunk_ptr, (void*)rb->el, (void*)rb->seg_row, (void*)rb->chunk_seg})
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
                    uint32_t B, uint32_t f0, uint32_t C, float* u) {
        k_rb_bkproj<BT><<<grid, kRbThreads, smem, st>>>(rv, c, B, f0, C, u);
    }
};

static bool region_fits(const RegionBlocks& rb, int frame_tile) {
    return ((size_t)1 << rb.rlog) * frame_tile * 4 <= kRegionTileBytes;
}

cudaError_t region_fwproj(const RegionBlocks& rb, const float* x, uint32_t B, uint32_t f0,
                          uint32_t C, float* fw, const LaunchCfg& cfg, cudaStream_t st) {
    if (!region_fits(rb, cfg.frame_tile)) return cudaErrorInvalidValue;
    if (rb.nchunks == 0) return cudaSuccess;
    const size_t smem = ((size_t)1 << rb.rlog) * cfg.frame_tile * 4;
    return rb_dispatch<RbFw>(cfg.frame_tile, region_grid(rb, cfg.frame_tile, cfg.sm_count), smem,
                             st, rb.view(), x, B, f0, C, fw);
}

cudaError_t region_bkproj(const RegionBlocks& rb, const float* c, uint32_t B, uint32_t f0,
                          uint32_t C, float* u, const LaunchCfg& cfg, cudaStream_t st) {
    if (!region_fits(rb, cfg.frame_tile)) return cudaErrorInvalidValue;
    if (rb.nchunks == 0) return cudaSuccess;
    const size_t smem = ((size_t)1 << rb.rlog) * cfg.frame_tile * 4;
    return rb_dispatch<RbBk>(cfg.frame_tile, region_grid(rb, cfg.frame_tile, cfg.sm_count), smem,
                             st, rb.view(), c, B, f0, C, u);
}

cudaError_t correl_inplace(float* f, const int32_t* s, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(cdiv(n, 256), kB200SMs * 16));
    k_correl_inplace<<<grid, 256, 0, st>>>(f, s, n);
    return cudaGetLastError();
}

}  // namespace mlem
