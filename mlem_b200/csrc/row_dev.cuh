// row_dev.cuh -- per-row device building blocks of the row-wise kernels
// (k_project.cu) and the multi-matrix kernel (k_batch.cu).
//
// Work decomposition.  G lanes (4..32) own one row (or column); a warp owns
// 32/G rows.  A tile of BT frames of the B frames interleaved in the vectors
// is handled per pass: each element's BT floats are split over FL = BT/VW
// lanes of VW <= 4 floats, so the G lanes work on EPS = G/FL consecutive
// elements at a time (lane (slot, sub) takes element b + slot + j*EPS and
// frames [sub*VW, sub*VW + VW) of the tile).
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace mlem {
namespace {

template <int BT>
struct Lanes {
    static constexpr int VW = BT < 4 ? BT : 4;  // floats per lane
    static constexpr int FL = BT / VW;          // lanes per element
};

__device__ __forceinline__ float2 ld_hot2(const float2* ptr, uint64_t pol) {
    float2 r;
    asm("ld.global.nc.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;" : "=f"(r.x), "=f"(r.y)
        : "l"(ptr), "l"(pol));
    return r;
}

template <int VW>
__device__ __forceinline__ void ld_vec(const float* __restrict__ p, float (&v)[VW], uint64_t pol) {
    if constexpr (VW == 4) {
        const float4 t = ld_hot4(reinterpret_cast<const float4*>(p), pol);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (VW == 2) {
        const float2 t = ld_hot2(reinterpret_cast<const float2*>(p), pol);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = ld_hot(p, pol);
    }
}

template <int VW>
__device__ __forceinline__ void ld_plain(const float* __restrict__ p, float (&v)[VW]) {
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

template <int VW>
__device__ __forceinline__ void st_vec(float* __restrict__ p, const float (&v)[VW]) {
    if constexpr (VW == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else if constexpr (VW == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else *p = v[0];
}

template <int VW>
__device__ __forceinline__ void ld_counts(const int32_t* __restrict__ p, int32_t (&v)[VW]) {
    if constexpr (VW == 4) {
        const int4 t = *reinterpret_cast<const int4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (VW == 2) {
        const int2 t = *reinterpret_cast<const int2*>(p);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = *p;
    }
}

// Visiting positions of a one-pass walk: *csr.n_dev for a device-built list
// (rows with counts), else csr.n.
__device__ __forceinline__ uint64_t visit_count(const SparseView& csr) {
    return csr.n_dev ? (uint64_t)__ldg(csr.n_dev) : (uint64_t)csr.n;
}

// L2 prefetch of the bytes [p, p + bytes) rounded out to 16-byte bounds (at
// most 64 KiB): a hint -- nothing completes or waits on it.  The caller keeps
// the rounded range inside the allocation (the element arrays carry a spare
// 16 bytes).
__device__ __forceinline__ void prefetch_l2(const void* p, uint64_t bytes) {
    const uint64_t a0 = reinterpret_cast<uint64_t>(p) & ~15ull;
    const uint64_t a1 = (reinterpret_cast<uint64_t>(p) + bytes + 15) & ~15ull;
    const uint32_t n = (uint32_t)(a1 - a0 < 65536 ? a1 - a0 : 65536);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"(n) : "memory");
}

// u[...] += w * c[...] for VW floats (one vector reduction, 4..16 bytes).
template <int VW>
__device__ __forceinline__ void red_vec(float* __restrict__ p, float w, const float (&c)[VW]) {
    if constexpr (VW == 4)
        atomicAdd(reinterpret_cast<float4*>(p), make_float4(w * c[0], w * c[1], w * c[2], w * c[3]));
    else if constexpr (VW == 2)
        atomicAdd(reinterpret_cast<float2*>(p), make_float2(w * c[0], w * c[1]));
    else
        atomicAdd(p, w * c[0]);
}

// Elements a lane loads before it gathers (memory-level parallelism).  A
// full-warp group takes 8 (a 150-250-element row is one batch); narrower
// groups take 4, which keeps their registers, and so their occupancy, lower
// (measured on the plain-full workload).
template <int G>
constexpr int batch_depth() { return G == 32 ? 8 : 4; }

// acc[0..VW) = sum over the row's elements of value * vec[col*B + off + ...].
// Each batch issues all of its (predicated) element loads, then all of its
// gathers, so a row costs about two memory latencies per batch instead of
// two per element.  When `keep` is non-null and the whole row fits in one
// batch, the lane's elements are left in keep[] (fused kernel) and true is
// returned.
template <int G, int BT, bool KEEP>
__device__ __forceinline__ bool row_dot(const uint2* __restrict__ el, uint64_t b, uint64_t e,
                                        int lane, const float* __restrict__ vec, uint32_t B,
                                        uint32_t off, float (&acc)[Lanes<BT>::VW], uint64_t ps,
                                        uint64_t ph, uint2* keep = nullptr) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL, EPS = G / FL;
    constexpr int kBatch = batch_depth<G>();
    const float* base = vec + off;
#pragma unroll
    for (int i = 0; i < VW; ++i) acc[i] = 0.0f;
    const bool one_batch = e - b <= (uint64_t)kBatch * EPS;
    // Elements go through L1 when the fused kernel may re-read them for its
    // scatter (rows longer than one batch).  A full warp at one frame holds 256
    // elements per batch, so the rows of a typical matrix stay in registers
    // and their elements skip L1, leaving its lines to the image gathers
    // (plain-full, chunked walk: 2.450 vs 2.471 ms; at 16 frames, where rows
    // span several batches, skipping L1 cost 13 %).
    constexpr bool kL1 = KEEP && !(G == 32 && BT == 1);
    for (uint64_t k0 = b + lane / FL; k0 < e; k0 += (uint64_t)kBatch * EPS) {
        uint2 q[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const uint64_t k = k0 + (uint64_t)u * EPS;
            q[u] = make_uint2(0u, 0u);  // value 0: contributes nothing
            if (k < e) q[u] = kL1 ? ld_keep2(el + k, ps) : ld_stream2(el + k, ps);
        }
        float xv[kBatch][VW];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            if (k0 + (uint64_t)u * EPS < e) {
                ld_vec<VW>(base + (size_t)q[u].x * B, xv[u], ph);
            } else {
#pragma unroll
                for (int i = 0; i < VW; ++i) xv[u][i] = 0.0f;
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const float v = __uint_as_float(q[u].y);
#pragma unroll
            for (int i = 0; i < VW; ++i) acc[i] = fmaf(v, xv[u][i], acc[i]);
        }
        if (keep && one_batch) {
#pragma unroll
            for (int u = 0; u < kBatch; ++u) keep[u] = q[u];
        }
    }
    return one_batch;
}

// Sum over the element slots of the group: afterwards every lane holds the
// row totals of its frames.  Every lane of the warp must call it.
template <int G, int BT>
__device__ __forceinline__ void slot_allreduce(float (&acc)[Lanes<BT>::VW]) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL;
#pragma unroll
    for (int o = FL; o < G; o <<= 1)
#pragma unroll
        for (int i = 0; i < VW; ++i) acc[i] += __shfl_xor_sync(MLEM_FULL_MASK, acc[i], o);
}


// One pass per row over rows [r_begin, r_end): forward projection, calcCorrel
// and the scatter of the row into the update vector.  `warp` / `nwarps`
// number the warps that share the range (grid-wide or block-wide).
// SORTED: the view carries the sorted visiting order with its row ranges
// (csr.vrange); otherwise rows are visited in file order (csr.order null).
// A compile-time choice: the file-order loop measured 2.49 vs 3.15 ms on the
// plain-full matrix when the sorted path was a runtime branch inside it.
template <int G, int BT, bool SORTED>
__device__ __forceinline__ void fused_row_range(const SparseView& csr, const float* __restrict__ x,
                                                uint32_t B, uint32_t f0,
                                                const int32_t* __restrict__ sino,
                                                float* __restrict__ u, uint64_t r_begin,
                                                uint64_t r_end, uint64_t warp, uint64_t nwarps) {
    // [r_begin, r_end) are visiting positions (rows in csr.order when set)
    constexpr int RPW = 32 / G;
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL, EPS = G / FL;
    constexpr int kBatch = batch_depth<G>();
    const int lw = threadIdx.x & 31;
    const int lane = lw & (G - 1);
    const int sub = lane % FL;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t base = r_begin + warp * RPW; base < r_end; base += nwarps * RPW) {
        const uint64_t v = base + lw / G;  // visiting position
        const bool active = v < r_end;
        uint64_t r = 0, b = 0, e = 0;
        if constexpr (SORTED) {
            if (active) {
                const ulonglong2 q = csr.vrange[v];
                r = csr.order[v];
                b = q.x;
                e = q.y;
            }
            // the row this lane group takes next: its range load goes out beside
            // this row's, and its elements are prefetched into L2 while this row
            // is worked on (in file order the next row of a grid-stride walk is
            // thousands of rows away and a prefetch only adds L2 requests)
            const uint64_t nv = v + nwarps * RPW;
            if (lane == 0 && nv < r_end) {
                const ulonglong2 nq = csr.vrange[nv];
                if (nq.y > nq.x) prefetch_l2(el + nq.x, (nq.y - nq.x) * 8);
            }
        } else {
            r = v;
            if (active) {
                b = csr.ptr[r];
                e = csr.ptr[r + 1];
            }
        }
        if (e - b > csr.long_len) e = b;  // left to the long-row kernels
        float acc[VW];
        uint2 kept[kBatch];
        const bool in_regs =
            row_dot<G, BT, true>(el, b, e, lane, x, B, f0 + sub * VW, acc, ps, ph, kept);
        slot_allreduce<G, BT>(acc);
        if (!active) continue;
        const uint64_t idx = r * B + f0 + sub * VW;
        int32_t s[VW];
        ld_counts<VW>(sino + idx, s);
        float cv[VW];
        bool any = false;
#pragma unroll
        for (int i = 0; i < VW; ++i) {
            cv[i] = correl_of(s[i], acc[i]);
            any |= (cv[i] != 0.0f);
        }
        if (!any) continue;
        float* ub = u + f0 + sub * VW;
        if (in_regs) {
            // the whole row is still in registers: scatter from there
#pragma unroll
            for (int q = 0; q < kBatch; ++q)
                if (b + lane / FL + (uint64_t)q * EPS < e)
                    red_vec<VW>(ub + (size_t)kept[q].x * B, __uint_as_float(kept[q].y), cv);
        } else {
            for (uint64_t k = b + lane / FL; k < e; k += EPS) {
                const uint2 q = ld_keep2(el + k, ps);
                red_vec<VW>(ub + (size_t)q.x * B, __uint_as_float(q.y), cv);
            }
        }
    }
}

}  // namespace
}  // namespace mlem
