// staged_dev.cuh -- the pipelined per-warp row walk of the staged row visit
// (MLEM_VISIT_SORTED_STAGED), shared by the single-matrix kernel
// (k_staged.cu) and the multi-matrix items kernel (k_batch.cu).
//
// In the row kernels of row_dev.cuh a row is a chain of dependent memory
// round trips: its range, then its elements, then the image gathers, then
// (after the warp reduction) its sinogram counts.  Here a warp runs a
// software pipeline over the rows it visits: while it works on row k, whose
// elements already sit in shared memory, the elements of row k+1 are in
// flight by cp.async (16 bytes per lane per instruction, cached in L2 only),
// the range of row k+2 and the counts of row k+1 are loading.  A row then
// waits for about one round trip (the gathers) instead of four.  A row longer
// than a stage (kStageCap elements, rounded out to whole 16-byte pairs) is
// read straight from global memory.
//
// Arithmetic per row is that of fused_row_range: f = sum of value * x over the
// row (the lanes' partial sums added by a butterfly), c = count / f (0 where
// f = 0), u[col] += value * c by vector reductions.
#pragma once

#include "common.cuh"
#include "kernels.h"
#include "row_dev.cuh"

namespace mlem {
namespace {

constexpr int kStageCap = 256;  // elements per stage: 2 KiB
constexpr int kStages = 2;      // this row and the next

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint64_t pol) {
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(dst),
                 "l"(src), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A range longer than long_len as an empty one: the long-row kernels take it.
__device__ __forceinline__ ulonglong2 clamp_long(ulonglong2 q, uint64_t long_len) {
    if (q.y - q.x > long_len) q.y = q.x;
    return q;
}

// Whole 16-byte pairs covering elements [q.x, q.y): first pair, pair count.
__device__ __forceinline__ bool stage_fits(ulonglong2 q) {
    const uint64_t a0 = q.x & ~1ull;
    return q.y > q.x && ((q.y - a0 + 1) >> 1) <= (uint64_t)(kStageCap / 2);
}

// Issue the copy of row range q into the stage at shared address `dst`
// (every lane of the warp calls it; one commit group per call, empty when
// the row does not fit or does not exist).  The rounded-out pair range stays
// inside the element array: it carries two spare elements.
__device__ __forceinline__ void stage_issue(const uint4* pairs, ulonglong2 q, bool exists,
                                            uint32_t dst, int lane, uint64_t pol) {
    if (exists && stage_fits(q)) {
        const uint64_t a0 = q.x >> 1;
        const uint32_t n = (uint32_t)(((q.y - (q.x & ~1ull)) + 1) >> 1);
        for (uint32_t c = lane; c < n; c += 32) cp_async16(dst + c * 16u, pairs + a0 + c, pol);
    }
    cp_commit();
}

// One row of the walk: forward sum, correlation, scatter.  The row's
// elements are read from its stage `st` (which holds them from element
// q.x & ~1 on) when it fits one, else straight from global memory; the same
// generic loads serve both.
template <int BT>
__device__ __forceinline__ void staged_row(const uint2* __restrict__ el, const uint2* st,
                                           ulonglong2 q, const int32_t (&s)[Lanes<BT>::VW],
                                           const float* __restrict__ x, uint32_t B, uint32_t off,
                                           float* __restrict__ u, int lane, uint64_t ph) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL, EPS = 32 / FL;
    constexpr int kBatch = VW == 4 ? 4 : 8;  // gathers in flight per lane
    const int slot = lane / FL;
    const uint2* row = stage_fits(q) ? st + (q.x & 1ull) : el + q.x;
    const int64_t n = (int64_t)(q.y - q.x);
    float acc[VW];
#pragma unroll
    for (int i = 0; i < VW; ++i) acc[i] = 0.0f;
    for (int64_t j0 = slot; j0 < n; j0 += kBatch * EPS) {
        uint2 e[kBatch];
        float xv[kBatch][VW];
#pragma unroll
        for (int t = 0; t < kBatch; ++t) {
            const int64_t j = j0 + t * EPS;
            e[t] = j < n ? row[j] : make_uint2(0u, 0u);
        }
#pragma unroll
        for (int t = 0; t < kBatch; ++t) {
            if (j0 + t * EPS < n) {
                ld_vec<VW>(x + off + (size_t)e[t].x * B, xv[t], ph);
            } else {
#pragma unroll
                for (int i = 0; i < VW; ++i) xv[t][i] = 0.0f;
            }
        }
#pragma unroll
        for (int t = 0; t < kBatch; ++t) {
            const float v = __uint_as_float(e[t].y);
#pragma unroll
            for (int i = 0; i < VW; ++i) acc[i] = fmaf(v, xv[t][i], acc[i]);
        }
    }
    slot_allreduce<32, BT>(acc);
    float cv[VW];
    bool any = false;
#pragma unroll
    for (int i = 0; i < VW; ++i) {
        cv[i] = correl_of(s[i], acc[i]);
        any |= (cv[i] != 0.0f);
    }
    if (!any) return;
    float* ub = u + off;
    for (int64_t j = slot; j < n; j += EPS) {
        const uint2 e = row[j];
        red_vec<VW>(ub + (size_t)e.x * B, __uint_as_float(e.y), cv);
    }
}

// The pipelined walk of one warp over visiting positions p0, p0 + S, ... <
// p_end for frames [f0, f0 + BT).  `sa` is the shared address of the warp's
// NS stages.
template <int BT, int NS>
__device__ __forceinline__ void staged_walk(const SparseView& csr, const float* __restrict__ x,
                                            uint32_t B, uint32_t f0,
                                            const int32_t* __restrict__ sino,
                                            float* __restrict__ u, uint64_t p0, uint64_t p_end,
                                            uint64_t S, const uint2* stages, uint32_t sa) {
    constexpr int VW = Lanes<BT>::VW, FL = Lanes<BT>::FL;
    const int lane = threadIdx.x & 31;
    const uint32_t off = f0 + (uint32_t)(lane % FL) * VW;
    const uint64_t ps = l2_evict_first(), ph = l2_evict_last();
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    if (p0 >= p_end) return;

    // ranges and rows of positions k .. k+NS-1 (k = the row being worked on)
    ulonglong2 qr[NS];
    uint32_t rr[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        const uint64_t p = p0 + (uint64_t)i * S;
        qr[i] = p < p_end ? clamp_long(csr.vrange[p], csr.long_len) : make_ulonglong2(0ull, 0ull);
        rr[i] = p < p_end ? csr.order[p] : 0u;
    }
#pragma unroll
    for (int i = 0; i + 1 < NS; ++i)
        stage_issue(csr.pairs, qr[i], p0 + (uint64_t)i * S < p_end,
                    sa + (uint32_t)i * (kStageCap * 8), lane, ps);
    int32_t s_cur[VW];
    ld_counts<VW>(sino + (size_t)rr[0] * B + off, s_cur);

    int stage = 0;
    for (uint64_t p = p0; p < p_end; p += S) {
        // the copy of row k+NS-1 goes out; the range of row k+NS and the
        // counts of row k+1 start loading
        const uint64_t pl = p + (uint64_t)(NS - 1) * S;
        const int sl = (stage + NS - 1) % NS;
        stage_issue(csr.pairs, qr[NS - 1], pl < p_end, sa + (uint32_t)sl * (kStageCap * 8), lane, ps);
        const uint64_t pn = pl + S;
        const ulonglong2 qn = pn < p_end ? clamp_long(csr.vrange[pn], csr.long_len) : make_ulonglong2(0ull, 0ull);
        const uint32_t rn = pn < p_end ? csr.order[pn] : 0u;
        int32_t s_nxt[VW];
        if (p + S < p_end) {
            ld_counts<VW>(sino + (size_t)rr[1 % NS] * B + off, s_nxt);
        } else {
#pragma unroll
            for (int i = 0; i < VW; ++i) s_nxt[i] = 0;
        }
        cp_wait<NS - 1>();
        __syncwarp();
        staged_row<BT>(el, stages + (size_t)stage * kStageCap, qr[0], s_cur, x, B, off, u, lane, ph);
        __syncwarp();  // this stage is refilled NS-1 rows from now
#pragma unroll
        for (int i = 0; i + 1 < NS; ++i) {
            qr[i] = qr[i + 1];
            rr[i] = rr[i + 1];
        }
        qr[NS - 1] = qn;
        rr[NS - 1] = rn;
#pragma unroll
        for (int i = 0; i < VW; ++i) s_cur[i] = s_nxt[i];
        stage = stage + 1 == NS ? 0 : stage + 1;
    }
    cp_wait<0>();
    __syncwarp();
}

// Dynamic shared memory of a CTA of `threads` threads running staged_walk.
constexpr size_t staged_smem_bytes(int threads) {
    return (size_t)(threads / 32) * kStages * kStageCap * 8;
}

}  // namespace
}  // namespace mlem
