// capi.cu -- the mlem_ctx device context behind include/mlem_b200.h (the
// multi-matrix batches are in capi_batch.cu).
//
// One context = one CSR4 matrix resident on one GPU (CSR copy, CSC copy,
// column sums) plus the state of B frames.  The iteration of
// mlem_seq/seqcsr4mlem.cpp:163-167 is enqueued by enqueue_iteration() and
// replayed from a captured CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <thread>
#include <utility>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "ctx.hpp"
#include "host/errors.hpp"
#include "kernels.h"
#include "mlem_b200.h"

using namespace mlem;


namespace {

int fail(mlem_ctx* ctx, int status, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
int fail(mlem_ctx* ctx, int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return set_error(ctx ? &ctx->err : nullptr, status, "%s", buf);
}

#define CK(ctx, call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((ctx), e_ == cudaErrorMemoryAllocation ? MLEM_ERR_NOMEM : MLEM_ERR_CUDA, \
                        "%s: %s (%s:%d)", cudaGetErrorName(e_), cudaGetErrorString(e_),    \
                        __FILE__, __LINE__);                                                \
    } while (0)


int dev_alloc(mlem_ctx* c, void** p, size_t bytes) {
    if (bytes == 0) bytes = 256;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(c, MLEM_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", bytes,
                    cudaGetErrorString(e));
    }
    c->device_bytes += bytes;
    return MLEM_OK;
}

template <typename T>
int dev_alloc(mlem_ctx* c, T** p, size_t count) {
    return dev_alloc(c, reinterpret_cast<void**>(p), count * sizeof(T));
}

}  // namespace

namespace mlem {
void dev_free(void* p) {
    if (p) cudaFree(p);
}
}  // namespace mlem

namespace {

}  // namespace

namespace mlem {
SparseView csr_view(const mlem_ctx* c) {
    return SparseView{c->row_ptr, reinterpret_cast<const uint4*>(c->elems), c->R, c->Z,
                      c->row_order, c->row_order ? c->row_ranges : nullptr};
}
}  // namespace mlem

namespace {
SparseView csc_view(const mlem_ctx* c) {
    return SparseView{c->col_ptr, reinterpret_cast<const uint4*>(c->celems), c->C, c->Z};
}

int sm_count(int device) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) n = 148;
    return n > 0 ? n : 148;
}

LaunchCfg cfg_of(const mlem_ctx* c, const mlem_tuning& t) {
    LaunchCfg cfg;
    cfg.group = t.group;
    cfg.frame_tile = t.frame_tile;
    cfg.blocks_per_sm = t.blocks_per_sm;
    cfg.sm_count = c->n_sm;
    return cfg;
}

// Interleave stride for B frames: every frame tile 1..16 that fits divides it.
uint32_t padded_frames(uint32_t B) {
    for (uint32_t p : {1u, 2u, 4u, 8u, 16u, 32u, 48u, 64u})
        if (B <= p) return p;
    return 0;
}

// Widest frame tile (<= 16) that divides Bp.
int default_tile(uint32_t Bp) {
    for (int t : {16, 8, 4, 2})
        if (Bp % t == 0) return t;
    return 1;
}

int set_device(mlem_ctx* c) {
    CK(c, cudaSetDevice(c->device));
    return MLEM_OK;
}

void default_tuning(mlem_ctx* c) {
    c->tuning.bk_mode = c->has_csc ? MLEM_BK_CSC : MLEM_BK_ATOMIC;
    c->tuning.group = 32;
    c->tuning.frame_tile = c->Bp ? std::min(default_tile(c->Bp), 16) : 1;
    c->tuning.blocks_per_sm = 8;
    c->tuning.visit = MLEM_VISIT_FILE;
    c->tuning.ms_per_iter = 0.0;
}

// ---------------------------------------------------------------------------
// Device voxel order.  A ray's consecutive voxels are neighbours in 3-D; in
// the natural order (ix + nx*(iy + ny*iz), scannerconfig.cpp getVoxelNr)
// only its x-steps stay inside a 128-byte line.  A Morton (Z-order) curve
// over the whole grid puts every 2x2x2 cube in one 32-byte sector, every
// 4x4x2 block in one 128-byte line, and every aligned block of 2^k voxels in
// a compact box -- the regions of the region-blocked method.  Axes are
// interleaved level by level while they have bits left (x lowest), so the
// codes are dense when every dimension is a power of two; otherwise they
// are ranked.  The relabelling changes no arithmetic: rows keep their
// element order and columns keep their ascending row order.
// ---------------------------------------------------------------------------
uint64_t morton_code(uint32_t x, uint32_t y, uint32_t z, const int bits[3]) {
    uint64_t m = 0;
    int out = 0;
    const int top = std::max(bits[0], std::max(bits[1], bits[2]));
    for (int b = 0; b < top; ++b) {
        if (b < bits[0]) m |= (uint64_t)((x >> b) & 1u) << out++;
        if (b < bits[1]) m |= (uint64_t)((y >> b) & 1u) << out++;
        if (b < bits[2]) m |= (uint64_t)((z >> b) & 1u) << out++;
    }
    return m;
}

void brick_order(uint32_t nx, uint32_t ny, uint32_t nz, std::vector<uint32_t>& perm) {
    const uint64_t C = (uint64_t)nx * ny * nz;
    int bits[3] = {0, 0, 0};
    const uint32_t n[3] = {nx, ny, nz};
    bool pow2 = true;
    for (int i = 0; i < 3; ++i) {
        while ((1ull << bits[i]) < n[i]) ++bits[i];
        pow2 = pow2 && (1ull << bits[i]) == n[i];
    }
    perm.resize(C);
    std::vector<uint64_t> code(pow2 ? 0 : C);
    for (uint32_t iz = 0; iz < nz; ++iz)
        for (uint32_t iy = 0; iy < ny; ++iy)
            for (uint32_t ix = 0; ix < nx; ++ix) {
                const uint64_t v = ix + (uint64_t)nx * (iy + (uint64_t)ny * iz);
                const uint64_t m = morton_code(ix, iy, iz, bits);
                if (pow2) perm[v] = (uint32_t)m;
                else code[v] = m;
            }
    if (pow2) return;
    std::vector<uint32_t> order(C);
    for (uint64_t v = 0; v < C; ++v) order[v] = (uint32_t)v;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return code[a] < code[b]; });
    for (uint64_t k = 0; k < C; ++k) perm[order[k]] = (uint32_t)k;
}

// Scratch for converting caller vectors between natural and device order.
int perm_scratch(mlem_ctx* c, size_t floats) {
    if (c->pscratch_floats >= floats) return MLEM_OK;
    for (auto& p : c->pscratch) {
        if (p) { cudaFree(p); c->device_bytes -= c->pscratch_floats * 4; }
        p = nullptr;
    }
    c->pscratch_floats = 0;
    for (auto& p : c->pscratch) TRY(dev_alloc(c, &p, floats));
    c->pscratch_floats = floats;
    return MLEM_OK;
}

// Region-blocked copy for the tile size `frame_tile` (built once per tile
// size; rebuilding frees the previous copy).  Never called during capture.
int ensure_region(mlem_ctx* c, int frame_tile) {
    int rlog = 0, sblog = 0;
    uint32_t gpw = 0;
    region_params(frame_tile, c->C, &rlog, &sblog, &gpw);
    if (c->rb.el_fw && c->rb.rlog == rlog && c->rb.sblog == sblog && c->rb.gpw == gpw) return MLEM_OK;
    if (c->rb.el_fw) {
        region_free(&c->rb);
        c->device_bytes -= c->rb_bytes;
        c->rb_bytes = 0;
    }
    size_t bytes = 0;
    int line = 0;
    const cudaError_t e =
        region_build(SparseView{c->row_ptr, reinterpret_cast<const uint4*>(c->elems), c->R, c->Z},
                     c->C, rlog, sblog, gpw, &c->rb, &bytes, &line, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, e == cudaErrorMemoryAllocation ? MLEM_ERR_NOMEM : MLEM_ERR_CUDA,
                    "region-blocked build (rlog %d, sblog %d) failed at k_region.cu:%d: %s", rlog,
                    sblog, line, cudaGetErrorString(e));
    }
    c->rb_bytes = bytes;
    c->device_bytes += bytes;
    c->graph_dirty = true;
    return MLEM_OK;
}

size_t keep_words(const mlem_ctx* c) { return ((size_t)c->R + 31) / 32 + 1; }

void free_csc_act(mlem_ctx* c) {
    if (c->csc_act) { dev_free(c->csc_act); c->device_bytes -= (c->Z + 2) * 8; }
    if (c->csc_act_len) { dev_free(c->csc_act_len); c->device_bytes -= (size_t)std::max<uint32_t>(c->C, 1) * 4; }
    if (c->pos_keep) { dev_free(c->pos_keep); c->device_bytes -= keep_words(c) * 4; }
    c->csc_act = nullptr;
    c->csc_act_len = nullptr;
    c->pos_keep = nullptr;
    c->csc_act_ready = false;
}

void free_csc_vis(mlem_ctx* c) {
    free_csc_act(c);
    if (c->celems_vis) { dev_free(c->celems_vis); c->device_bytes -= (c->Z + 2) * 8; }
    if (c->row_pos) { dev_free(c->row_pos); c->device_bytes -= (size_t)std::max<uint32_t>(c->R, 1) * 4; }
    c->celems_vis = nullptr;
    c->row_pos = nullptr;
}

bool csc_by_visit(const mlem_ctx* c, const mlem_tuning& t);

// The CSC in visiting order cut to the rays with counts, for the CSC method's
// back projection under tuning t (its other entries meet calcCorrel 0 in
// every frame), from the current list of rows with counts.  The copy is made
// only when the device keeps 2 GiB free beside it; without it the back
// projection walks every entry of celems_vis.
int build_csc_act(mlem_ctx* c, const mlem_tuning& t) {
    c->csc_act_ready = false;
    if (!csc_by_visit(c, t) || !c->celems_vis || !c->row_pos || !c->act_ready || !c->sino ||
        c->Bp == 0)
        return MLEM_OK;
    if (!c->csc_act) {
        const size_t need = (c->Z + 2) * 8 + (size_t)std::max<uint32_t>(c->C, 1) * 4 +
                            keep_words(c) * 4;
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            return MLEM_OK;
        }
        if (free_b < need + (2ull << 30)) return MLEM_OK;
        int s = dev_alloc(c, &c->csc_act, c->Z + 2);
        if (s == MLEM_OK) s = dev_alloc(c, &c->csc_act_len, std::max<uint32_t>(c->C, 1));
        if (s == MLEM_OK) s = dev_alloc(c, &c->pos_keep, keep_words(c));
        if (s != MLEM_OK) {  // no room: every entry stays in the walk
            free_csc_act(c);
            c->err.clear();
            return MLEM_OK;
        }
        CK(c, cudaMemsetAsync(c->csc_act + c->Z, 0, 2 * sizeof(uint2), c->stream));
    }
    SparseView vis = csc_view(c);
    vis.pairs = reinterpret_cast<const uint4*>(c->celems_vis);
    CK(c, csc_active_build(csr_view(c), c->sino, c->Bp, vis, c->pos_keep, c->csc_act,
                           c->csc_act_len, c->stream));
    c->csc_act_ready = true;
    return MLEM_OK;
}

// The CSC in visiting order (mlem_ctx::celems_vis), built once on first use:
// the transpose keyed by every row's visiting position.  Deterministic like
// the CSC: a column's entries are summed in ascending visiting position.
int ensure_csc_vis(mlem_ctx* c) {
    if (c->celems_vis) return MLEM_OK;
    if (!c->has_csc || !c->row_order)
        return fail(c, MLEM_ERR_STATE, "the CSC in visiting order needs the CSC and the row order");
    uint64_t* col_ptr = nullptr;
    void* scratch = nullptr;
    const size_t sb = transpose_scratch_bytes(c->C);
    int s = dev_alloc(c, &c->row_pos, std::max<uint32_t>(c->R, 1));
    if (s == MLEM_OK) s = dev_alloc(c, &c->celems_vis, c->Z + 2);
    if (s == MLEM_OK) s = dev_alloc(c, &col_ptr, (size_t)c->C + 1);
    if (s == MLEM_OK) s = dev_alloc(c, &scratch, sb);
    if (s == MLEM_OK) {
        cudaError_t e = cudaMemsetAsync(c->celems_vis + c->Z, 0, 2 * sizeof(uint2), c->stream);
        if (e == cudaSuccess) e = invert_permutation(c->row_order, c->row_pos, c->R, c->stream);
        if (e == cudaSuccess)
            e = transpose(SparseView{c->row_ptr, reinterpret_cast<const uint4*>(c->elems), c->R,
                                     c->Z},
                          c->C, col_ptr, c->celems_vis, scratch, nullptr, c->stream, c->row_pos,
                          c->row_order);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            s = fail(c, e == cudaErrorMemoryAllocation ? MLEM_ERR_NOMEM : MLEM_ERR_CUDA,
                     "CSC in visiting order: %s", cudaGetErrorString(e));
        }
    }
    if (col_ptr) { dev_free(col_ptr); c->device_bytes -= ((size_t)c->C + 1) * 8; }
    if (scratch) { dev_free(scratch); c->device_bytes -= sb; }
    if (s != MLEM_OK) {
        free_csc_vis(c);
        return s;
    }
    c->graph_dirty = true;
    return MLEM_OK;
}

// The CSC method walks the CSC in visiting order with the sorted row visit.
bool csc_by_visit(const mlem_ctx* c, const mlem_tuning& t) {
    return t.bk_mode == MLEM_BK_CSC && t.visit != MLEM_VISIT_FILE && c->row_order && c->has_csc;
}

bool region_ready(const mlem_ctx* c, int frame_tile) {
    int rlog = 0, sblog = 0;
    uint32_t gpw = 0;
    region_params(frame_tile, c->C, &rlog, &sblog, &gpw);
    return c->rb.el_fw && c->rb.rlog == rlog && c->rb.sblog == sblog && c->rb.gpw == gpw;
}

// The segment table of the rows longer than kLongRowElems (one-pass method).
int build_long_rows(mlem_ctx* c) {
    std::vector<uint64_t> rp((size_t)c->R + 1);
    CK(c, cudaMemcpyAsync(rp.data(), c->row_ptr, rp.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    std::vector<LongSeg> segs;
    uint32_t n_long = 0;
    for (uint32_t r = 0; r < c->R; ++r) {
        const uint64_t b = rp[r], e = rp[(size_t)r + 1];
        if (e - b <= kLongRowElems) continue;
        for (uint64_t k = b; k < e; k += kLongSegElems)
            segs.push_back(LongSeg{k, std::min(e, k + kLongSegElems), n_long, r});
        ++n_long;
    }
    if (segs.size() > 0xffffffffull) return fail(c, MLEM_ERR_INVALID, "too many long-row segments");
    if (segs.empty()) return MLEM_OK;
    TRY(dev_alloc(c, &c->long_segs, segs.size()));
    CK(c, cudaMemcpyAsync(c->long_segs, segs.data(), segs.size() * sizeof(LongSeg),
                          cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    c->n_long_segs = (uint32_t)segs.size();
    c->n_long = n_long;
    return MLEM_OK;
}

// The natural-order and host copies of the column sums (c->norm, device
// order) and initImage's sum of them (seqcsr4mlem.cpp:55-56: a sequential
// double sum).
int norm_views(mlem_ctx* c) {
    if (c->bricked)
        CK(c, permute_to_natural(c->norm, c->norm_nat, c->perm, c->C, 1, c->stream));
    else if (c->C)
        CK(c, cudaMemcpyAsync(c->norm_nat, c->norm, (size_t)c->C * 4, cudaMemcpyDeviceToDevice,
                              c->stream));
    c->norm_host.resize(c->C);
    if (c->C)
        CK(c, cudaMemcpyAsync(c->norm_host.data(), c->norm_nat, (size_t)c->C * 4,
                              cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    double s = 0.0;
    for (uint32_t i = 0; i < c->C; ++i) s += c->norm_host[i];
    c->sumnorm = s;
    return MLEM_OK;
}

// ---------------------------------------------------------------------------
// Setup common to all create paths: validate, voxel order, CSC, column sums.
// ---------------------------------------------------------------------------
int finish_create(mlem_ctx* c) {
    // device-side validation: offsets non-decreasing, last offset == Z, columns < C
    unsigned int* bad = nullptr;
    TRY(dev_alloc(c, &bad, 1));
    CK(c, validate_csr(csr_view(c), c->C, bad, c->stream));
    unsigned int hbad = 0;
    CK(c, cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    cudaFree(bad);
    c->device_bytes -= sizeof(unsigned int);
    if (hbad & 1u) return fail(c, MLEM_ERR_MATRIX, "row offsets decrease");
    if (hbad & 2u) return fail(c, MLEM_ERR_MATRIX, "last row offset differs from nnz");
    if (hbad & 4u) return fail(c, MLEM_ERR_MATRIX, "a column index is >= the number of columns");

    const uint64_t gC = (uint64_t)c->grid[0] * c->grid[1] * c->grid[2];
    if (!(c->flags & MLEM_FLAG_NATURAL_LAYOUT) && gC == c->C && c->C > 0) {
        brick_order(c->grid[0], c->grid[1], c->grid[2], c->perm_host);
        c->iperm_host.resize(c->C);
        for (uint32_t v = 0; v < c->C; ++v) c->iperm_host[c->perm_host[v]] = v;
        TRY(dev_alloc(c, &c->perm, c->C));
        CK(c, cudaMemcpyAsync(c->perm, c->perm_host.data(), (size_t)c->C * 4,
                              cudaMemcpyHostToDevice, c->stream));
        CK(c, remap_columns(c->elems, c->Z, c->perm, c->stream));
        c->bricked = true;
    }

    if (!(c->flags & MLEM_FLAG_NO_CSC)) {
        TRY(dev_alloc(c, &c->col_ptr, (size_t)c->C + 1));
        TRY(dev_alloc(c, &c->celems, c->Z + 2));
        CK(c, cudaMemsetAsync(c->celems + c->Z, 0, 2 * sizeof(uint2), c->stream));
        void* scratch = nullptr;
        const size_t sb = transpose_scratch_bytes(c->C);
        TRY(dev_alloc(c, &scratch, sb));
        cudaError_t e = transpose(csr_view(c), c->C, c->col_ptr, c->celems, scratch,
                                  &c->max_col_len, c->stream);
        cudaFree(scratch);
        c->device_bytes -= sb;
        CK(c, e);
        c->has_csc = true;
        CK(c, column_sums_exact(csc_view(c), c->norm, c->stream));
    } else {
        CK(c, column_sums_atomic(csr_view(c), c->C, c->norm, c->stream));
    }
    TRY(dev_alloc(c, &c->norm_nat, std::max<uint32_t>(c->C, 1)));
    TRY(norm_views(c));
    TRY(dev_alloc(c, &c->counter, 64));
    // Row visiting order, from the device column indices (after the remap).
    if (!(c->flags & MLEM_FLAG_NO_ROW_ORDER) && c->R > 1) {
        uint32_t* order = nullptr;
        TRY(dev_alloc(c, &order, c->R));
        const cudaError_t e = row_order_build(csr_view(c), c->C, order, c->stream);
        if (e != cudaSuccess) {
            cudaFree(order);
            c->device_bytes -= (size_t)c->R * 4;
            CK(c, e);
        }
        c->row_order = order;
        TRY(dev_alloc(c, &c->row_ranges, c->R));
        CK(c, row_ranges_build(csr_view(c), c->row_order, c->row_ranges, c->stream));
    }
    if (c->max_row_len > kLongRowElems) TRY(build_long_rows(c));
    default_tuning(c);
    return MLEM_OK;
}

int alloc_matrix(mlem_ctx* c) {
    TRY(dev_alloc(c, &c->row_ptr, (size_t)c->R + 1));
    TRY(dev_alloc(c, &c->elems, c->Z + 2));  // even element count + one spare pair word
    TRY(dev_alloc(c, &c->norm, (size_t)std::max<uint32_t>(c->C, 1)));
    CK(c, cudaMemsetAsync(c->row_ptr, 0, 8, c->stream));
    CK(c, cudaMemsetAsync(c->elems + c->Z, 0, 2 * sizeof(uint2), c->stream));
    return MLEM_OK;
}

int new_ctx(mlem_ctx** out, uint32_t R, uint32_t C, uint64_t Z, uint32_t flags, int device) {
    *out = nullptr;
    int n_dev = 0;
    cudaError_t e = cudaGetDeviceCount(&n_dev);
    if (e != cudaSuccess || n_dev == 0)
        return fail(nullptr, MLEM_ERR_CUDA, "no CUDA device available (%s)",
                    e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
    if (device < 0 || device >= n_dev)
        return fail(nullptr, MLEM_ERR_INVALID, "device %d out of range (%d devices)", device, n_dev);
    if (flags & ~(MLEM_FLAG_EXACT | MLEM_FLAG_NO_CSC | MLEM_FLAG_CHECKED | MLEM_FLAG_NATURAL_LAYOUT |
                  MLEM_FLAG_NO_ROW_ORDER | MLEM_FLAG_EXPAND_SYMMETRY | MLEM_FLAG_MIRROR_KERNELS))
        return fail(nullptr, MLEM_ERR_INVALID, "unknown flags 0x%x", flags);
    if ((flags & MLEM_FLAG_EXACT) && (flags & MLEM_FLAG_NO_CSC))
        return fail(nullptr, MLEM_ERR_INVALID, "MLEM_FLAG_EXACT needs the CSC copy");
    if ((flags & MLEM_FLAG_EXACT) && (flags & MLEM_FLAG_MIRROR_KERNELS))
        return fail(nullptr, MLEM_ERR_INVALID,
                    "MLEM_FLAG_EXACT needs the full matrix (MLEM_FLAG_EXPAND_SYMMETRY), not "
                    "MLEM_FLAG_MIRROR_KERNELS");
    mlem_ctx* c = new mlem_ctx();
    c->device = device;
    c->R = R;
    c->C = C;
    c->Z = Z;
    c->flags = flags;
    int s = set_device(c);
    c->n_sm = sm_count(device);
    if (s == MLEM_OK) {
        cudaError_t e2 = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
        if (e2 != cudaSuccess) s = fail(c, MLEM_ERR_CUDA, "stream: %s", cudaGetErrorString(e2));
        c->stream = c->own_stream;
    }
    if (s != MLEM_OK) {
        global_error() = c->err;
        mlem_destroy(c);
        return s;
    }
    *out = c;
    return MLEM_OK;
}

// ---------------------------------------------------------------------------
// Frames.
// ---------------------------------------------------------------------------
int ensure_stage(mlem_ctx* c, size_t bytes) {
    if (c->stage_bytes >= bytes) return MLEM_OK;
    if (c->stage) { cudaFree(c->stage); c->device_bytes -= c->stage_bytes; }
    c->stage = nullptr;
    c->stage_bytes = 0;
    TRY(dev_alloc(c, &c->stage, bytes));
    c->stage_bytes = bytes;
    return MLEM_OK;
}

void free_frames(mlem_ctx* c) {
    for (void* p : {(void*)c->sino, (void*)c->x, (void*)c->correl, (void*)c->update,
                    (void*)c->stats_scratch, (void*)c->inits_dev, (void*)c->f_long,
                    (void*)c->sino_alt})
        dev_free(p);
    if (c->graph_alt) cudaGraphExecDestroy(c->graph_alt);
    c->graph_alt = nullptr;
    c->sino_alt = nullptr;
    c->sino = nullptr; c->x = nullptr; c->correl = nullptr; c->update = nullptr;
    c->stats_scratch = nullptr; c->inits_dev = nullptr; c->f_long = nullptr;
    c->B = c->Bp = 0;
    c->images_ready = false;
    c->act_ready = false;
}

int alloc_frames(mlem_ctx* c, uint32_t B) {
    const uint32_t Bp = padded_frames(B);
    if (B == 0 || Bp == 0) return fail(c, MLEM_ERR_INVALID, "n_frames must be 1..64 (got %u)", B);
    if (c->B == B && c->sino) return MLEM_OK;
    free_frames(c);
    c->B = B;
    c->Bp = Bp;
    TRY(dev_alloc(c, &c->sino, (size_t)c->R * Bp));
    TRY(dev_alloc(c, &c->x, (size_t)c->C * Bp));
    TRY(dev_alloc(c, &c->correl, (size_t)c->R * Bp));
    TRY(dev_alloc(c, &c->update, (size_t)c->C * Bp));
    TRY(dev_alloc(c, &c->stats_scratch, stats_scratch_bytes(Bp)));
    TRY(dev_alloc(c, &c->inits_dev, Bp));
    if (c->n_long) TRY(dev_alloc(c, &c->f_long, (size_t)c->n_long * Bp));
    CK(c, cudaMemsetAsync(c->sino, 0, (size_t)c->R * Bp * 4, c->stream));
    CK(c, cudaMemsetAsync(c->x, 0, (size_t)c->C * Bp * 4, c->stream));
    CK(c, cudaMemsetAsync(c->correl, 0, (size_t)c->R * Bp * 4, c->stream));
    CK(c, cudaMemsetAsync(c->update, 0, (size_t)c->C * Bp * 4, c->stream));
    c->tuning.frame_tile = std::min(c->tuning.frame_tile > 0 ? c->tuning.frame_tile : 16,
                                    default_tile(Bp));
    c->graph_dirty = true;
    return MLEM_OK;
}

// Frame-major host [B][n] -> interleaved device [n][Bp] (pad frames untouched).
template <typename T>
int upload_frames(mlem_ctx* c, const T* host, T* dev, uint64_t n) {
    const bool voxels = std::is_same<T, float>::value && c->bricked;
    if (c->Bp == 1 && !voxels) {
        CK(c, cudaMemcpyAsync(dev, host, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
        return MLEM_OK;
    }
    TRY(ensure_stage(c, n * c->B * sizeof(T)));
    CK(c, cudaMemcpyAsync(c->stage, host, n * c->B * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    if (std::is_same<T, int32_t>::value)
        CK(c, interleave_i32(reinterpret_cast<const int32_t*>(c->stage),
                             reinterpret_cast<int32_t*>(dev), n, c->B, c->Bp, c->stream));
    else
        CK(c, interleave_f32(reinterpret_cast<const float*>(c->stage),
                             reinterpret_cast<float*>(dev), n, c->B, c->Bp,
                             voxels ? c->perm : nullptr, c->stream));
    return MLEM_OK;
}

int download_images(mlem_ctx* c, float* host) {
    if (c->Bp == 1 && !c->bricked) {
        CK(c, cudaMemcpyAsync(host, c->x, (size_t)c->C * 4, cudaMemcpyDeviceToHost, c->stream));
        return MLEM_OK;
    }
    TRY(ensure_stage(c, (size_t)c->C * c->B * 4));
    float* st = static_cast<float*>(c->stage);
    CK(c, deinterleave_f32(c->x, st, c->C, c->B, c->Bp, c->bricked ? c->perm : nullptr, c->stream));
    CK(c, cudaMemcpyAsync(host, st, (size_t)c->C * c->B * 4, cudaMemcpyDeviceToHost, c->stream));
    return MLEM_OK;
}

// The one-pass iteration's sorted visiting list without the rows whose counts
// are zero in every frame (active_rows_build), rebuilt whenever the
// sinograms change.  Contexts without a row order and the bit-exact mode
// keep every row; so does a context with no room for the list.  read_back:
// wait for the list and record its size (mlem_info.rows_with_counts).  cut:
// also refill the CSC method's copy cut to the rays with counts (made where
// several iterations follow the sinograms; dropped otherwise).
int build_active_list(mlem_ctx* c, bool read_back, bool cut) {
    c->act_ready = false;
    c->csc_act_ready = false;
    // the mirrored kernels walk stored rows, whose counts are the mirrored rows'
    if (!c->row_order || (c->flags & MLEM_FLAG_EXACT) || c->mirrored || c->R == 0 ||
        c->R > 0x7fffffffu)
        return MLEM_OK;
    if (!c->act_tmp) {
        const size_t tb = active_rows_tmp_bytes(c->R);
        int s = MLEM_OK;
        if (!c->act_order) s = dev_alloc(c, &c->act_order, c->R);
        if (s == MLEM_OK && !c->act_ranges) s = dev_alloc(c, &c->act_ranges, c->R);
        if (s == MLEM_OK && !c->act_n) s = dev_alloc(c, &c->act_n, 1);
        if (s == MLEM_OK && !c->act_z) s = dev_alloc(c, &c->act_z, 1);
        if (s == MLEM_OK) s = dev_alloc(c, &c->act_tmp, tb);
        if (s != MLEM_OK) {  // no room: every row stays in the walk
            c->err.clear();
            return MLEM_OK;
        }
        c->act_tmp_bytes = tb;
    }
    CK(c, active_rows_build(csr_view(c), c->sino, c->Bp, c->act_tmp,
                            c->act_tmp_bytes, c->act_order, c->act_ranges, c->act_n, c->act_z,
                            c->stream));
    if (read_back) {
        uint32_t n = 0;
        unsigned long long z = 0;
        CK(c, cudaMemcpyAsync(&n, c->act_n, 4, cudaMemcpyDeviceToHost, c->stream));
        CK(c, cudaMemcpyAsync(&z, c->act_z, 8, cudaMemcpyDeviceToHost, c->stream));
        CK(c, cudaStreamSynchronize(c->stream));
        c->act_rows = n;
        c->act_nnz = z;
    }
    c->act_ready = true;
    return cut ? build_csc_act(c, c->tuning) : MLEM_OK;
}

// The subsets' sorted lists without their rows without counts (ordered
// subsets walk them with the sorted visits); needs the main list's buffers.
int build_subset_lists(mlem_ctx* c) {
    c->sub_act_ready = false;
    if (c->n_subsets < 2 || !c->sub_sorted || !c->sub_act_order || !c->act_ready || !c->act_tmp)
        return MLEM_OK;
    for (uint32_t k = 0; k < c->n_subsets; ++k) {
        SparseView v = csr_view(c);
        const uint64_t o = c->sub_off[k];
        v.order = c->sub_sorted + o;
        v.vrange = c->sub_sorted_ranges + o;
        v.n = (uint32_t)(c->sub_off[k + 1] - o);
        CK(c, active_rows_build(v, c->sino, c->Bp, c->act_tmp, c->act_tmp_bytes,
                                c->sub_act_order + o, c->sub_act_ranges + o, c->sub_act_n + k,
                                c->sub_act_z + k, c->stream));
    }
    c->sub_act_ready = true;
    return MLEM_OK;
}

// A captured iteration holds the list or the full visiting order: capture
// again when that changes (not when the list is only rebuilt in place).
int build_active(mlem_ctx* c, bool read_back, bool cut) {
    const bool was = c->act_ready, sub_was = c->sub_act_ready, csc_was = c->csc_act_ready;
    int s = build_active_list(c, read_back, cut);
    if (s == MLEM_OK) s = build_subset_lists(c);
    if (c->act_ready != was || c->sub_act_ready != sub_was || c->csc_act_ready != csc_was)
        c->graph_dirty = true;
    return s;
}

// ---------------------------------------------------------------------------
// One MLEM iteration (seqcsr4mlem.cpp:164-167) plus the image statistics.
// ---------------------------------------------------------------------------

int mark(mlem_ctx* c, const PhaseEvents* pe, int i) {
    if (pe) CK(c, cudaEventRecord(pe->ev[i], c->stream));
    return MLEM_OK;
}

// The CSR as the row kernels of tuning t walk it.
SparseView csr_visit(const mlem_ctx* c, const mlem_tuning& t) {
    SparseView v = csr_view(c);
    if (t.visit == MLEM_VISIT_FILE) {
        v.order = nullptr;
        v.vrange = nullptr;
    }
    return v;
}

// MLEM_VISIT_SORTED_CHUNKED: resident CTAs per SM (blocks_per_sm 1, 2 or 4
// picks CTAs of 1024, 512 or 256 threads; larger values mean 4) and rows per
// chunk: about 16 chunks for every resident CTA (measured best on the
// plain-full matrix with 16 frames), at least 32 rows.
int chunk_ctas_per_sm(const mlem_tuning& t) {
    return t.blocks_per_sm <= 1 ? 1 : t.blocks_per_sm == 2 ? 2 : 4;
}
// MLEM_VISIT_SORTED_STAGED: 1..4 resident CTAs of 256 threads per SM.
int staged_ctas_per_sm(const mlem_tuning& t) { return std::min(4, std::max(1, t.blocks_per_sm)); }
bool chunk_visit(int visit) {
    return visit == MLEM_VISIT_SORTED_CHUNKED || visit == MLEM_VISIT_SORTED_STAGED;
}
uint32_t chunk_rows_of(const mlem_ctx* c, const mlem_tuning& t, uint64_t rows) {
    const uint64_t ctas = (uint64_t)c->n_sm * (t.visit == MLEM_VISIT_SORTED_STAGED
                                                   ? staged_ctas_per_sm(t)
                                                   : chunk_ctas_per_sm(t));
    (void)c;
    return (uint32_t)std::max<uint64_t>(32, (rows + ctas * 16 - 1) / (ctas * 16));
}

// The rows of subset s as the row kernels of tuning t walk them: the subset's
// visiting list (sorted for the sorted visits when the row order exists, else
// file order) as the view's order.
SparseView subset_view(const mlem_ctx* c, const mlem_tuning& t, uint32_t s) {
    SparseView v = csr_view(c);
    const bool sorted = t.visit != MLEM_VISIT_FILE && c->sub_sorted;
    const uint64_t o = c->sub_off[s];
    v.order = (sorted ? c->sub_sorted : c->sub_file) + o;
    v.vrange = (sorted ? c->sub_sorted_ranges : c->sub_file_ranges) + o;
    v.n = (uint32_t)(c->sub_off[s + 1] - o);
    return v;
}

// One-pass method over the rows of `csr` (all rows, or one subset's): u +=
// A^T calcCorrel(sino, A x) for B interleaved frames.  `counter` is the work
// counter of the chunked and staged walks.
int fused_pass(mlem_ctx* c, const mlem_tuning& t, const SparseView& csr, const float* x,
               const int32_t* sino, float* u, uint32_t B, unsigned int* counter,
               cudaStream_t st) {
    const uint32_t T = (uint32_t)t.frame_tile;
    if (t.visit == MLEM_VISIT_SORTED_STAGED)
        CK(c, fused_staged(csr, x, B, t.frame_tile, sino, u, chunk_rows_of(c, t, csr.n),
                           staged_ctas_per_sm(t), counter, c->n_sm, st));
    else if (t.visit == MLEM_VISIT_SORTED_CHUNKED)
        CK(c, fused_chunked(csr, x, B, t.frame_tile, sino, u, chunk_rows_of(c, t, csr.n),
                            chunk_ctas_per_sm(t), counter, c->n_sm, st));
    else
        for (uint32_t f0 = 0; f0 < B; f0 += T)
            CK(c, fused_row(csr, x, B, f0, sino, u, cfg_of(c, t), st));
    return MLEM_OK;
}
int fused_pass(mlem_ctx* c, const mlem_tuning& t, const SparseView& csr, cudaStream_t st) {
    return fused_pass(c, t, csr, c->x, c->sino, c->update, c->Bp, c->counter, st);
}

int enqueue_iteration(mlem_ctx* c, const mlem_tuning& t, bool stats,
                      const PhaseEvents* pe = nullptr) {
    const SparseView csr = csr_visit(c, t);
    const uint32_t Bp = c->Bp;
    cudaStream_t st = c->stream;
    TRY(mark(c, pe, 0));
    if (c->flags & MLEM_FLAG_EXACT) {
        CK(c, fwproj_exact(csr, c->x, Bp, c->sino, c->correl, nullptr, st));
        TRY(mark(c, pe, 1));
        CK(c, bkproj_exact(csc_view(c), c->correl, Bp, c->norm, c->x, nullptr, st));
        TRY(mark(c, pe, 2));
    } else {
        const LaunchCfg cfg = cfg_of(c, t);
        const uint32_t T = (uint32_t)t.frame_tile;
        if (c->n_subsets > 1 && t.bk_mode != MLEM_BK_FUSED)
            return fail(c, MLEM_ERR_STATE,
                        "ordered subsets run on the one-pass method (MLEM_BK_FUSED), not mode %d",
                        t.bk_mode);
        if (c->mirrored != (t.bk_mode == MLEM_BK_MIRRORED))
            return fail(c, MLEM_ERR_STATE, c->mirrored
                            ? "a context made with MLEM_FLAG_MIRROR_KERNELS runs MLEM_BK_MIRRORED only"
                            : "MLEM_BK_MIRRORED needs a context made with MLEM_FLAG_MIRROR_KERNELS");
        switch (t.bk_mode) {
            case MLEM_BK_CSC: {
                if (!c->has_csc) return fail(c, MLEM_ERR_STATE, "no CSC copy (MLEM_FLAG_NO_CSC)");
                // with a sorted visit: correlations by visiting position, and the
                // CSC that lists each column's rays in that order
                const bool by_visit = csc_by_visit(c, t);
                if (by_visit && !c->celems_vis)
                    return fail(c, MLEM_ERR_STATE, "the CSC in visiting order is not built");
                SparseView fw = csr;
                SparseView bk = csc_view(c);
                if (by_visit) {
                    fw.out_by_visit = true;
                    bk.pairs = reinterpret_cast<const uint4*>(c->celems_vis);
                    if (c->act_ready && c->row_pos) {
                        // walk only the rows with counts; the others keep calcCorrel 0
                        fw.order = c->act_order;
                        fw.vrange = c->act_ranges;
                        fw.n_dev = c->act_n;
                        fw.out_pos = c->row_pos;
                        CK(c, cudaMemsetAsync(c->correl, 0, (size_t)c->R * Bp * 4, st));
                        if (c->csc_act_ready) {  // and only the entries of those rows
                            bk.pairs = reinterpret_cast<const uint4*>(c->csc_act);
                            bk.len = c->csc_act_len;
                        }
                    }
                }
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, fwproj(fw, c->x, Bp, f0, c->sino, c->correl, nullptr, cfg, st));
                TRY(mark(c, pe, 1));
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, bkproj_csc(bk, c->correl, Bp, f0, c->norm, c->x, nullptr, cfg, st));
                TRY(mark(c, pe, 2));
                break;
            }
            case MLEM_BK_ATOMIC:
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, fwproj(csr, c->x, Bp, f0, c->sino, c->correl, nullptr, cfg, st));
                TRY(mark(c, pe, 1));
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, bkproj_scatter(csr, c->correl, Bp, f0, c->update, cfg, st));
                TRY(mark(c, pe, 2));
                CK(c, apply_update(c->x, c->update, c->norm, c->C, Bp, true, st));
                break;
            case MLEM_BK_FUSED:
                if (c->n_subsets > 1) {
                    // ordered subsets: a one-pass sub-iteration and its update per
                    // subset; the sorted visits walk each subset's rows with counts
                    for (uint32_t s = 0; s < c->n_subsets; ++s) {
                        SparseView v = subset_view(c, t, s);
                        if (c->sub_act_ready && t.visit != MLEM_VISIT_FILE) {
                            v.order = c->sub_act_order + c->sub_off[s];
                            v.vrange = c->sub_act_ranges + c->sub_off[s];
                            v.n_dev = c->sub_act_n + s;
                        }
                        TRY(fused_pass(c, t, v, st));
                        CK(c, apply_update_subset(c->x, c->update, c->sub_norm + (size_t)s * c->C,
                                                  c->norm, c->C, Bp, st));
                    }
                    TRY(mark(c, pe, 1));
                    TRY(mark(c, pe, 2));
                    break;
                }
                {
                    // sorted visits walk only the rows with counts (their list is
                    // rebuilt with every new sinogram); the long rows are cut into
                    // segments for their own kernels
                    SparseView v = csr;
                    if (c->act_ready && t.visit != MLEM_VISIT_FILE) {
                        v.order = c->act_order;
                        v.vrange = c->act_ranges;
                        v.n_dev = c->act_n;
                    }
                    if (c->n_long) v.long_len = kLongRowElems;
                    TRY(fused_pass(c, t, v, st));
                    if (c->n_long)
                        CK(c, long_rows_pass(csr, c->long_segs, c->n_long_segs, c->n_long, c->x,
                                             Bp, t.frame_tile, c->sino, c->f_long, c->update,
                                             c->n_sm, st));
                }
                TRY(mark(c, pe, 1));
                TRY(mark(c, pe, 2));
                CK(c, apply_update(c->x, c->update, c->norm, c->C, Bp, true, st));
                break;
            case MLEM_BK_REGION:
                if (!region_ready(c, t.frame_tile))
                    return fail(c, MLEM_ERR_STATE, "region-blocked copy not built for this frame tile");
                CK(c, cudaMemsetAsync(c->correl, 0, (size_t)c->R * Bp * 4, st));
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, region_fwproj(c->rb, c->x, Bp, f0, c->C, c->correl, cfg, st));
                CK(c, correl_inplace(c->correl, c->sino, (uint64_t)c->R * Bp, st));
                TRY(mark(c, pe, 1));
                // back projection with calcUpdate applied per region (no update vector)
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, region_bkproj_update(c->rb, c->correl, Bp, f0, c->C, c->norm, c->x, cfg, st));
                TRY(mark(c, pe, 2));
                break;
            case MLEM_BK_MIRRORED:
                // per-row sums of the full matrix (correl holds them), then the scatter
                CK(c, cudaMemsetAsync(c->correl, 0, (size_t)c->R * Bp * 4, st));
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, mirror_fwproj(csr, c->mirror, c->x, Bp, f0, t.frame_tile, c->correl,
                                        c->n_sm, t.blocks_per_sm, st));
                TRY(mark(c, pe, 1));
                for (uint32_t f0 = 0; f0 < Bp; f0 += T)
                    CK(c, mirror_bkproj(csr, c->mirror, c->correl, c->sino, Bp, f0, t.frame_tile,
                                        c->update, c->n_sm, t.blocks_per_sm, st));
                TRY(mark(c, pe, 2));
                CK(c, apply_update(c->x, c->update, c->norm, c->C, Bp, true, st));
                break;
            default:
                return fail(c, MLEM_ERR_INVALID, "unknown back-projection mode %d", t.bk_mode);
        }
    }
    TRY(mark(c, pe, 3));
    if (stats)
        CK(c, image_stats(c->x, c->C, Bp, c->B, c->stats_scratch, c->stats_slot, c->hist_sums,
                          c->hist_zeros, c->hist_subn, st));
    TRY(mark(c, pe, 4));
    return MLEM_OK;
}

// Algorithmic bytes of each phase per iteration: every matrix element and
// offset once per pass over the matrix (one pass per frame tile), every
// vector entry once per read or write, for the B real frames.
}  // namespace

namespace mlem {
void phase_bytes_for(const mlem_ctx* c, int bk_mode, int frame_tile, double* bytes,
                     int* launches, bool active_rows) {
    const double C = c->C, B = c->B;
    // the one-pass sorted walk, and the CSC method's forward pass over the CSC
    // in visiting order, visit only the rows with counts
    const bool csc_act = bk_mode == MLEM_BK_CSC && c->row_pos && csc_by_visit(c, c->tuning);
    const bool act = active_rows && c->act_ready && (bk_mode == MLEM_BK_FUSED || csc_act) &&
                     c->n_subsets == 1 && !(c->flags & MLEM_FLAG_EXACT);
    const double R = act ? (double)c->act_rows : (double)c->R;
    const double Z = act ? (double)c->act_nnz : (double)c->Z;
    const bool exact = (c->flags & MLEM_FLAG_EXACT) != 0;
    const int mode = exact ? MLEM_BK_CSC : bk_mode;
    const double tiles = exact ? 1.0 : (double)(c->Bp / (uint32_t)frame_tile);
    const double csr_pass = 8.0 * (R + 1) + 8.0 * Z;
    // every column; every element, or those of the rows with counts (csc_act)
    const double csc_pass = act && csc_act && c->csc_act_ready
                                ? 8.0 * (C + 1) + 4.0 * C + 8.0 * (double)c->act_nnz
                                : 8.0 * (C + 1) + 8.0 * (double)c->Z;
    for (int p = 0; p < MLEM_N_PHASES; ++p) { bytes[p] = 0.0; launches[p] = 0; }
    const int nt = (int)tiles;
    if (mode == MLEM_BK_REGION) {
        // one region-major element copy and the segment rows per pass; per
        // segment one partial (forward) or one correlation (backward) of B
        // floats; x once, fw zeroing + correl pass over R x B
        const double S = (double)c->rb.nseg, ZR = (double)c->rb.nel, ZB = (double)c->rb.nel_bk;
        bytes[0] = tiles * (8.0 * ZR + 4.0 * S) + B * (4.0 * C + 4.0 * S) + B * 16.0 * R;
        bytes[1] = tiles * (8.0 * ZB + 4.0 * S) + B * (4.0 * S + 8.0 * C) + 4.0 * C;  // c per segment, x r/w, norm
        launches[0] = nt + 1;
        launches[1] = nt;
        bytes[3] = 4.0 * C * B;
        launches[3] = 2;
        return;
    }
    if (mode == MLEM_BK_MIRRORED) {
        // the stored matrix once per pass and frame tile; forward: x, the row
        // sums zeroed and written; backward: sinogram and row sums, update
        bytes[0] = tiles * csr_pass + B * (4.0 * C + 8.0 * R);
        bytes[1] = tiles * csr_pass + B * (8.0 * R + 4.0 * C);
        launches[0] = nt;
        launches[1] = nt;
        bytes[3] = 4.0 * C * B;
        launches[3] = 2;
        bytes[2] = 4.0 * C + B * (4.0 * C + 8.0 * C + 4.0 * C);  // norm, update, x r/w, zeroing
        launches[2] = 1;
        return;
    }
    if (mode == MLEM_BK_FUSED && !exact && c->n_subsets > 1) {
        // ordered subsets: the matrix once, x and the update once per subset,
        // and per subset an update pass (norm_s, norm, u and x r/w) inside phase 0
        const double S = (double)c->n_subsets;
        bytes[0] = tiles * csr_pass + B * 4.0 * R + S * B * 8.0 * C +
                   S * (8.0 * C + B * 16.0 * C);
        launches[0] = (int)S * ((chunk_visit(c->tuning.visit) ? 1 : nt) + 1);
        bytes[3] = 4.0 * C * B;
        launches[3] = 2;
        return;
    }
    if (mode == MLEM_BK_FUSED) {
        bytes[0] = tiles * csr_pass + B * (4.0 * C + 4.0 * R + 4.0 * C);  // x, sino, update
        launches[0] = (!exact && chunk_visit(c->tuning.visit)) ? 1 : nt;
        if (!exact && c->n_long) launches[0] += 2;  // the long-row kernels
    } else {
        bytes[0] = tiles * csr_pass + B * (4.0 * C + 4.0 * R + 4.0 * R);  // x, sino, correl
        if (act && csc_act) bytes[0] += B * 4.0 * (double)c->R;  // the correlations zeroed
        launches[0] = exact ? 1 : nt;
    }
    if (mode == MLEM_BK_CSC) {
        bytes[1] = tiles * (csc_pass + 4.0 * C) + B * (4.0 * R + 8.0 * C);  // norm, correl, x r/w
        launches[1] = exact ? 1 : nt;
    } else if (mode == MLEM_BK_ATOMIC) {
        bytes[1] = tiles * csr_pass + B * (4.0 * R + 4.0 * C);  // correl, update
        launches[1] = nt;
    }
    if (mode != MLEM_BK_CSC) {
        bytes[2] = 4.0 * C + B * (4.0 * C + 8.0 * C + 4.0 * C);  // norm, update, x r/w, zeroing
        launches[2] = 1;
    }
    bytes[3] = 4.0 * C * B;
    launches[3] = 2;
}

void voxel_permutation(uint32_t nx, uint32_t ny, uint32_t nz, std::vector<uint32_t>& perm) {
    brick_order(nx, ny, nz, perm);
}
}  // namespace mlem

namespace {

void phase_bytes(const mlem_ctx* c, double* bytes, int* launches) {
    phase_bytes_for(c, c->tuning.bk_mode, c->tuning.frame_tile, bytes, launches,
                    c->tuning.visit != MLEM_VISIT_FILE);
}

}  // namespace

namespace mlem {
int ensure_history(mlem_ctx* c, int n) {
    if (!c->stats_slot) TRY(dev_alloc(c, &c->stats_slot, 1));
    if (c->hist_cap >= n && c->hist_sums) return MLEM_OK;
    dev_free(c->hist_sums); dev_free(c->hist_zeros); dev_free(c->hist_subn);
    c->hist_sums = nullptr; c->hist_zeros = nullptr; c->hist_subn = nullptr;
    const int cap = std::max(n, 64);
    TRY(dev_alloc(c, &c->hist_sums, (size_t)cap * 64));
    TRY(dev_alloc(c, &c->hist_zeros, (size_t)cap * 64));
    TRY(dev_alloc(c, &c->hist_subn, (size_t)cap * 64));
    c->hist_cap = cap;
    c->graph_dirty = true;  // graphs hold the history pointers
    return MLEM_OK;
}
}  // namespace mlem

namespace {

// Drops the iteration graph and the streaming steps' second one (any new
// capture of the first invalidates the second).
void drop_graph(mlem_ctx* c) {
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->graph_alt) cudaGraphExecDestroy(c->graph_alt);
    c->graph = nullptr;
    c->graph_alt = nullptr;
    c->graph_iters = 0;
}

// Capture `n` iterations (slot reset + n x (iteration + statistics)) into *out.
int capture_into(mlem_ctx* c, int n, cudaGraphExec_t* out) {
    CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int s = MLEM_OK;
    cudaError_t e = cudaMemsetAsync(c->stats_slot, 0, sizeof(unsigned int), c->stream);
    if (e != cudaSuccess) s = fail(c, MLEM_ERR_CUDA, "capture memset: %s", cudaGetErrorString(e));
    for (int i = 0; i < n && s == MLEM_OK; ++i) s = enqueue_iteration(c, c->tuning, true);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    if (s != MLEM_OK) { if (g) cudaGraphDestroy(g); return s; }
    if (e2 != cudaSuccess) return fail(c, MLEM_ERR_CUDA, "end capture: %s", cudaGetErrorString(e2));
    e2 = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
        *out = nullptr;
        return fail(c, MLEM_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e2));
    }
    return MLEM_OK;
}

int capture(mlem_ctx* c, int n) {
    drop_graph(c);
    TRY(capture_into(c, n, &c->graph));
    c->graph_iters = n;
    c->graph_dirty = false;
    return MLEM_OK;
}

int ensure_tmp(mlem_ctx* c) {
    if (c->tmp_r[0]) return MLEM_OK;
    for (auto& p : c->tmp_r) TRY(dev_alloc(c, &p, std::max<uint32_t>(c->R, 1)));
    for (auto& p : c->tmp_c) TRY(dev_alloc(c, &p, std::max<uint32_t>(c->C, 1)));
    TRY(dev_alloc(c, &c->tmp_sino, std::max<uint32_t>(c->R, 1)));
    return MLEM_OK;
}

LaunchCfg cfg_for_frames(const mlem_ctx* c, uint32_t B) {
    LaunchCfg cfg = cfg_of(c, c->tuning);
    int t = 1;
    for (int v : {16, 8, 4, 2})
        if (B % v == 0) { t = v; break; }
    cfg.frame_tile = t;
    return cfg;
}

// Mirrors applied in the kernels (MLEM_FLAG_MIRROR_KERNELS), set up on a
// context that holds the stored matrix: the detector maps of the identity
// and the header's mirrors (generateSyms order), the device voxel maps, and
// the full matrix's column sums in place of the stored matrix's.
int mirror_setup(mlem_ctx* c, const mlem_symmetry& sym, uint32_t nC) {
    std::vector<uint32_t> lut8;
    sym_detector_luts(sym.n_layers, sym.n_blocks, sym.block_size, sym.n_rings, lut8);
    std::vector<uint32_t> ids = {0u};
    for (uint32_t m : sym_mirrors(sym.sym)) ids.push_back(m);
    MirrorView mv;
    mv.n = (uint32_t)ids.size();
    mv.n_crystals = nC;
    mv.C = c->C;
    std::vector<uint32_t> lut((size_t)mv.n * nC);
    for (uint32_t j = 0; j < mv.n; ++j)
        std::copy(lut8.begin() + (size_t)ids[j] * nC, lut8.begin() + (size_t)(ids[j] + 1) * nC,
                  lut.begin() + (size_t)j * nC);
    TRY(dev_alloc(c, &c->mirror_lut, lut.size()));
    CK(c, cudaMemcpyAsync(c->mirror_lut, lut.data(), lut.size() * 4, cudaMemcpyHostToDevice,
                          c->stream));
    mv.lut = c->mirror_lut;
    const uint32_t nx = c->grid[0], ny = c->grid[1], nz = c->grid[2];
    int bits[3] = {0, 0, 0};
    bool pow2 = true;
    for (int i = 0; i < 3; ++i) {
        while ((1ull << bits[i]) < c->grid[i]) ++bits[i];
        pow2 = pow2 && (1ull << bits[i]) == c->grid[i];
    }
    std::vector<uint32_t> vox;
    if (c->bricked && pow2) {
        // the device index is the Morton code itself: a mirror flips one axis's bits
        const uint64_t mx = morton_code(nx - 1, 0, 0, bits), my = morton_code(0, ny - 1, 0, bits),
                       mz = morton_code(0, 0, nz - 1, bits);
        for (uint32_t j = 0; j < mv.n; ++j)
            mv.xor_mask[j] = (uint32_t)(((ids[j] & 1u) ? mx : 0) | ((ids[j] & 2u) ? my : 0) |
                                        ((ids[j] & 4u) ? mz : 0));
    } else {
        vox.resize((size_t)mv.n * c->C);
        const uint64_t slice = (uint64_t)nx * ny;
        for (uint32_t j = 0; j < mv.n; ++j)
            for (uint32_t d = 0; d < c->C; ++d) {
                const uint32_t v = c->bricked ? c->iperm_host[d] : d;
                uint32_t z = (uint32_t)(v / slice);
                const uint32_t rem = (uint32_t)(v - z * slice);
                uint32_t y = rem / nx, x = rem - y * nx;
                if (ids[j] & 1u) x = nx - 1 - x;
                if (ids[j] & 2u) y = ny - 1 - y;
                if (ids[j] & 4u) z = nz - 1 - z;
                const uint32_t w = (uint32_t)(z * slice + (uint64_t)y * nx + x);
                vox[(size_t)j * c->C + d] = c->bricked ? c->perm_host[w] : w;
            }
        TRY(dev_alloc(c, &c->mirror_vox, vox.size()));
        CK(c, cudaMemcpyAsync(c->mirror_vox, vox.data(), vox.size() * 4, cudaMemcpyHostToDevice,
                              c->stream));
        mv.vox = c->mirror_vox;
    }
    c->mirror = mv;
    float* full = nullptr;
    TRY(dev_alloc(c, &full, std::max<uint32_t>(c->C, 1)));
    cudaError_t e = mirror_norm(c->norm, mv, full, c->stream);
    if (e == cudaSuccess && c->C)
        e = cudaMemcpyAsync(c->norm, full, (size_t)c->C * 4, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // lut and vox leave scope
    dev_free(full);
    c->device_bytes -= (uint64_t)std::max<uint32_t>(c->C, 1) * 4;
    CK(c, e);
    TRY(norm_views(c));
    c->mirrored = true;
    c->tuning.bk_mode = MLEM_BK_MIRRORED;
    c->tuning.group = 32;
    c->tuning.visit = c->row_order ? MLEM_VISIT_SORTED : MLEM_VISIT_FILE;
    c->tuning.blocks_per_sm = 8;
    return MLEM_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* mlem_last_error(const mlem_ctx* ctx) {
    return ctx ? ctx->err.c_str() : global_error().c_str();
}
const char* mlem_global_error(void) { return global_error().c_str(); }
int mlem_version(void) { return MLEM_B200_VERSION; }

const char* mlem_status_string(int s) {
    switch (s) {
        case MLEM_OK: return "ok";
        case MLEM_ERR_INVALID: return "invalid argument";
        case MLEM_ERR_CUDA: return "CUDA error";
        case MLEM_ERR_IO: return "I/O error";
        case MLEM_ERR_FORMAT: return "bad file format";
        case MLEM_ERR_NOMEM: return "out of memory";
        case MLEM_ERR_STATE: return "call out of order";
        case MLEM_ERR_MATRIX: return "invalid matrix";
        case MLEM_NO_CHECKPOINT: return "no checkpoint";
        default: return "unknown status";
    }
}

namespace {
// Host-to-device copy of a large pageable array (a matrix's elements, often a
// file mapping): host threads copy 16 MiB chunks into a ring of page-locked
// buffers, two per thread, and each chunk goes out with its own
// cudaMemcpyAsync as soon as it is filled, so the threads' page faults and
// copies overlap one another and the copy engine.  Returns once the copies
// have finished.  Small arrays, and hosts where page-locked memory cannot be
// had, take one plain copy.
cudaError_t upload_pageable(int device, cudaStream_t st, void* dst, const void* src, size_t bytes) {
    constexpr size_t kChunk = size_t(16) << 20;
    const int T = (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
    auto plain = [&]() {
        const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
        return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
    };
    if (bytes < 8 * kChunk || T < 2) return plain();
    const int K = 2 * T;
    unsigned char* ring = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&ring), (size_t)K * kChunk, cudaHostAllocDefault) !=
        cudaSuccess) {
        cudaGetLastError();
        return plain();
    }
    std::vector<cudaEvent_t> ev(K, nullptr);
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < K && e == cudaSuccess; ++b)
        e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
    const size_t n = (bytes + kChunk - 1) / kChunk;
    const unsigned char* from = static_cast<const unsigned char*>(src);
    unsigned char* to = static_cast<unsigned char*>(dst);
    std::mutex enqueue;
    std::atomic<int> bad{0};  // the first failure's cudaError_t
    // thread t takes chunks t, t + T, ...; its j-th chunk uses buffer t + (j & 1) T
    auto worker = [&](int t) {
        cudaError_t we = cudaSetDevice(device);
        bool used[2] = {false, false};
        for (size_t i = (size_t)t; we == cudaSuccess && i < n && !bad.load(); i += (size_t)T) {
            const int slot = (int)((i / (size_t)T) & 1u), b = t + slot * T;
            if (used[slot] && (we = cudaEventSynchronize(ev[b])) != cudaSuccess) break;
            const size_t off = i * kChunk, len = std::min(kChunk, bytes - off);
            std::memcpy(ring + (size_t)b * kChunk, from + off, len);
            std::lock_guard<std::mutex> g(enqueue);
            we = cudaMemcpyAsync(to + off, ring + (size_t)b * kChunk, len, cudaMemcpyHostToDevice, st);
            if (we == cudaSuccess) we = cudaEventRecord(ev[b], st);
            used[slot] = true;
        }
        if (we != cudaSuccess) {
            int none = 0;
            bad.compare_exchange_strong(none, (int)we);
        }
    };
    if (e == cudaSuccess) {
        std::vector<std::thread> pool;
        int started = 0;
        try {
            for (; started < T; ++started) pool.emplace_back(worker, started);
        } catch (...) {  // no more threads: the calling thread takes the rest
        }
        for (int t = started; t < T; ++t) worker(t);
        for (std::thread& th : pool) th.join();
        if (bad.load()) e = static_cast<cudaError_t>(bad.load());
    }
    const cudaError_t es = cudaStreamSynchronize(st);  // the ring is read until here
    if (e == cudaSuccess) e = es;
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    cudaFreeHost(ring);
    return e;
}
}  // namespace

int mlem_create(mlem_ctx** out, const uint64_t* row_end, const void* elems, uint32_t n_rows,
                uint32_t n_cols, uint64_t nnz, uint32_t flags, int device) {
    return mlem_create_grid(out, row_end, elems, n_rows, n_cols, nnz, nullptr, flags, device);
}

int mlem_create_grid(mlem_ctx** out, const uint64_t* row_end, const void* elems, uint32_t n_rows,
                     uint32_t n_cols, uint64_t nnz, const uint32_t grid[3], uint32_t flags,
                     int device) {
    if (!out) return fail(nullptr, MLEM_ERR_INVALID, "out is null");
    *out = nullptr;
    if ((n_rows && !row_end) || (nnz && !elems))
        return fail(nullptr, MLEM_ERR_INVALID, "null matrix arrays");
    // host checks of the offsets (cheap, R values)
    uint64_t prev = 0, max_row = 0;
    for (uint32_t r = 0; r < n_rows; ++r) {
        if (row_end[r] < prev) return fail(nullptr, MLEM_ERR_MATRIX, "row offsets decrease at row %u", r);
        max_row = std::max(max_row, row_end[r] - prev);
        prev = row_end[r];
    }
    if (prev != nnz)
        return fail(nullptr, MLEM_ERR_MATRIX, "last row END offset %llu differs from nnz %llu",
                    (unsigned long long)prev, (unsigned long long)nnz);
    mlem_ctx* c = nullptr;
    TRY(new_ctx(&c, n_rows, n_cols, nnz, flags, device));
    if (grid)
        for (int i = 0; i < 3; ++i) c->grid[i] = grid[i];
    c->max_row_len = (uint32_t)std::min<uint64_t>(max_row, 0xffffffffu);
    int s = alloc_matrix(c);
    if (s == MLEM_OK && n_rows) {
        cudaError_t e = cudaMemcpyAsync(c->row_ptr + 1, row_end, (size_t)n_rows * 8,
                                        cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess && nnz) e = upload_pageable(c->device, c->stream, c->elems, elems, nnz * 8);
        if (e != cudaSuccess) s = fail(c, MLEM_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
    }
    if (s == MLEM_OK) s = finish_create(c);
    if (s != MLEM_OK) {
        global_error() = c->err;
        mlem_destroy(c);
        return s;
    }
    *out = c;
    return MLEM_OK;
}

int mlem_create_symmetric(mlem_ctx** out, const uint64_t* row_end, const void* elems,
                          uint32_t n_rows, uint32_t n_cols, uint64_t nnz, const mlem_symmetry* sym,
                          uint32_t flags, int device) {
    if (!out || !sym) return fail(nullptr, MLEM_ERR_INVALID, "null argument");
    *out = nullptr;
    if (sym->sym == 0)
        return mlem_create_grid(out, row_end, elems, n_rows, n_cols, nnz, sym->grid, flags, device);
    if (sym->sym > 7u) return fail(nullptr, MLEM_ERR_INVALID, "symmetry flags 0x%x", sym->sym);
    if ((n_rows && !row_end) || (nnz && !elems))
        return fail(nullptr, MLEM_ERR_INVALID, "null matrix arrays");
    const uint64_t nC = (uint64_t)sym->block_size * sym->n_blocks * sym->n_layers * sym->n_rings;
    if (nC == 0 || nC * nC != n_rows)
        return fail(nullptr, MLEM_ERR_MATRIX,
                    "%u rows are not the %llu x %llu LORs of the scanner block", n_rows,
                    (unsigned long long)nC, (unsigned long long)nC);
    const uint64_t gC = (uint64_t)sym->grid[0] * sym->grid[1] * sym->grid[2];
    if (gC == 0 || gC != n_cols)
        return fail(nullptr, MLEM_ERR_MATRIX, "%u columns are not the %llu voxels of the grid",
                    n_cols, (unsigned long long)gC);
    uint64_t prev = 0;
    for (uint32_t r = 0; r < n_rows; ++r) {
        if (row_end[r] < prev) return fail(nullptr, MLEM_ERR_MATRIX, "row offsets decrease at row %u", r);
        prev = row_end[r];
    }
    if (prev != nnz)
        return fail(nullptr, MLEM_ERR_MATRIX, "last row END offset %llu differs from nnz %llu",
                    (unsigned long long)prev, (unsigned long long)nnz);
    if (flags & MLEM_FLAG_MIRROR_KERNELS) {
        // the stored elements as an ordinary matrix on the grid, then the mirrors
        mlem_ctx* c = nullptr;
        TRY(mlem_create_grid(&c, row_end, elems, n_rows, n_cols, nnz, sym->grid, flags, device));
        const int s = mirror_setup(c, *sym, (uint32_t)nC);
        if (s != MLEM_OK) {
            global_error() = c->err;
            mlem_destroy(c);
            return s;
        }
        *out = c;
        return MLEM_OK;
    }
    mlem_ctx* c = nullptr;
    TRY(new_ctx(&c, n_rows, n_cols, 0, flags, device));
    const uint64_t base_bytes = c->device_bytes;
    for (int i = 0; i < 3; ++i) c->grid[i] = sym->grid[i];
    std::vector<uint32_t> lut;
    sym_detector_luts(sym->n_layers, sym->n_blocks, sym->block_size, sym->n_rings, lut);
    const std::vector<uint32_t> mirrors = sym_mirrors(sym->sym);
    int s = MLEM_OK;
    uint64_t* sptr = nullptr;
    uint2* sel = nullptr;
    uint32_t* dlut = nullptr;
    unsigned long long* counts = nullptr;
    void* scratch = nullptr;
    unsigned int* bad = nullptr;
    const size_t sb = scan_scratch_bytes(n_rows);
    do {
        // the stored matrix on the device, its columns checked before mirroring
        if ((s = dev_alloc(c, &sptr, (size_t)n_rows + 1)) != MLEM_OK) break;
        if ((s = dev_alloc(c, &sel, std::max<uint64_t>(nnz, 1))) != MLEM_OK) break;
        if ((s = dev_alloc(c, &dlut, lut.size())) != MLEM_OK) break;
        if ((s = dev_alloc(c, &counts, std::max<uint32_t>(n_rows, 1))) != MLEM_OK) break;
        if ((s = dev_alloc(c, &scratch, sb)) != MLEM_OK) break;
        if ((s = dev_alloc(c, &bad, 1)) != MLEM_OK) break;
        cudaError_t e = cudaMemsetAsync(sptr, 0, 8, c->stream);
        if (e == cudaSuccess && n_rows)
            e = cudaMemcpyAsync(sptr + 1, row_end, (size_t)n_rows * 8, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess && nnz) e = upload_pageable(c->device, c->stream, sel, elems, nnz * 8);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dlut, lut.data(), lut.size() * 4, cudaMemcpyHostToDevice, c->stream);
        const SparseView stored{sptr, reinterpret_cast<const uint4*>(sel), n_rows, nnz};
        if (e == cudaSuccess) e = validate_csr(stored, n_cols, bad, c->stream);
        unsigned int hbad = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { s = fail(c, MLEM_ERR_CUDA, "symmetry upload: %s", cudaGetErrorString(e)); break; }
        if (hbad & 4u) { s = fail(c, MLEM_ERR_MATRIX, "a column index is >= the number of columns"); break; }
        // full row lengths, offsets, then the elements mirror by mirror
        const SymExpand sx{sptr, sel, n_rows, dlut, (uint32_t)nC,
                           {sym->grid[0], sym->grid[1], sym->grid[2]}};
        e = cudaMemsetAsync(counts, 0, (size_t)n_rows * 8, c->stream);
        if (e == cudaSuccess) e = sym_count(sx, 0, counts, c->stream);
        for (uint32_t m : mirrors)
            if (e == cudaSuccess) e = sym_count(sx, m, counts, c->stream);
        if ((s = dev_alloc(c, &c->row_ptr, (size_t)n_rows + 1)) != MLEM_OK) break;
        if (e == cudaSuccess)
            e = exclusive_scan_u64(reinterpret_cast<const uint64_t*>(counts), c->row_ptr, n_rows,
                                   scratch, sb, c->stream);
        uint64_t Z = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&Z, c->row_ptr + n_rows, 8, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { s = fail(c, MLEM_ERR_CUDA, "symmetry count: %s", cudaGetErrorString(e)); break; }
        c->Z = Z;
        if ((s = dev_alloc(c, &c->elems, Z + 2)) != MLEM_OK) break;
        if ((s = dev_alloc(c, &c->norm, std::max<uint32_t>(c->C, 1))) != MLEM_OK) break;
        e = cudaMemsetAsync(c->elems + Z, 0, 2 * sizeof(uint2), c->stream);
        // the cursors start at the full rows' offsets (the counts buffer is reused)
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(counts, c->row_ptr, (size_t)n_rows * 8, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = sym_fill(sx, 0, counts, c->elems, c->stream);
        for (uint32_t m : mirrors)
            if (e == cudaSuccess) e = sym_fill(sx, m, counts, c->elems, c->stream);
        std::vector<uint64_t> rp((size_t)n_rows + 1);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(rp.data(), c->row_ptr, rp.size() * 8, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { s = fail(c, MLEM_ERR_CUDA, "symmetry fill: %s", cudaGetErrorString(e)); break; }
        uint64_t mr = 0;
        for (uint32_t r = 0; r < n_rows; ++r) mr = std::max(mr, rp[r + 1] - rp[r]);
        c->max_row_len = (uint32_t)std::min<uint64_t>(mr, 0xffffffffu);
    } while (0);
    for (void* p : {(void*)sptr, (void*)sel, (void*)dlut, (void*)counts, scratch, (void*)bad}) dev_free(p);
    // only the full matrix stays
    c->device_bytes = base_bytes + (c->row_ptr ? ((uint64_t)n_rows + 1) * 8 : 0) +
                      (c->elems ? (c->Z + 2) * 8 : 0) +
                      (c->norm ? (uint64_t)std::max<uint32_t>(c->C, 1) * 4 : 0);
    if (s == MLEM_OK) s = finish_create(c);
    if (s != MLEM_OK) {
        global_error() = c->err;
        mlem_destroy(c);
        return s;
    }
    *out = c;
    return MLEM_OK;
}

int mlem_create_siddon(mlem_ctx** out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t n_rows,
                       uint32_t min_count, uint32_t max_count, double radius_scale,
                       double min_len, uint64_t seed, uint32_t flags, int device) {
    if (!out) return fail(nullptr, MLEM_ERR_INVALID, "out is null");
    *out = nullptr;
    if (nx == 0 || ny == 0 || nz == 0) return fail(nullptr, MLEM_ERR_INVALID, "empty voxel grid");
    const uint64_t C64 = (uint64_t)nx * ny * nz;
    if (C64 > 0xffffffffull) return fail(nullptr, MLEM_ERR_INVALID, "grid has more than 2^32 voxels");
    if (!(min_len > 0.0)) return fail(nullptr, MLEM_ERR_INVALID, "min_len must be > 0");
    mlem_ctx* c = nullptr;
    TRY(new_ctx(&c, n_rows, (uint32_t)C64, 0, flags, device));
    c->grid[0] = nx;
    c->grid[1] = ny;
    c->grid[2] = nz;
    SiddonSpec spec{nx, ny, nz, n_rows, min_count, max_count, radius_scale, min_len, seed};
    int s = MLEM_OK;
    uint64_t* counts = nullptr;
    void* scratch = nullptr;
    const size_t sb = scan_scratch_bytes(n_rows);
    do {
        if ((s = dev_alloc(c, &c->row_ptr, (size_t)n_rows + 1)) != MLEM_OK) break;
        if ((s = dev_alloc(c, &counts, std::max<uint32_t>(n_rows, 1))) != MLEM_OK) break;
        if ((s = dev_alloc(c, &scratch, sb)) != MLEM_OK) break;
        cudaError_t e = siddon_counts(spec, counts, c->stream);
        if (e == cudaSuccess) e = exclusive_scan_u64(counts, c->row_ptr, n_rows, scratch, sb, c->stream);
        uint64_t Z = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&Z, c->row_ptr + n_rows, 8, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { s = fail(c, MLEM_ERR_CUDA, "generator: %s", cudaGetErrorString(e)); break; }
        c->Z = Z;
        if ((s = dev_alloc(c, &c->elems, Z + 2)) != MLEM_OK) break;
        if ((s = dev_alloc(c, &c->norm, std::max<uint32_t>(c->C, 1))) != MLEM_OK) break;
        e = cudaMemsetAsync(c->elems + Z, 0, 2 * sizeof(uint2), c->stream);
        if (e == cudaSuccess) e = siddon_fill(spec, c->row_ptr, c->elems, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { s = fail(c, MLEM_ERR_CUDA, "generator fill: %s", cudaGetErrorString(e)); break; }
        // longest row, for the info block
        std::vector<uint64_t> rp((size_t)n_rows + 1);
        e = cudaMemcpy(rp.data(), c->row_ptr, rp.size() * 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { s = fail(c, MLEM_ERR_CUDA, "%s", cudaGetErrorString(e)); break; }
        uint64_t mr = 0;
        for (uint32_t r = 0; r < n_rows; ++r) mr = std::max(mr, rp[r + 1] - rp[r]);
        c->max_row_len = (uint32_t)mr;
    } while (0);
    dev_free(counts);
    dev_free(scratch);
    if (s == MLEM_OK) s = finish_create(c);
    if (s != MLEM_OK) {
        global_error() = c->err;
        mlem_destroy(c);
        return s;
    }
    *out = c;
    return MLEM_OK;
}

void mlem_destroy(mlem_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    free_frames(c);
    region_free(&c->rb);
    for (void* p : {(void*)c->row_ptr, (void*)c->elems, (void*)c->col_ptr, (void*)c->celems,
                    (void*)c->norm, c->stage, (void*)c->stats_slot, (void*)c->hist_sums,
                    (void*)c->hist_zeros, (void*)c->hist_subn, (void*)c->tmp_r[0],
                    (void*)c->tmp_r[1], (void*)c->tmp_c[0], (void*)c->tmp_c[1], (void*)c->tmp_c[2],
                    (void*)c->tmp_sino, (void*)c->tmp_d, (void*)c->norm_nat, (void*)c->perm,
                    (void*)c->pscratch[0], (void*)c->pscratch[1], (void*)c->row_order,
                    (void*)c->row_ranges, (void*)c->counter, (void*)c->long_segs, (void*)c->f_long_d,
                    (void*)c->sub_norm,
                    (void*)c->sub_file, (void*)c->sub_file_ranges, (void*)c->sub_sorted,
                    (void*)c->sub_sorted_ranges, (void*)c->mirror_lut, (void*)c->mirror_vox,
                    (void*)c->f_mirror_d, (void*)c->act_order, (void*)c->act_ranges,
                    (void*)c->act_tmp, (void*)c->act_n, (void*)c->act_z,
                    (void*)c->celems_vis, (void*)c->row_pos, (void*)c->csc_act,
                    (void*)c->csc_act_len, (void*)c->pos_keep, (void*)c->act_order_alt,
                    (void*)c->act_ranges_alt, (void*)c->act_n_alt, (void*)c->act_z_alt})
        dev_free(p);
    if (c->act_host) cudaFreeHost(c->act_host);
    for (cudaStream_t q : {c->up_stream, c->down_stream})
        if (q) { cudaStreamSynchronize(q); cudaStreamDestroy(q); }
    for (int i = 0; i < 2; ++i) {
        dev_free(c->sstage[i]);
        dev_free(c->istage[i]);
        for (cudaEvent_t ev : {c->ev_up[i], c->ev_sfree[i], c->ev_img[i], c->ev_dfree[i]})
            if (ev) cudaEventDestroy(ev);
    }
    if (c->own_stream) cudaStreamSynchronize(c->own_stream);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

int mlem_get_info(const mlem_ctx* c, mlem_info* out) {
    if (!c || !out) return fail(nullptr, MLEM_ERR_INVALID, "null argument");
    out->n_rows = c->R;
    out->n_cols = c->C;
    out->nnz = c->Z;
    out->n_frames = c->B;
    out->flags = c->flags;
    out->device = c->device;
    out->has_csc = c->has_csc ? 1 : 0;
    out->max_col_len = c->max_col_len;
    out->max_row_len = c->max_row_len;
    out->device_bytes = c->device_bytes;
    out->nnz_with_counts = c->act_nnz;
    out->rows_with_counts = c->act_rows;
    return MLEM_OK;
}

int mlem_set_stream(mlem_ctx* c, void* stream) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    TRY(set_device(c));
    CK(c, cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    c->graph_dirty = true;
    return MLEM_OK;
}

int mlem_kernels_per_iteration(const mlem_ctx* c, int* n) {
    if (!c || !n) return fail(nullptr, MLEM_ERR_INVALID, "null argument");
    if (!c->Bp) return fail(const_cast<mlem_ctx*>(c), MLEM_ERR_STATE, "no frames");
    const int tiles = (int)(c->Bp / (uint32_t)c->tuning.frame_tile);
    int k = 2;  // image statistics
    if (c->flags & MLEM_FLAG_EXACT) k += 2;
    else if (c->tuning.bk_mode == MLEM_BK_CSC) k += 2 * tiles;
    else if (c->tuning.bk_mode == MLEM_BK_ATOMIC) k += 2 * tiles + 1;
    else if (c->tuning.bk_mode == MLEM_BK_REGION) k += 2 * tiles + 1;  // + correl
    else if (c->tuning.bk_mode == MLEM_BK_MIRRORED) k += 2 * tiles + 1;  // + update
    else if (c->n_subsets > 1)  // per subset: the one-pass launch(es) and the update
        k += (int)c->n_subsets * ((chunk_visit(c->tuning.visit) ? 1 : tiles) + 1);
    else if (chunk_visit(c->tuning.visit)) k += 2 + (c->n_long ? 2 : 0);  // all tiles in one launch
    else k += tiles + 1 + (c->n_long ? 2 : 0);
    *n = k;
    return MLEM_OK;
}

int mlem_get_csr(mlem_ctx* c, uint64_t* row_end, void* elems) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    TRY(set_device(c));
    if (row_end && c->R)
        CK(c, cudaMemcpy(row_end, c->row_ptr + 1, (size_t)c->R * 8, cudaMemcpyDeviceToHost));
    if (elems && c->Z) {
        CK(c, cudaMemcpy(elems, c->elems, c->Z * 8, cudaMemcpyDeviceToHost));
        if (c->bricked) {
            uint32_t* w = static_cast<uint32_t*>(elems);
            for (uint64_t k = 0; k < c->Z; ++k) w[2 * k] = c->iperm_host[w[2 * k]];
        }
    }
    return MLEM_OK;
}

int mlem_get_csc(mlem_ctx* c, uint64_t* col_ptr, void* elems) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    if (!c->has_csc) return fail(c, MLEM_ERR_STATE, "context has no CSC copy");
    TRY(set_device(c));
    if (!c->bricked) {
        if (col_ptr)
            CK(c, cudaMemcpy(col_ptr, c->col_ptr, ((size_t)c->C + 1) * 8, cudaMemcpyDeviceToHost));
        if (elems && c->Z) CK(c, cudaMemcpy(elems, c->celems, c->Z * 8, cudaMemcpyDeviceToHost));
        return MLEM_OK;
    }
    // device columns are in brick order: reassemble in natural column order
    std::vector<uint64_t> dptr((size_t)c->C + 1);
    CK(c, cudaMemcpy(dptr.data(), c->col_ptr, dptr.size() * 8, cudaMemcpyDeviceToHost));
    std::vector<uint2> del(c->Z);
    if (c->Z) CK(c, cudaMemcpy(del.data(), c->celems, c->Z * 8, cudaMemcpyDeviceToHost));
    uint64_t pos = 0;
    uint2* eo = static_cast<uint2*>(elems);
    for (uint32_t v = 0; v < c->C; ++v) {
        const uint32_t d = c->perm_host[v];
        if (col_ptr) col_ptr[v] = pos;
        for (uint64_t k = dptr[d]; k < dptr[d + 1]; ++k, ++pos)
            if (eo) eo[pos] = del[k];
    }
    if (col_ptr) col_ptr[c->C] = pos;
    return MLEM_OK;
}

// ---- the five reference functions on host buffers ---------------------------
int mlem_calc_column_sums(mlem_ctx* c, float* norm) {
    if (!c || !norm) return fail(c, MLEM_ERR_INVALID, "null argument");
    std::memcpy(norm, c->norm_host.data(), (size_t)c->C * 4);
    return MLEM_OK;
}

int mlem_init_value(mlem_ctx* c, const int32_t* sino, uint64_t len, float* initial) {
    if (!c || !initial || (len && !sino)) return fail(c, MLEM_ERR_INVALID, "null argument");
    double sumin = 0.0;
    for (uint64_t i = 0; i < len; ++i) sumin += sino[i];
    *initial = (float)(sumin / c->sumnorm);
    return MLEM_OK;
}

int mlem_calc_fwproj(mlem_ctx* c, const float* image, float* out) {
    if (!c || !image || !out) return fail(c, MLEM_ERR_INVALID, "null argument");
    TRY(set_device(c));
    TRY(ensure_tmp(c));
    CK(c, cudaMemcpyAsync(c->tmp_c[0], image, (size_t)c->C * 4, cudaMemcpyHostToDevice, c->stream));
    const float* xd = c->tmp_c[0];
    if (c->bricked) {
        CK(c, permute_to_device(c->tmp_c[0], c->tmp_c[1], c->perm, c->C, 1, c->stream));
        xd = c->tmp_c[1];
    }
    if (c->flags & MLEM_FLAG_EXACT) {
        CK(c, fwproj_exact(csr_view(c), xd, 1, nullptr, nullptr, c->tmp_r[0], c->stream));
    } else if (c->mirrored) {
        CK(c, cudaMemsetAsync(c->tmp_r[0], 0, (size_t)c->R * 4, c->stream));
        CK(c, mirror_fwproj(csr_visit(c, c->tuning), c->mirror, xd, 1, 0, 1, c->tmp_r[0], c->n_sm,
                            c->tuning.blocks_per_sm, c->stream));
    } else {
        CK(c, fwproj(csr_visit(c, c->tuning), xd, 1, 0, nullptr, nullptr, c->tmp_r[0], cfg_for_frames(c, 1),
                     c->stream));
    }
    CK(c, cudaMemcpyAsync(out, c->tmp_r[0], (size_t)c->R * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MLEM_OK;
}

int mlem_calc_correl(mlem_ctx* c, const float* f, const int32_t* sino, uint64_t len, float* out) {
    if (!c || !f || !sino || !out) return fail(c, MLEM_ERR_INVALID, "null argument");
    if (len != c->R)
        return fail(c, MLEM_ERR_INVALID, "sinogram has %llu entries, matrix has %u rows",
                    (unsigned long long)len, c->R);
    TRY(set_device(c));
    TRY(ensure_tmp(c));
    CK(c, cudaMemcpyAsync(c->tmp_r[0], f, (size_t)c->R * 4, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemcpyAsync(c->tmp_sino, sino, (size_t)c->R * 4, cudaMemcpyHostToDevice, c->stream));
    CK(c, correl_elementwise(c->tmp_r[0], c->tmp_sino, c->tmp_r[1], c->R, c->stream));
    CK(c, cudaMemcpyAsync(out, c->tmp_r[1], (size_t)c->R * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MLEM_OK;
}

int mlem_calc_bkproj(mlem_ctx* c, const float* correl, float* update) {
    if (!c || !correl || !update) return fail(c, MLEM_ERR_INVALID, "null argument");
    TRY(set_device(c));
    TRY(ensure_tmp(c));
    CK(c, cudaMemcpyAsync(c->tmp_r[0], correl, (size_t)c->R * 4, cudaMemcpyHostToDevice, c->stream));
    float* ud = c->bricked ? c->tmp_c[1] : c->tmp_c[0];
    if (c->flags & MLEM_FLAG_EXACT) {
        CK(c, bkproj_exact(csc_view(c), c->tmp_r[0], 1, nullptr, nullptr, ud, c->stream));
    } else if (c->mirrored) {
        CK(c, cudaMemsetAsync(ud, 0, (size_t)c->C * 4, c->stream));
        CK(c, mirror_bkproj(csr_visit(c, c->tuning), c->mirror, c->tmp_r[0], nullptr, 1, 0, 1, ud,
                            c->n_sm, c->tuning.blocks_per_sm, c->stream));
    } else if (c->has_csc) {
        CK(c, bkproj_csc(csc_view(c), c->tmp_r[0], 1, 0, nullptr, nullptr, ud,
                         cfg_for_frames(c, 1), c->stream));
    } else {
        CK(c, cudaMemsetAsync(ud, 0, (size_t)c->C * 4, c->stream));
        CK(c, bkproj_scatter(csr_visit(c, c->tuning), c->tmp_r[0], 1, 0, ud, cfg_for_frames(c, 1), c->stream));
    }
    if (c->bricked) CK(c, permute_to_natural(ud, c->tmp_c[0], c->perm, c->C, 1, c->stream));
    CK(c, cudaMemcpyAsync(update, c->tmp_c[0], (size_t)c->C * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MLEM_OK;
}

int mlem_calc_update(mlem_ctx* c, const float* update, const float* norm, float* image) {
    if (!c || !update || !norm || !image) return fail(c, MLEM_ERR_INVALID, "null argument");
    TRY(set_device(c));
    TRY(ensure_tmp(c));
    const size_t nb = (size_t)c->C * 4;
    CK(c, cudaMemcpyAsync(c->tmp_c[0], update, nb, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemcpyAsync(c->tmp_c[1], norm, nb, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemcpyAsync(c->tmp_c[2], image, nb, cudaMemcpyHostToDevice, c->stream));
    CK(c, apply_update(c->tmp_c[2], c->tmp_c[0], c->tmp_c[1], c->C, 1, false, c->stream));
    CK(c, cudaMemcpyAsync(image, c->tmp_c[2], nb, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MLEM_OK;
}

// ---- device-resident reconstruction -----------------------------------------
int mlem_set_sinograms(mlem_ctx* c, const int32_t* sino, uint32_t B) {
    if (!c || !sino) return fail(c, MLEM_ERR_INVALID, "null argument");
    TRY(set_device(c));
    TRY(alloc_frames(c, B));
    c->sumin.assign(B, 0.0);
    for (uint32_t b = 0; b < B; ++b) {
        double s = 0.0;  // seqcsr4mlem.cpp:57-58
        const int32_t* p = sino + (size_t)b * c->R;
        for (uint32_t i = 0; i < c->R; ++i) s += p[i];
        c->sumin[b] = s;
    }
    TRY(upload_frames<int32_t>(c, sino, c->sino, c->R));
    TRY(build_active(c, true, true));
    ++c->sino_gen;
    CK(c, cudaStreamSynchronize(c->stream));
    c->images_ready = false;
    return MLEM_OK;
}

int mlem_init_images(mlem_ctx* c, float* initial) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    if (!c->B) return fail(c, MLEM_ERR_STATE, "mlem_set_sinograms must come first");
    TRY(set_device(c));
    std::vector<float> init(c->Bp, 0.0f);
    for (uint32_t b = 0; b < c->B; ++b) init[b] = (float)(c->sumin[b] / c->sumnorm);
    CK(c, cudaMemcpyAsync(c->inits_dev, init.data(), c->Bp * 4, cudaMemcpyHostToDevice, c->stream));
    CK(c, fill_frames(c->x, c->C, c->Bp, c->B, c->inits_dev, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    if (initial) std::memcpy(initial, init.data(), c->B * 4);
    c->images_ready = true;
    return MLEM_OK;
}

int mlem_set_images(mlem_ctx* c, const float* images) {
    if (!c || !images) return fail(c, MLEM_ERR_INVALID, "null argument");
    if (!c->B) return fail(c, MLEM_ERR_STATE, "mlem_set_sinograms must come first");
    TRY(set_device(c));
    TRY(upload_frames<float>(c, images, c->x, c->C));
    CK(c, cudaStreamSynchronize(c->stream));
    c->images_ready = true;
    return MLEM_OK;
}

int mlem_iterate(mlem_ctx* c, int n, double* sums, uint64_t* zeros, uint64_t* subn) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    if (n < 0) return fail(c, MLEM_ERR_INVALID, "negative iteration count");
    if (!c->images_ready) return fail(c, MLEM_ERR_STATE, "images not initialised");
    if (n == 0) return MLEM_OK;
    TRY(set_device(c));
    if (c->tuning.bk_mode == MLEM_BK_REGION && !(c->flags & MLEM_FLAG_EXACT))
        TRY(ensure_region(c, c->tuning.frame_tile));
    // Chunks of up to 64 iterations, each one graph launch.
    const int chunk = std::min(n, 64);
    TRY(ensure_history(c, chunk));
    if (c->graph_dirty || !c->graph || c->graph_iters != chunk) TRY(capture(c, chunk));
    int done = 0;
    while (done < n) {
        const int k = std::min(chunk, n - done);
        if (k == chunk) {
            CK(c, cudaGraphLaunch(c->graph, c->stream));
        } else {
            CK(c, cudaMemsetAsync(c->stats_slot, 0, 4, c->stream));
            for (int i = 0; i < k; ++i) TRY(enqueue_iteration(c, c->tuning, true));
        }
        const size_t cnt = (size_t)k * c->B;
        if (sums) CK(c, cudaMemcpyAsync(sums + (size_t)done * c->B, c->hist_sums, cnt * 8,
                                        cudaMemcpyDeviceToHost, c->stream));
        if (zeros) CK(c, cudaMemcpyAsync(zeros + (size_t)done * c->B, c->hist_zeros, cnt * 8,
                                         cudaMemcpyDeviceToHost, c->stream));
        if (subn) CK(c, cudaMemcpyAsync(subn + (size_t)done * c->B, c->hist_subn, cnt * 8,
                                        cudaMemcpyDeviceToHost, c->stream));
        if (sums || zeros || subn) CK(c, cudaStreamSynchronize(c->stream));
        done += k;
    }
    CK(c, cudaStreamSynchronize(c->stream));
    return MLEM_OK;
}

int mlem_get_images(mlem_ctx* c, float* images) {
    if (!c || !images) return fail(c, MLEM_ERR_INVALID, "null argument");
    if (!c->B) return fail(c, MLEM_ERR_STATE, "no frames");
    TRY(set_device(c));
    TRY(download_images(c, images));
    CK(c, cudaStreamSynchronize(c->stream));
    return MLEM_OK;
}

int mlem_step_host(mlem_ctx* c, const int32_t* sino, float* images, uint32_t B) {
    if (!c || !sino || !images) return fail(c, MLEM_ERR_INVALID, "null argument");
    TRY(set_device(c));
    if (c->B != B) TRY(alloc_frames(c, B));
    TRY(upload_frames<int32_t>(c, sino, c->sino, c->R));
    TRY(build_active(c, false, false));
    ++c->sino_gen;
    // the list's row and element counts for mlem_get_info: copied with the
    // step, read after its final synchronisation
    if (c->act_ready && !c->act_host &&
        cudaHostAlloc(reinterpret_cast<void**>(&c->act_host), 16, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        c->act_host = nullptr;
    }
    const bool counts = c->act_ready && c->act_host;
    if (counts) {
        CK(c, cudaMemcpyAsync(c->act_host, c->act_n, 4, cudaMemcpyDeviceToHost, c->stream));
        CK(c, cudaMemcpyAsync(c->act_host + 1, c->act_z, 8, cudaMemcpyDeviceToHost, c->stream));
    }
    TRY(upload_frames<float>(c, images, c->x, c->C));
    c->images_ready = true;
    if (c->tuning.bk_mode == MLEM_BK_REGION && !(c->flags & MLEM_FLAG_EXACT))
        TRY(ensure_region(c, c->tuning.frame_tile));
    if (c->graph_dirty || !c->graph || c->graph_iters != 1) {
        TRY(ensure_history(c, 1));
        TRY(capture(c, 1));
    }
    CK(c, cudaGraphLaunch(c->graph, c->stream));
    TRY(download_images(c, images));
    CK(c, cudaStreamSynchronize(c->stream));
    if (counts) {
        c->act_rows = static_cast<uint32_t>(c->act_host[0] & 0xffffffffull);
        c->act_nnz = c->act_host[1];
    } else if (!c->act_ready) {
        c->act_rows = 0;
        c->act_nnz = 0;
    }
    return MLEM_OK;
}

// The copy streams, events and double-buffered staging of mlem_stream_host
// (created on first use, sized for the current frames).
static int ensure_streaming(mlem_ctx* c) {
    for (cudaStream_t* q : {&c->up_stream, &c->down_stream})
        if (!*q) CK(c, cudaStreamCreateWithFlags(q, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i)
        for (cudaEvent_t* ev : {&c->ev_up[i], &c->ev_sfree[i], &c->ev_img[i], &c->ev_dfree[i]})
            if (!*ev) CK(c, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    const size_t sn = (size_t)c->R * c->B, in = (size_t)c->C * c->B;
    for (int i = 0; i < 2; ++i) {
        if (c->sstage_n < sn) {
            if (c->sstage[i]) { dev_free(c->sstage[i]); c->device_bytes -= c->sstage_n * 4; c->sstage[i] = nullptr; }
            TRY(dev_alloc(c, &c->sstage[i], std::max<size_t>(sn, 1)));
        }
        if (c->istage_n < in) {
            if (c->istage[i]) { dev_free(c->istage[i]); c->device_bytes -= c->istage_n * 4; c->istage[i] = nullptr; }
            TRY(dev_alloc(c, &c->istage[i], std::max<size_t>(in, 1)));
        }
    }
    c->sstage_n = std::max(c->sstage_n, sn);
    c->istage_n = std::max(c->istage_n, in);
    return MLEM_OK;
}

// The steps of mlem_stream_host, enqueued on the three streams.
static int stream_steps(mlem_ctx* c, const int32_t* const* sinos, float* const* images, uint32_t n) {
    const uint32_t B = c->B, Bp = c->Bp;
    const size_t sbytes = (size_t)c->R * B * 4, ibytes = (size_t)c->C * B * 4;
    CK(c, cudaMemcpyAsync(c->sstage[0], sinos[0], sbytes, cudaMemcpyHostToDevice, c->up_stream));
    CK(c, cudaEventRecord(c->ev_up[0], c->up_stream));
    for (uint32_t k = 0; k < n; ++k) {
        const int cur = (int)(k & 1), nxt = cur ^ 1;
        if (k + 1 < n) {  // the next sinograms, once iteration k - 1 has copied that buffer out
            CK(c, cudaStreamWaitEvent(c->up_stream, c->ev_sfree[nxt], 0));
            CK(c, cudaMemcpyAsync(c->sstage[nxt], sinos[k + 1], sbytes, cudaMemcpyHostToDevice,
                                  c->up_stream));
            CK(c, cudaEventRecord(c->ev_up[nxt], c->up_stream));
        }
        CK(c, cudaStreamWaitEvent(c->stream, c->ev_up[cur], 0));
        if (Bp == 1)
            CK(c, cudaMemcpyAsync(c->sino, c->sstage[cur], sbytes, cudaMemcpyDeviceToDevice, c->stream));
        else
            CK(c, interleave_i32(c->sstage[cur], c->sino, c->R, B, Bp, c->stream));
        CK(c, cudaEventRecord(c->ev_sfree[cur], c->stream));
        TRY(build_active(c, false, false));
        ++c->sino_gen;
        if (c->graph_dirty || !c->graph || c->graph_iters != 1) {
            TRY(ensure_history(c, 1));
            TRY(capture(c, 1));
        }
        CK(c, cudaGraphLaunch(c->graph, c->stream));
        if (images && images[k]) {  // this iteration's images, once the buffer's last download is done
            CK(c, cudaStreamWaitEvent(c->stream, c->ev_dfree[cur], 0));
            if (Bp == 1 && !c->bricked)
                CK(c, cudaMemcpyAsync(c->istage[cur], c->x, ibytes, cudaMemcpyDeviceToDevice, c->stream));
            else
                CK(c, deinterleave_f32(c->x, c->istage[cur], c->C, B, Bp, c->bricked ? c->perm : nullptr,
                                       c->stream));
            CK(c, cudaEventRecord(c->ev_img[cur], c->stream));
            CK(c, cudaStreamWaitEvent(c->down_stream, c->ev_img[cur], 0));
            CK(c, cudaMemcpyAsync(images[k], c->istage[cur], ibytes, cudaMemcpyDeviceToHost,
                                  c->down_stream));
            CK(c, cudaEventRecord(c->ev_dfree[cur], c->down_stream));
        }
    }
    return MLEM_OK;
}

// The per-sinogram buffers the iteration graph reads: the sinogram and the
// list of rows with counts.
struct SinoSet {
    int32_t* sino;
    uint32_t* order;
    ulonglong2* ranges;
    uint32_t* n;
    unsigned long long* z;
};

static void swap_sets(mlem_ctx* c) {
    std::swap(c->sino, c->sino_alt);
    std::swap(c->act_order, c->act_order_alt);
    std::swap(c->act_ranges, c->act_ranges_alt);
    std::swap(c->act_n, c->act_n_alt);
    std::swap(c->act_z, c->act_z_alt);
}

// The overlapped steps run where the iteration walks the list of rows with
// counts (built for the current sinograms) and no subsets.
static bool stream_overlap_ok(const mlem_ctx* c) {
    return c->act_ready && c->act_tmp && c->n_subsets == 1 && !c->mirrored &&
           !(c->flags & MLEM_FLAG_EXACT);
}

static int ensure_stream_alt(mlem_ctx* c) {
    if (!c->sino_alt) {
        TRY(dev_alloc(c, &c->sino_alt, std::max<size_t>((size_t)c->R * c->Bp, 1)));
        CK(c, cudaMemsetAsync(c->sino_alt, 0, (size_t)c->R * c->Bp * 4, c->stream));  // pad frames
        if (c->graph_alt) { cudaGraphExecDestroy(c->graph_alt); c->graph_alt = nullptr; }
    }
    if (!c->act_order_alt) {
        TRY(dev_alloc(c, &c->act_order_alt, std::max<uint32_t>(c->R, 1)));
        TRY(dev_alloc(c, &c->act_ranges_alt, std::max<uint32_t>(c->R, 1)));
        TRY(dev_alloc(c, &c->act_n_alt, 1));
        TRY(dev_alloc(c, &c->act_z_alt, 1));
    }
    return MLEM_OK;
}

// mlem_stream_host's steps with two sets of per-sinogram buffers, each with
// its own one-iteration graph: the upload of step k+1's sinograms and the
// rebuild of their list of rows with counts run on the copy stream, into the
// other set, while step k iterates; the compute stream only waits for its
// set, launches its graph and copies the images out.
static int stream_steps_overlap(mlem_ctx* c, const int32_t* const* sinos, float* const* images,
                                uint32_t n) {
    const uint32_t B = c->B, Bp = c->Bp;
    const size_t sbytes = (size_t)c->R * B * 4, ibytes = (size_t)c->C * B * 4;
    TRY(ensure_stream_alt(c));
    if (c->csc_act_ready) {  // one iteration per sinogram: the whole CSC in visiting order
        c->csc_act_ready = false;
        c->graph_dirty = true;
    }
    if (c->graph_dirty || !c->graph || c->graph_iters != 1) {
        TRY(ensure_history(c, 1));
        TRY(capture(c, 1));
    }
    if (!c->graph_alt) {
        swap_sets(c);
        const int s = capture_into(c, 1, &c->graph_alt);
        swap_sets(c);
        TRY(s);
    }
    const SinoSet set[2] = {{c->sino, c->act_order, c->act_ranges, c->act_n, c->act_z},
                            {c->sino_alt, c->act_order_alt, c->act_ranges_alt, c->act_n_alt,
                             c->act_z_alt}};
    const cudaGraphExec_t graph[2] = {c->graph, c->graph_alt};
    // set q takes step j's sinograms once the step two before has iterated on it
    auto upload = [&](uint32_t j, int q) -> int {
        CK(c, cudaStreamWaitEvent(c->up_stream, c->ev_sfree[q], 0));
        if (Bp == 1) {
            CK(c, cudaMemcpyAsync(set[q].sino, sinos[j], sbytes, cudaMemcpyHostToDevice,
                                  c->up_stream));
        } else {
            CK(c, cudaMemcpyAsync(c->sstage[q], sinos[j], sbytes, cudaMemcpyHostToDevice,
                                  c->up_stream));
            CK(c, interleave_i32(c->sstage[q], set[q].sino, c->R, B, Bp, c->up_stream));
        }
        CK(c, active_rows_build(csr_view(c), set[q].sino, Bp, c->act_tmp, c->act_tmp_bytes,
                                set[q].order, set[q].ranges, set[q].n, set[q].z, c->up_stream));
        CK(c, cudaEventRecord(c->ev_up[q], c->up_stream));
        return MLEM_OK;
    };
    // both sets are free once the work already on the compute stream is done
    for (int q = 0; q < 2; ++q) CK(c, cudaEventRecord(c->ev_sfree[q], c->stream));
    TRY(upload(0, 0));
    for (uint32_t k = 0; k < n; ++k) {
        const int p = (int)(k & 1);
        if (k + 1 < n) TRY(upload(k + 1, p ^ 1));
        CK(c, cudaStreamWaitEvent(c->stream, c->ev_up[p], 0));
        CK(c, cudaGraphLaunch(graph[p], c->stream));
        CK(c, cudaEventRecord(c->ev_sfree[p], c->stream));
        ++c->sino_gen;
        if (images && images[k]) {  // this iteration's images, once the buffer's last download is done
            CK(c, cudaStreamWaitEvent(c->stream, c->ev_dfree[p], 0));
            if (Bp == 1 && !c->bricked)
                CK(c, cudaMemcpyAsync(c->istage[p], c->x, ibytes, cudaMemcpyDeviceToDevice, c->stream));
            else
                CK(c, deinterleave_f32(c->x, c->istage[p], c->C, B, Bp, c->bricked ? c->perm : nullptr,
                                       c->stream));
            CK(c, cudaEventRecord(c->ev_img[p], c->stream));
            CK(c, cudaStreamWaitEvent(c->down_stream, c->ev_img[p], 0));
            CK(c, cudaMemcpyAsync(images[k], c->istage[p], ibytes, cudaMemcpyDeviceToHost,
                                  c->down_stream));
            CK(c, cudaEventRecord(c->ev_dfree[p], c->down_stream));
        }
    }
    if ((n - 1) & 1) {  // the last sinograms are in the second set: it becomes the first
        swap_sets(c);
        std::swap(c->graph, c->graph_alt);
    }
    return MLEM_OK;
}

int mlem_stream_host(mlem_ctx* c, const int32_t* const* sinos, float* const* images, uint32_t n) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    if (n == 0) return MLEM_OK;
    if (!sinos) return fail(c, MLEM_ERR_INVALID, "null argument");
    for (uint32_t k = 0; k < n; ++k)
        if (!sinos[k]) return fail(c, MLEM_ERR_INVALID, "sinograms of iteration %u: null", k);
    if (!c->B) return fail(c, MLEM_ERR_STATE, "mlem_set_sinograms must come first");
    if (!c->images_ready) return fail(c, MLEM_ERR_STATE, "images not initialised");
    TRY(set_device(c));
    TRY(ensure_streaming(c));
    if (c->tuning.bk_mode == MLEM_BK_REGION && !(c->flags & MLEM_FLAG_EXACT))
        TRY(ensure_region(c, c->tuning.frame_tile));
    if (c->act_ready && !c->act_host &&
        cudaHostAlloc(reinterpret_cast<void**>(&c->act_host), 16, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        c->act_host = nullptr;
    }
    int s = stream_overlap_ok(c) ? stream_steps_overlap(c, sinos, images, n)
                                 : stream_steps(c, sinos, images, n);
    const bool counts = s == MLEM_OK && c->act_ready && c->act_host;
    if (counts &&
        (cudaMemcpyAsync(c->act_host, c->act_n, 4, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
         cudaMemcpyAsync(c->act_host + 1, c->act_z, 8, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess))
        s = fail(c, MLEM_ERR_CUDA, "row counts: %s", cudaGetErrorString(cudaGetLastError()));
    // every copy that names a caller buffer ends before the call returns, failed or not
    cudaError_t e = cudaSuccess;
    for (cudaStream_t q : {c->up_stream, c->stream, c->down_stream}) {
        const cudaError_t eq = cudaStreamSynchronize(q);
        if (e == cudaSuccess) e = eq;
    }
    if (s != MLEM_OK) return s;
    if (e != cudaSuccess) return fail(c, MLEM_ERR_CUDA, "streamed iterations: %s", cudaGetErrorString(e));
    if (counts) {
        c->act_rows = static_cast<uint32_t>(c->act_host[0] & 0xffffffffull);
        c->act_nnz = c->act_host[1];
    } else if (!c->act_ready) {
        c->act_rows = 0;
        c->act_nnz = 0;
    }
    return MLEM_OK;
}

int mlem_profile_phases(mlem_ctx* c, int n, double* ms, double* bytes, int* launches) {
    if (!c || n <= 0) return fail(c, MLEM_ERR_INVALID, "bad argument");
    if (!c->images_ready) return fail(c, MLEM_ERR_STATE, "images not initialised");
    TRY(set_device(c));
    TRY(ensure_history(c, 1));
    if (c->tuning.bk_mode == MLEM_BK_REGION && !(c->flags & MLEM_FLAG_EXACT))
        TRY(ensure_region(c, c->tuning.frame_tile));
    std::vector<PhaseEvents> evs((size_t)n);
    for (auto& pe : evs)
        for (auto& e : pe.ev) CK(c, cudaEventCreate(&e));
    int s = MLEM_OK;
    for (int i = 0; i < n && s == MLEM_OK; ++i) {
        if (cudaMemsetAsync(c->stats_slot, 0, 4, c->stream) != cudaSuccess)
            s = fail(c, MLEM_ERR_CUDA, "memset");
        else
            s = enqueue_iteration(c, c->tuning, true, &evs[(size_t)i]);
    }
    if (s == MLEM_OK && cudaStreamSynchronize(c->stream) != cudaSuccess)
        s = fail(c, MLEM_ERR_CUDA, "synchronize");
    double acc[MLEM_N_PHASES] = {0, 0, 0, 0};
    for (auto& pe : evs)
        for (int p = 0; p < MLEM_N_PHASES && s == MLEM_OK; ++p) {
            float t = 0.0f;
            if (cudaEventElapsedTime(&t, pe.ev[p], pe.ev[p + 1]) != cudaSuccess)
                s = fail(c, MLEM_ERR_CUDA, "event timing");
            acc[p] += t;
        }
    for (auto& pe : evs)
        for (auto& e : pe.ev) cudaEventDestroy(e);
    if (s != MLEM_OK) return s;
    double b[MLEM_N_PHASES];
    int l[MLEM_N_PHASES];
    phase_bytes(c, b, l);
    for (int p = 0; p < MLEM_N_PHASES; ++p) {
        if (ms) ms[p] = acc[p] / n;
        if (bytes) bytes[p] = b[p];
        if (launches) launches[p] = l[p];
    }
    return MLEM_OK;
}

// ---- tuning -------------------------------------------------------------------
int mlem_get_tuning(const mlem_ctx* c, mlem_tuning* out) {
    if (!c || !out) return fail(nullptr, MLEM_ERR_INVALID, "null argument");
    *out = c->tuning;
    return MLEM_OK;
}

int mlem_set_tuning(mlem_ctx* c, const mlem_tuning* t) {
    if (!c || !t) return fail(c, MLEM_ERR_INVALID, "null argument");
    mlem_tuning n = *t;
    if (n.bk_mode == MLEM_BK_AUTO)
        n.bk_mode = c->mirrored ? MLEM_BK_MIRRORED : c->has_csc ? MLEM_BK_CSC : MLEM_BK_ATOMIC;
    if (n.bk_mode == MLEM_BK_CSC && !c->has_csc)
        return fail(c, MLEM_ERR_INVALID, "MLEM_BK_CSC needs the CSC copy");
    if (n.bk_mode < MLEM_BK_CSC || n.bk_mode > MLEM_BK_MIRRORED)
        return fail(c, MLEM_ERR_INVALID, "unknown back-projection mode %d", n.bk_mode);
    if (c->mirrored != (n.bk_mode == MLEM_BK_MIRRORED))
        return fail(c, MLEM_ERR_INVALID, c->mirrored
                        ? "a context made with MLEM_FLAG_MIRROR_KERNELS runs MLEM_BK_MIRRORED only"
                        : "MLEM_BK_MIRRORED needs a context made with MLEM_FLAG_MIRROR_KERNELS");
    if (n.bk_mode == MLEM_BK_MIRRORED &&
        (n.group != 32 || (n.visit != MLEM_VISIT_FILE && n.visit != MLEM_VISIT_SORTED)))
        return fail(c, MLEM_ERR_INVALID,
                    "MLEM_BK_MIRRORED runs 32 lanes per row (group 32) in file or sorted order");
    LaunchCfg cfg;
    cfg.group = n.group;
    cfg.frame_tile = n.frame_tile;
    cfg.blocks_per_sm = n.blocks_per_sm;
    if (!cfg_valid(cfg))
        return fail(c, MLEM_ERR_INVALID, "invalid launch configuration (group %d, tile %d, blocks %d)",
                    n.group, n.frame_tile, n.blocks_per_sm);
    if (c->Bp && (c->Bp % (uint32_t)n.frame_tile))
        return fail(c, MLEM_ERR_INVALID, "frame tile %d does not divide the padded frame count %u",
                    n.frame_tile, c->Bp);
    if (n.visit < MLEM_VISIT_FILE || n.visit > MLEM_VISIT_SORTED_STAGED)
        return fail(c, MLEM_ERR_INVALID, "unknown row visiting order %d", n.visit);
    if (n.visit != MLEM_VISIT_FILE && !c->row_order)
        return fail(c, MLEM_ERR_INVALID,
                    "sorted row visiting needs the row order (context made with MLEM_FLAG_NO_ROW_ORDER)");
    if (chunk_visit(n.visit) && n.group != 32)
        return fail(c, MLEM_ERR_INVALID, "the chunked row visits run 32 lanes per row (group 32)");
    if (c->n_subsets > 1 && n.bk_mode != MLEM_BK_FUSED)
        return fail(c, MLEM_ERR_INVALID,
                    "ordered subsets run on the one-pass method (MLEM_BK_FUSED) only");
    if (n.bk_mode == MLEM_BK_REGION) {
        TRY(set_device(c));
        TRY(ensure_region(c, n.frame_tile));
    }
    if (csc_by_visit(c, n)) {
        TRY(set_device(c));
        TRY(ensure_csc_vis(c));
        if (!c->csc_act_ready) {
            TRY(build_csc_act(c, n));
            CK(c, cudaStreamSynchronize(c->stream));
        }
    }
    c->tuning = n;
    c->graph_dirty = true;
    return MLEM_OK;
}

int mlem_autotune(mlem_ctx* c, int deterministic_only, mlem_tuning* best_out) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    if (!c->B || !c->images_ready) return fail(c, MLEM_ERR_STATE, "set sinograms and images first");
    if (c->flags & MLEM_FLAG_EXACT) {
        if (best_out) *best_out = c->tuning;
        return MLEM_OK;
    }
    TRY(set_device(c));
    // Save the images: tuning runs real iterations.
    float* saved = nullptr;
    const size_t xb = (size_t)c->C * c->Bp * 4;
    TRY(dev_alloc(c, &saved, (size_t)c->C * c->Bp));
    CK(c, cudaMemcpyAsync(saved, c->x, xb, cudaMemcpyDeviceToDevice, c->stream));
    std::vector<int> modes;
    if (c->mirrored) {  // one method; mlem_set_subsets refuses mirrored contexts
        if (deterministic_only) {
            cudaFree(saved);
            c->device_bytes -= xb;
            return fail(c, MLEM_ERR_STATE,
                        "the mirrored kernels (MLEM_FLAG_MIRROR_KERNELS) have no deterministic method");
        }
        modes.push_back(MLEM_BK_MIRRORED);
    } else if (c->n_subsets > 1) {
        if (deterministic_only) {
            cudaFree(saved);
            c->device_bytes -= xb;
            return fail(c, MLEM_ERR_STATE, "ordered subsets have no deterministic method");
        }
        modes.push_back(MLEM_BK_FUSED);
    } else {
        if (c->has_csc) modes.push_back(MLEM_BK_CSC);
        if (!deterministic_only)
            for (int m : {MLEM_BK_ATOMIC, MLEM_BK_FUSED, MLEM_BK_REGION}) modes.push_back(m);
    }
    cudaEvent_t e0, e1;
    CK(c, cudaEventCreate(&e0));
    CK(c, cudaEventCreate(&e1));
    mlem_tuning best = c->tuning;
    best.ms_per_iter = 1e30;
    const mlem_tuning orig = c->tuning;
    for (int mode : modes)
        for (int group : {8, 16, 32})
            for (int tile : {1, 2, 4, 8, 16}) {
                if (c->Bp % (uint32_t)tile) continue;
                if (mode == MLEM_BK_REGION) {
                    if (group != 32) continue;  // lane groups follow the tile: no group
                    if (ensure_region(c, tile) != MLEM_OK) continue;  // e.g. no memory: skip
                }
                for (int bps : {4, 8})
                for (int visit : {MLEM_VISIT_FILE, MLEM_VISIT_SORTED, MLEM_VISIT_SORTED_CHUNKED,
                                  MLEM_VISIT_SORTED_STAGED}) {
                    if (mode == MLEM_BK_REGION && bps == 4) continue;  // grid is fixed by the tile
                    // the sorted orders need the row order; the region method has its
                    // own layout; only the one-pass method walks chunks
                    if (visit != MLEM_VISIT_FILE && (!c->row_order || mode == MLEM_BK_REGION))
                        continue;
                    if (chunk_visit(visit) && mode != MLEM_BK_FUSED) continue;
                    if (mode == MLEM_BK_MIRRORED && group != 32) continue;
                    // chunked: warp-wide rows; CTAs per SM 4 (bps 4) or 1 (bps 8 -> 1 below);
                    // staged: 4 or 3 CTAs of 256 threads
                    if (chunk_visit(visit) && group != 32) continue;
                    if (mode == MLEM_BK_CSC && visit != MLEM_VISIT_FILE &&
                        ensure_csc_vis(c) != MLEM_OK)
                        continue;  // e.g. no memory for the second CSC: skip
                    const int ctas = visit == MLEM_VISIT_SORTED_CHUNKED ? (bps == 8 ? 1 : bps)
                                     : visit == MLEM_VISIT_SORTED_STAGED ? (bps == 8 ? 3 : bps)
                                                                         : bps;
                    mlem_tuning t{mode, group, tile, ctas, visit, 0.0};
                    // the cut copy of the CSC in visiting order, as the method runs
                    int s = c->csc_act_ready ? MLEM_OK : build_csc_act(c, t);
                    // warm-up once, then time two iterations
                    if (s == MLEM_OK) s = enqueue_iteration(c, t, false);
                    if (s != MLEM_OK) { c->tuning = orig; return s; }
                    CK(c, cudaEventRecord(e0, c->stream));
                    for (int i = 0; i < 2; ++i) TRY(enqueue_iteration(c, t, false));
                    CK(c, cudaEventRecord(e1, c->stream));
                    CK(c, cudaEventSynchronize(e1));
                    float ms = 0.0f;
                    CK(c, cudaEventElapsedTime(&ms, e0, e1));
                    t.ms_per_iter = ms / 2.0;
                    if (t.ms_per_iter < best.ms_per_iter) best = t;
                    CK(c, cudaMemcpyAsync(c->x, saved, xb, cudaMemcpyDeviceToDevice, c->stream));
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(c, cudaMemcpyAsync(c->x, saved, xb, cudaMemcpyDeviceToDevice, c->stream));
    CK(c, cudaMemsetAsync(c->update, 0, xb, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    cudaFree(saved);
    c->device_bytes -= xb;
    if (best.bk_mode == MLEM_BK_REGION) TRY(ensure_region(c, best.frame_tile));
    if (!csc_by_visit(c, best) && c->celems_vis)  // tried, not chosen: give the memory back
        free_csc_vis(c);
    c->tuning = best;
    c->graph_dirty = true;
    if (best_out) *best_out = best;
    return MLEM_OK;
}

// ---- ordered subsets ----------------------------------------------------------

namespace {

void free_subsets(mlem_ctx* c) {
    for (void** p : {(void**)&c->sub_norm, (void**)&c->sub_file, (void**)&c->sub_file_ranges,
                     (void**)&c->sub_sorted, (void**)&c->sub_sorted_ranges,
                     (void**)&c->sub_act_order, (void**)&c->sub_act_ranges, (void**)&c->sub_act_n,
                     (void**)&c->sub_act_z}) {
        dev_free(*p);
        *p = nullptr;
    }
    c->sub_act_ready = false;
    c->sub_off.clear();
    c->n_subsets = 1;
    c->device_bytes -= c->sub_bytes;
    c->sub_bytes = 0;
}

// Upload a visiting list (every subset's rows back to back) and build its ranges.
int upload_list(mlem_ctx* c, const std::vector<uint32_t>& list, uint32_t** order,
                ulonglong2** ranges) {
    TRY(dev_alloc(c, order, c->R));
    TRY(dev_alloc(c, ranges, c->R));
    CK(c, cudaMemcpyAsync(*order, list.data(), (size_t)c->R * 4, cudaMemcpyHostToDevice, c->stream));
    CK(c, row_ranges_build(csr_view(c), *order, *ranges, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));  // `list` is freed by the caller
    return MLEM_OK;
}

}  // namespace

int mlem_set_subsets(mlem_ctx* c, uint32_t n) {
    if (!c) return fail(nullptr, MLEM_ERR_INVALID, "null context");
    if (n == 0) return fail(c, MLEM_ERR_INVALID, "at least one subset");
    if (n > 1 && (c->flags & MLEM_FLAG_EXACT))
        return fail(c, MLEM_ERR_INVALID, "ordered subsets do not run in the bit-exact mode");
    if (n > 1 && c->mirrored)
        return fail(c, MLEM_ERR_INVALID,
                    "ordered subsets run over the full matrix's rows, not with MLEM_FLAG_MIRROR_KERNELS");
    if (n > 1 && n > c->R)
        return fail(c, MLEM_ERR_INVALID, "%u subsets for %u rows", n, c->R);
    TRY(set_device(c));
    CK(c, cudaStreamSynchronize(c->stream));
    free_subsets(c);
    c->graph_dirty = true;
    if (n == 1) return MLEM_OK;
    const size_t before = c->device_bytes;
    auto bail = [&](int s) {
        c->sub_bytes = c->device_bytes - before;
        free_subsets(c);
        return s;
    };
    // column sums of every subset (device voxel order)
    int s = dev_alloc(c, &c->sub_norm, (size_t)n * c->C);
    if (s != MLEM_OK) return bail(s);
    cudaError_t e = cudaSuccess;
    if (c->has_csc) {
        for (uint32_t k = 0; k < n && e == cudaSuccess; ++k)
            e = subset_column_sums_exact(csc_view(c), n, k, c->sub_norm + (size_t)k * c->C, c->stream);
    } else {
        e = subset_column_sums_atomic(csr_view(c), n, c->C, c->sub_norm, c->stream);
    }
    if (e != cudaSuccess) return bail(fail(c, MLEM_ERR_CUDA, "subset column sums: %s", cudaGetErrorString(e)));
    // visiting lists: subset k holds rows k, k + n, ... (file order), or those
    // rows in the order of the row sort
    c->sub_off.assign((size_t)n + 1, 0);
    for (uint32_t k = 0; k < n; ++k)
        c->sub_off[k + 1] = c->sub_off[k] + (k < c->R ? (c->R - k + n - 1) / n : 0);
    std::vector<uint32_t> list(c->R);
    for (uint32_t k = 0; k < n; ++k) {
        uint64_t o = c->sub_off[k];
        for (uint32_t r = k; r < c->R; r += n) list[o++] = r;
    }
    s = upload_list(c, list, &c->sub_file, &c->sub_file_ranges);
    if (s != MLEM_OK) return bail(s);
    if (c->row_order) {
        std::vector<uint32_t> order(c->R);
        e = cudaMemcpy(order.data(), c->row_order, (size_t)c->R * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return bail(fail(c, MLEM_ERR_CUDA, "row order: %s", cudaGetErrorString(e)));
        std::vector<uint64_t> next(c->sub_off.begin(), c->sub_off.end() - 1);
        for (uint32_t r : order) list[next[r % n]++] = r;  // stable partition by subset
        s = upload_list(c, list, &c->sub_sorted, &c->sub_sorted_ranges);
        if (s != MLEM_OK) return bail(s);
        // room for the lists without the rows without counts
        if ((s = dev_alloc(c, &c->sub_act_order, c->R)) != MLEM_OK ||
            (s = dev_alloc(c, &c->sub_act_ranges, c->R)) != MLEM_OK ||
            (s = dev_alloc(c, &c->sub_act_n, n)) != MLEM_OK ||
            (s = dev_alloc(c, &c->sub_act_z, n)) != MLEM_OK)
            return bail(s);
    }
    c->n_subsets = n;
    c->sub_bytes = c->device_bytes - before;
    if (c->B && c->sino) {  // sinograms already set: their lists now
        s = build_subset_lists(c);
        if (s == MLEM_OK) CK(c, cudaStreamSynchronize(c->stream));
        if (s != MLEM_OK) return bail(s);
    }
    return MLEM_OK;
}

int mlem_get_subsets(const mlem_ctx* c, uint32_t* n) {
    if (!c || !n) return fail(const_cast<mlem_ctx*>(c), MLEM_ERR_INVALID, "null argument");
    *n = c->n_subsets;
    return MLEM_OK;
}

int mlem_subset_column_sums(mlem_ctx* c, uint32_t s, float* out) {
    if (!c || !out) return fail(c, MLEM_ERR_INVALID, "null argument");
    if (c->n_subsets < 2 || s >= c->n_subsets)
        return fail(c, MLEM_ERR_INVALID, "subset %u of %u", s, c->n_subsets);
    TRY(set_device(c));
    const float* src = c->sub_norm + (size_t)s * c->C;
    std::vector<float> dev(c->C);
    CK(c, cudaMemcpyAsync(dev.data(), src, (size_t)c->C * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    for (uint32_t i = 0; i < c->C; ++i) out[i] = dev[c->bricked ? c->perm_host[i] : i];
    return MLEM_OK;
}

// ---- device-pointer entry points ---------------------------------------------
// Caller vectors are in natural voxel order; with the brick layout they are
// converted through the context's scratch buffers.
int mlem_fwproj_d(mlem_ctx* c, const float* x, float* y, uint32_t B, void* stream) {
    if (!c || !x || !y || B == 0) return fail(c, MLEM_ERR_INVALID, "bad argument");
    TRY(set_device(c));
    cudaStream_t st = (cudaStream_t)stream;
    const float* xd = x;
    if (c->bricked) {
        TRY(perm_scratch(c, (size_t)c->C * B));
        CK(c, permute_to_device(x, c->pscratch[0], c->perm, c->C, B, st));
        xd = c->pscratch[0];
    }
    const LaunchCfg cfg = cfg_for_frames(c, B);
    if (c->mirrored) {
        CK(c, cudaMemsetAsync(y, 0, (size_t)c->R * B * 4, st));
        for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile)
            CK(c, mirror_fwproj(csr_visit(c, c->tuning), c->mirror, xd, B, f0, cfg.frame_tile, y,
                                c->n_sm, c->tuning.blocks_per_sm, st));
        return MLEM_OK;
    }
    for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile)
        CK(c, fwproj(csr_visit(c, c->tuning), xd, B, f0, nullptr, nullptr, y, cfg, st));
    return MLEM_OK;
}

int mlem_bkproj_d(mlem_ctx* c, const float* y, float* x, uint32_t B, void* stream) {
    if (!c || !x || !y || B == 0) return fail(c, MLEM_ERR_INVALID, "bad argument");
    TRY(set_device(c));
    const LaunchCfg cfg = cfg_for_frames(c, B);
    cudaStream_t st = (cudaStream_t)stream;
    float* xd = x;
    if (c->bricked) {
        TRY(perm_scratch(c, (size_t)c->C * B));
        xd = c->pscratch[0];
    }
    for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile) {
        if (c->mirrored) {
            if (f0 == 0) CK(c, cudaMemsetAsync(xd, 0, (size_t)c->C * B * 4, st));
            CK(c, mirror_bkproj(csr_visit(c, c->tuning), c->mirror, y, nullptr, B, f0,
                                cfg.frame_tile, xd, c->n_sm, c->tuning.blocks_per_sm, st));
        } else if (c->has_csc) {
            CK(c, bkproj_csc(csc_view(c), y, B, f0, nullptr, nullptr, xd, cfg, st));
        } else {
            if (f0 == 0) CK(c, cudaMemsetAsync(xd, 0, (size_t)c->C * B * 4, st));
            CK(c, bkproj_scatter(csr_visit(c, c->tuning), y, B, f0, xd, cfg, st));
        }
    }
    if (c->bricked) CK(c, permute_to_natural(xd, x, c->perm, c->C, B, st));
    return MLEM_OK;
}

int mlem_fwproj_correl_d(mlem_ctx* c, const float* x, const int32_t* sino, float* correl,
                         uint32_t B, void* stream) {
    if (!c || !x || !sino || !correl || B == 0) return fail(c, MLEM_ERR_INVALID, "bad argument");
    TRY(set_device(c));
    cudaStream_t st = (cudaStream_t)stream;
    const float* xd = x;
    if (c->bricked) {
        TRY(perm_scratch(c, (size_t)c->C * B));
        CK(c, permute_to_device(x, c->pscratch[0], c->perm, c->C, B, st));
        xd = c->pscratch[0];
    }
    const LaunchCfg cfg = cfg_for_frames(c, B);
    if (c->mirrored) {  // the full rows' sums, then calcCorrel in place
        CK(c, cudaMemsetAsync(correl, 0, (size_t)c->R * B * 4, st));
        for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile)
            CK(c, mirror_fwproj(csr_visit(c, c->tuning), c->mirror, xd, B, f0, cfg.frame_tile,
                                correl, c->n_sm, c->tuning.blocks_per_sm, st));
        CK(c, correl_inplace(correl, sino, (uint64_t)c->R * B, st));
        return MLEM_OK;
    }
    for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile)
        CK(c, fwproj(csr_visit(c, c->tuning), xd, B, f0, sino, correl, nullptr, cfg, st));
    return MLEM_OK;
}

int mlem_fused_update_d(mlem_ctx* c, const float* x, const int32_t* sino, float* u, uint32_t B,
                        void* stream) {
    if (!c || !x || !u || B == 0) return fail(c, MLEM_ERR_INVALID, "bad argument");
    if (c->flags & MLEM_FLAG_EXACT)
        return fail(c, MLEM_ERR_STATE, "the one-pass method does not run in the bit-exact mode");
    // sino NULL: the context's own sinograms, whose list of rows with counts
    // the sorted visits walk (frames interleaved as the caller's vectors)
    const bool own = sino == nullptr;
    if (own) {
        if (!c->sino || c->B != B || c->Bp != B)
            return fail(c, MLEM_ERR_STATE,
                        "sino NULL needs the context's own sinograms with %u frames (it has %u, "
                        "padded to %u)", B, c->B, c->Bp);
        sino = c->sino;
    }
    TRY(set_device(c));
    cudaStream_t st = (cudaStream_t)stream;
    if (c->mirrored) {  // the full rows' sums in a buffer of the context, then the scatter
        const LaunchCfg cfg = cfg_for_frames(c, B);
        const float* xd = x;
        float* ud = u;
        if (c->bricked) {
            TRY(perm_scratch(c, (size_t)c->C * B));
            CK(c, permute_to_device(x, c->pscratch[0], c->perm, c->C, B, st));
            xd = c->pscratch[0];
            ud = c->pscratch[1];
        }
        if (c->f_mirror_d_floats < (size_t)c->R * B) {
            dev_free(c->f_mirror_d);
            c->f_mirror_d = nullptr;
            c->f_mirror_d_floats = 0;
            TRY(dev_alloc(c, &c->f_mirror_d, (size_t)c->R * B));
            c->f_mirror_d_floats = (size_t)c->R * B;
        }
        const SparseView v = csr_visit(c, c->tuning);
        CK(c, cudaMemsetAsync(c->f_mirror_d, 0, (size_t)c->R * B * 4, st));
        CK(c, cudaMemsetAsync(ud, 0, (size_t)c->C * B * 4, st));
        for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile)
            CK(c, mirror_fwproj(v, c->mirror, xd, B, f0, cfg.frame_tile, c->f_mirror_d, c->n_sm,
                                c->tuning.blocks_per_sm, st));
        for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile)
            CK(c, mirror_bkproj(v, c->mirror, c->f_mirror_d, sino, B, f0, cfg.frame_tile, ud,
                                c->n_sm, c->tuning.blocks_per_sm, st));
        if (c->bricked) CK(c, permute_to_natural(ud, u, c->perm, c->C, B, st));
        return MLEM_OK;
    }
    // the context's one-pass tuning when it has one, else sorted rows in chunks
    mlem_tuning t = c->tuning;
    if (t.bk_mode != MLEM_BK_FUSED) {
        t.visit = c->row_order ? MLEM_VISIT_SORTED_CHUNKED : MLEM_VISIT_FILE;
        t.blocks_per_sm = c->row_order ? 4 : 8;
        t.group = 32;
    }
    t.bk_mode = MLEM_BK_FUSED;
    t.frame_tile = cfg_for_frames(c, B).frame_tile;
    if (chunk_visit(t.visit)) t.group = 32;
    const float* xd = x;
    float* ud = u;
    if (c->bricked) {
        TRY(perm_scratch(c, (size_t)c->C * B));
        CK(c, permute_to_device(x, c->pscratch[0], c->perm, c->C, B, st));
        xd = c->pscratch[0];
        ud = c->pscratch[1];
    }
    if (c->n_long && c->f_long_d_floats < (size_t)c->n_long * B) {
        dev_free(c->f_long_d);
        c->f_long_d = nullptr;
        c->f_long_d_floats = 0;
        TRY(dev_alloc(c, &c->f_long_d, (size_t)c->n_long * B));
        c->f_long_d_floats = (size_t)c->n_long * B;
    }
    CK(c, cudaMemsetAsync(ud, 0, (size_t)c->C * B * 4, st));
    SparseView v = csr_visit(c, t);
    if (c->n_long) v.long_len = kLongRowElems;
    if (own && c->act_ready && t.visit != MLEM_VISIT_FILE) {
        v.order = c->act_order;
        v.vrange = c->act_ranges;
        v.n_dev = c->act_n;
    }
    // a counter of its own (a cache sector from the iteration's), so that this
    // call and the context's graph never share one
    TRY(fused_pass(c, t, v, xd, sino, ud, B, c->counter + 8, st));
    if (c->n_long)
        CK(c, long_rows_pass(csr_view(c), c->long_segs, c->n_long_segs, c->n_long, xd, B,
                             t.frame_tile, sino, c->f_long_d, ud, c->n_sm, st));
    if (c->bricked) CK(c, permute_to_natural(ud, u, c->perm, c->C, B, st));
    return MLEM_OK;
}

// The two one-pass kernels of the unrolled MLEM's backward pass (k_adjoint.cu):
// vectors in natural voxel order, one frame, row vectors by row.
static int backward_pass(mlem_ctx* c, int op, const float* x, const int32_t* sino, float* rows,
                         float* u, void* stream) {
    if (!c || !x || !sino || !rows || !u) return fail(c, MLEM_ERR_INVALID, "null argument");
    if (c->flags & MLEM_FLAG_EXACT)
        return fail(c, MLEM_ERR_STATE, "the one-pass method does not run in the bit-exact mode");
    if (c->mirrored)
        return fail(c, MLEM_ERR_STATE,
                    "the backward-pass kernels walk full rows (not MLEM_FLAG_MIRROR_KERNELS)");
    TRY(set_device(c));
    cudaStream_t st = (cudaStream_t)stream;
    const float* xd = x;
    float* ud = u;
    if (c->bricked) {
        TRY(perm_scratch(c, (size_t)c->C));
        CK(c, permute_to_device(x, c->pscratch[0], c->perm, c->C, 1, st));
        xd = c->pscratch[0];
        ud = c->pscratch[1];
    }
    CK(c, cudaMemsetAsync(ud, 0, (size_t)c->C * 4, st));
    // the counter slot of mlem_fused_update_d: these calls, like it, must not
    // run concurrently with the context's own iterations
    CK(c, adjoint_pass(op, csr_view(c), xd, sino, rows, ud, c->counter + 8, c->n_sm, st));
    if (c->bricked) CK(c, permute_to_natural(ud, u, c->perm, c->C, 1, st));
    return MLEM_OK;
}

int mlem_ratio_rows_d(mlem_ctx* c, const float* x, const int32_t* sino, float* rows, float* update,
                      void* stream) {
    return backward_pass(c, kOpRatio, x, sino, rows, update, stream);
}

int mlem_adjoint_update_d(mlem_ctx* c, const float* du, const int32_t* sino, const float* rows,
                          float* update, void* stream) {
    return backward_pass(c, kOpAdjoint, du, sino, const_cast<float*>(rows), update, stream);
}

int mlem_bkproj_update_d(mlem_ctx* c, const float* correl, float* x, uint32_t B, void* stream) {
    if (!c || !x || !correl || B == 0) return fail(c, MLEM_ERR_INVALID, "bad argument");
    if (!c->has_csc || c->mirrored)
        return fail(c, MLEM_ERR_STATE, "fused back projection needs the CSC copy of the full matrix");
    TRY(set_device(c));
    cudaStream_t st = (cudaStream_t)stream;
    float* xd = x;
    if (c->bricked) {
        TRY(perm_scratch(c, (size_t)c->C * B));
        CK(c, permute_to_device(x, c->pscratch[0], c->perm, c->C, B, st));
        xd = c->pscratch[0];
    }
    const LaunchCfg cfg = cfg_for_frames(c, B);
    for (uint32_t f0 = 0; f0 < B; f0 += (uint32_t)cfg.frame_tile)
        CK(c, bkproj_csc(csc_view(c), correl, B, f0, c->norm, xd, nullptr, cfg, st));
    if (c->bricked) CK(c, permute_to_natural(xd, x, c->perm, c->C, B, st));
    return MLEM_OK;
}

int mlem_apply_update_d(mlem_ctx* c, const float* update, float* x, uint32_t B, void* stream) {
    if (!c || !x || !update || B == 0) return fail(c, MLEM_ERR_INVALID, "bad argument");
    TRY(set_device(c));
    CK(c, apply_update(x, const_cast<float*>(update), c->norm_nat, c->C, B, false,
                       (cudaStream_t)stream));
    return MLEM_OK;
}

int mlem_norm_d(mlem_ctx* c, const float** norm) {
    if (!c || !norm) return fail(c, MLEM_ERR_INVALID, "null argument");
    *norm = c->norm_nat;
    return MLEM_OK;
}

int mlem_set_norm_d(mlem_ctx* c, const float* norm, void* stream) {
    if (!c || !norm) return fail(c, MLEM_ERR_INVALID, "null argument");
    TRY(set_device(c));
    cudaStream_t st = (cudaStream_t)stream;
    CK(c, cudaMemcpyAsync(c->norm_nat, norm, (size_t)c->C * 4, cudaMemcpyDeviceToDevice, st));
    if (c->bricked) CK(c, permute_to_device(c->norm_nat, c->norm, c->perm, c->C, 1, st));
    else CK(c, cudaMemcpyAsync(c->norm, norm, (size_t)c->C * 4, cudaMemcpyDeviceToDevice, st));
    CK(c, cudaMemcpyAsync(c->norm_host.data(), c->norm_nat, (size_t)c->C * 4,
                          cudaMemcpyDeviceToHost, st));
    CK(c, cudaStreamSynchronize(st));
    double s = 0.0;
    for (uint32_t i = 0; i < c->C; ++i) s += c->norm_host[i];
    c->sumnorm = s;
    return MLEM_OK;
}

int mlem_project_f64(mlem_ctx* c, const float* x, double* out) {
    if (!c || !x || !out) return fail(c, MLEM_ERR_INVALID, "null argument");
    if (c->mirrored)
        return fail(c, MLEM_ERR_STATE, "the FP64 projection reads the full matrix "
                    "(MLEM_FLAG_EXPAND_SYMMETRY), not the stored one");
    TRY(set_device(c));
    TRY(ensure_tmp(c));
    if (!c->tmp_d) TRY(dev_alloc(c, &c->tmp_d, std::max<uint32_t>(c->R, 1)));
    CK(c, cudaMemcpyAsync(c->tmp_c[0], x, (size_t)c->C * 4, cudaMemcpyHostToDevice, c->stream));
    const float* xd = c->tmp_c[0];
    if (c->bricked) {
        CK(c, permute_to_device(c->tmp_c[0], c->tmp_c[1], c->perm, c->C, 1, c->stream));
        xd = c->tmp_c[1];
    }
    CK(c, project_f64(csr_view(c), xd, c->tmp_d, c->stream));
    CK(c, cudaMemcpyAsync(out, c->tmp_d, (size_t)c->R * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MLEM_OK;
}

}  // extern "C"
