// capi_batch.cu -- multi-matrix batches (mlem_batch_* of include/mlem_b200.h):
// several contexts iterated together by persistent kernels (k_batch.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.hpp"
#include "host/errors.hpp"
#include "kernels.h"
#include "mlem_b200.h"

using namespace mlem;

// ===========================================================================
// Multi-matrix batches (mlem_batch_*): several contexts, one persistent
// kernel per iteration over work items cut from all their rows.
// ===========================================================================
struct mlem_batch {
    std::vector<mlem_ctx*> ctx;
    int device = 0;
    int n_sm = 148;
    cudaStream_t stream = nullptr;               // the first context's stream
    // Element prefix of each matrix in file order and in sorted order (empty
    // without a row order), for cutting items of equal cost.
    std::vector<std::vector<uint64_t>> pre_file, pre_sorted;
    // Per context, its sorted list of the rows with counts (ctx act_order,
    // rebuilt with each sinogram): the element prefix over it, its length, and
    // the sinogram upload it was read for.  The sorted visits walk it.
    std::vector<std::vector<uint64_t>> pre_active;
    std::vector<uint32_t> n_active;
    std::vector<char> has_active;
    std::vector<uint64_t> gen_seen;
    int policy = MLEM_BATCH_INTERLEAVED;
    int visit = MLEM_VISIT_FILE;
    int tile = 0;  // frames per pass of every context without a tile of its own
    std::vector<int> tiles;  // per context: 0 = the batch tile, else its own frame tile
    std::vector<int> visits;  // per context: -1 = the batch visit, else its own row visit
    uint32_t items_per_block = 4;
    int blocks_per_sm = 4;  // k_batch_fused is bounded to 64 registers: 4 x 256 threads per SM
    double ms_per_iter = 0.0;

    // The contexts that share a frame tile and a row visit form a group: one
    // kernel per group and iteration, heaviest group first.  A group's table
    // is the kernels' parameter; its items are b->items[item0, item0 +
    // n_items), with `mat` indexing the group's table; ctx_of maps the table
    // back to contexts.
    struct Group {
        int tile = 1;
        int visit = MLEM_VISIT_FILE;
        double cost = 0.0;
        BatchTable table{};
        std::vector<size_t> ctx_of;
        uint32_t item0 = 0, n_items = 0;
    };
    std::vector<Group> groups;
    BatchTable table{};  // every context in order; the groups' tables are cut from it
    std::vector<BatchItem> items;
    BatchItem* items_d = nullptr;
    size_t items_cap = 0;
    unsigned int* counter = nullptr;  // one counter per group, kCounterStride apart
    bool scheduled = false;

    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    bool graph_dirty = true;
    std::vector<const void*> graph_sig;  // context pointers the graph holds

    std::string err;
};

namespace {

int bfail(mlem_batch* b, int status, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
int bfail(mlem_batch* b, int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return set_error(b ? &b->err : nullptr, status, "%s", buf);
}

#define BCK(b, call)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? MLEM_ERR_NOMEM : MLEM_ERR_CUDA, \
                         "%s: %s (%s:%d)", cudaGetErrorName(e_), cudaGetErrorString(e_),   \
                         __FILE__, __LINE__);                                               \
    } while (0)

// A context's status, carried over into the batch's message.
int bctx(mlem_batch* b, mlem_ctx* c, int s) {
    if (s == MLEM_OK) return s;
    return bfail(b, s, "%s", c->err.c_str());
}

bool tile_ok(int t, uint32_t Bp) {
    return (t == 1 || t == 2 || t == 4 || t == 8 || t == 16) && Bp % (uint32_t)t == 0;
}

bool tile_ok_all(const mlem_batch* b, int t) {
    for (const mlem_ctx* c : b->ctx)
        if (!tile_ok(t, c->Bp)) return false;
    return true;
}

// The batch tile must divide the padded frame count of every context that
// has no tile of its own.
bool batch_tile_ok(const mlem_batch* b, int t) {
    for (size_t i = 0; i < b->ctx.size(); ++i)
        if (!b->tiles[i] && !tile_ok(t, b->ctx[i]->Bp)) return false;
    return true;
}

// Widest tile (<= 16) dividing every padded frame count.
int batch_default_tile(const mlem_batch* b) {
    for (int t : {16, 8, 4, 2})
        if (tile_ok_all(b, t)) return t;
    return 1;
}

int eff_tile(const mlem_batch* b, size_t i) { return b->tiles[i] ? b->tiles[i] : b->tile; }
int eff_visit(const mlem_batch* b, size_t i) { return b->visits[i] >= 0 ? b->visits[i] : b->visit; }

// Context i's sorted visit walks only its rows with counts (as its own
// one-pass iteration does); its visiting positions are then [0, n_active).
bool uses_active(const mlem_batch* b, size_t i) {
    return b->has_active[i] && eff_visit(b, i) != MLEM_VISIT_FILE;
}
uint32_t rows_of(const mlem_batch* b, size_t i) {
    return uses_active(b, i) ? b->n_active[i] : b->ctx[i]->R;
}

// Per-group counters sit a cache sector apart.  Groups are distinct (tile,
// visit) pairs: at most 5 tiles x 3 visits.
constexpr uint32_t kCounterStride = 8;
constexpr uint32_t kMaxGroups = 16;
static_assert(5 * 3 <= kMaxGroups, "one counter per (frame tile, row visit) group");

// Cost of rows [r0, r1) of context i: element bytes once per frame-tile
// pass, one gather and one scatter of 4 bytes per element and frame, and the
// row's offsets, sinogram entries and sums.
double item_cost(const mlem_batch* b, size_t i, uint32_t r0, uint32_t r1) {
    const mlem_ctx* c = b->ctx[i];
    const std::vector<uint64_t>& pre =
        uses_active(b, i) ? b->pre_active[i]
        : (eff_visit(b, i) != MLEM_VISIT_FILE && !b->pre_sorted[i].empty()) ? b->pre_sorted[i]
                                                                             : b->pre_file[i];
    const double nnz = (double)(pre[r1] - pre[r0]);
    const double passes = (double)(c->Bp / (uint32_t)eff_tile(b, i));
    return nnz * (8.0 * passes + 8.0 * c->Bp) + (double)(r1 - r0) * (16.0 + 8.0 * c->Bp);
}

// Group the contexts by frame tile and row visit (heaviest group first) with each group's
// table taken from b->table.  Returns true when the grouping differs from
// the current one (the items must then be cut again); the item ranges of an
// unchanged grouping are kept.
bool build_groups(mlem_batch* b) {
    std::vector<mlem_batch::Group> gs;
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        const int t = eff_tile(b, i), v = eff_visit(b, i);
        auto it = std::find_if(gs.begin(), gs.end(),
                               [&](const mlem_batch::Group& g) { return g.tile == t && g.visit == v; });
        if (it == gs.end()) {
            gs.emplace_back();
            gs.back().tile = t;
            gs.back().visit = v;
            gs.back().table.n = 0;
            gs.back().table.row_base[0] = 0;
            it = gs.end() - 1;
        }
        BatchTable& t_ = it->table;
        t_.mats[t_.n] = b->table.mats[i];
        t_.row_base[t_.n + 1] = t_.row_base[t_.n] + rows_of(b, i);
        ++t_.n;
        it->ctx_of.push_back(i);
        it->cost += item_cost(b, i, 0, rows_of(b, i));
    }
    std::stable_sort(gs.begin(), gs.end(), [](const mlem_batch::Group& a, const mlem_batch::Group& c) {
        return a.cost > c.cost;
    });
    bool same = gs.size() == b->groups.size();
    for (size_t g = 0; same && g < gs.size(); ++g)
        same = gs[g].tile == b->groups[g].tile && gs[g].visit == b->groups[g].visit &&
               gs[g].ctx_of == b->groups[g].ctx_of;
    if (same)
        for (size_t g = 0; g < gs.size(); ++g) {
            gs[g].item0 = b->groups[g].item0;
            gs[g].n_items = b->groups[g].n_items;
        }
    b->groups = std::move(gs);
    return !same;
}

// Context i's list of rows with counts, read from the device after a
// sinogram upload, and the element prefix over it (for cutting items).
int read_active(mlem_batch* b, size_t i) {
    mlem_ctx* c = b->ctx[i];
    b->has_active[i] = 0;
    b->n_active[i] = 0;
    b->pre_active[i].clear();
    if (!c->act_ready || !c->row_order) return MLEM_OK;
    uint32_t n = 0;
    BCK(b, cudaMemcpyAsync(&n, c->act_n, 4, cudaMemcpyDeviceToHost, c->stream));
    BCK(b, cudaStreamSynchronize(c->stream));
    std::vector<uint32_t> ord(n);
    if (n) BCK(b, cudaMemcpyAsync(ord.data(), c->act_order, (size_t)n * 4, cudaMemcpyDeviceToHost,
                                  c->stream));
    BCK(b, cudaStreamSynchronize(c->stream));
    const std::vector<uint64_t>& pf = b->pre_file[i];
    std::vector<uint64_t>& pa = b->pre_active[i];
    pa.resize((size_t)n + 1);
    pa[0] = 0;
    for (uint32_t k = 0; k < n; ++k) pa[k + 1] = pa[k] + (pf[ord[k] + 1] - pf[ord[k]]);
    c->act_rows = n;
    b->n_active[i] = n;
    b->has_active[i] = 1;
    return MLEM_OK;
}

// Cut the rows of every group's matrices into items of about group total /
// (resident blocks x items_per_block) cost; within a group, full items of
// the costliest matrix first in row order (neighbouring rows share image
// voxels in L2), then the ragged remainders, heaviest first.
int batch_schedule(mlem_batch* b) {
    b->items.clear();
    if (b->policy != MLEM_BATCH_ITEMS) {  // the interleaved schedule needs no items
        for (auto& g : b->groups) g.item0 = g.n_items = 0;
        b->scheduled = true;
        b->graph_dirty = true;
        return MLEM_OK;
    }
    const double resident = (double)b->n_sm * (double)b->blocks_per_sm;
    for (auto& g : b->groups) {
        const size_t n = g.ctx_of.size();
        std::vector<double> total(n, 0.0);
        for (size_t j = 0; j < n; ++j) total[j] = item_cost(b, g.ctx_of[j], 0, rows_of(b, g.ctx_of[j]));
        const double target = std::max(g.cost / (resident * (double)b->items_per_block), 1.0);
        std::vector<size_t> order(n);
        for (size_t j = 0; j < n; ++j) order[j] = j;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t c) { return total[a] > total[c]; });
        std::vector<BatchItem> full;
        std::vector<std::pair<double, BatchItem>> tail;
        for (size_t j : order) {
            const size_t i = g.ctx_of[j];
            const uint32_t R = rows_of(b, i);
            uint32_t r0 = 0;
            while (r0 < R) {
                uint32_t lo = r0 + 1, hi = R;  // smallest r1 whose cost reaches the target
                while (lo < hi) {
                    const uint32_t mid = lo + (hi - lo) / 2;
                    if (item_cost(b, i, r0, mid) >= target) hi = mid;
                    else lo = mid + 1;
                }
                const BatchItem it{(uint32_t)j, r0, lo, 0u};
                const double cost = item_cost(b, i, r0, lo);
                if (cost >= 0.5 * target) full.push_back(it);
                else tail.emplace_back(cost, it);
                r0 = lo;
            }
        }
        std::stable_sort(tail.begin(), tail.end(),
                         [](const std::pair<double, BatchItem>& a,
                            const std::pair<double, BatchItem>& c) { return a.first > c.first; });
        if (b->items.size() + full.size() + tail.size() > 0xffffffffull)
            return bfail(b, MLEM_ERR_INVALID, "too many work items");
        g.item0 = (uint32_t)b->items.size();
        b->items.insert(b->items.end(), full.begin(), full.end());
        for (auto& t : tail) b->items.push_back(t.second);
        g.n_items = (uint32_t)b->items.size() - g.item0;
    }
    if (b->items.size() > b->items_cap) {
        dev_free(b->items_d);
        b->items_d = nullptr;
        b->items_cap = 0;
        BCK(b, cudaMalloc(&b->items_d, b->items.size() * sizeof(BatchItem)));
        b->items_cap = b->items.size();
    }
    if (!b->items.empty())
        BCK(b, cudaMemcpyAsync(b->items_d, b->items.data(), b->items.size() * sizeof(BatchItem),
                               cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    b->scheduled = true;
    b->graph_dirty = true;
    return MLEM_OK;
}

// Check the contexts, make room for `chunk` iterations of statistics, fill
// the matrix table and (re)schedule when a context changed.
int batch_refresh(mlem_batch* b, int chunk) {
    bool reschedule = !b->scheduled;
    std::vector<const void*> sig;
    BatchTable& t = b->table;
    t.n = (uint32_t)b->ctx.size();
    t.row_base[0] = 0;
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        mlem_ctx* c = b->ctx[i];
        if (!c->B || !c->images_ready)
            return bfail(b, MLEM_ERR_STATE, "context %zu: sinograms and images not set", i);
        if (c->n_subsets > 1)
            return bfail(b, MLEM_ERR_STATE, "context %zu: ordered subsets do not run in a batch", i);
        if (c->stream != b->stream) BCK(b, cudaStreamSynchronize(c->stream));
        TRY(bctx(b, c, ensure_history(c, chunk)));
        if (c->sino_gen != b->gen_seen[i]) {  // new sinograms: another list of rows with counts
            TRY(read_active(b, i));
            b->gen_seen[i] = c->sino_gen;
            reschedule = true;
            b->graph_dirty = true;
        }
        if (t.mats[i].Bp != c->Bp) reschedule = true;
        SparseView v = csr_view(c);
        if (c->n_long) v.long_len = kLongRowElems;  // long rows: segments in their own kernels
        if (eff_visit(b, i) == MLEM_VISIT_FILE) {
            v.order = nullptr;
            v.vrange = nullptr;
        } else if (uses_active(b, i)) {
            v.order = c->act_order;
            v.vrange = c->act_ranges;
            v.n = b->n_active[i];
        }
        t.mats[i] = BatchMat{v, c->x, c->sino, c->update, c->Bp, 0u};
        t.row_base[i + 1] = t.row_base[i] + rows_of(b, i);
        for (const void* p : {(const void*)c->x, (const void*)c->sino, (const void*)c->update,
                              (const void*)c->norm, (const void*)c->stats_scratch,
                              (const void*)c->stats_slot, (const void*)c->hist_sums,
                              (const void*)c->hist_zeros, (const void*)c->hist_subn})
            sig.push_back(p);
        sig.push_back(reinterpret_cast<const void*>((uintptr_t)c->Bp));
        sig.push_back(reinterpret_cast<const void*>((uintptr_t)c->B));
    }
    for (size_t i = 0; i < b->ctx.size(); ++i)
        if (b->tiles[i] && !tile_ok(b->tiles[i], b->ctx[i]->Bp)) {  // new frame count
            b->tiles[i] = 0;
            reschedule = true;
        }
    if (!batch_tile_ok(b, b->tile)) {
        b->tile = batch_default_tile(b);
        reschedule = true;
    }
    if (sig != b->graph_sig) {
        b->graph_dirty = true;
        b->graph_sig = sig;
    }
    if (build_groups(b)) reschedule = true;
    if (reschedule) TRY(batch_schedule(b));
    return MLEM_OK;
}

int bmark(mlem_batch* b, const PhaseEvents* pe, int i) {
    if (pe) BCK(b, cudaEventRecord(pe->ev[i], b->stream));
    return MLEM_OK;
}

// One iteration of every context: the multi-matrix pass, then per context
// calcUpdate (zeroing its update vector) and the image statistics.
int batch_enqueue(mlem_batch* b, bool stats, const PhaseEvents* pe = nullptr) {
    cudaStream_t st = b->stream;
    TRY(bmark(b, pe, 0));
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        const mlem_batch::Group& g = b->groups[gi];
        unsigned int* counter = b->counter + gi * kCounterStride;
        const BatchItem* items = b->items_d + g.item0;
        if (b->policy == MLEM_BATCH_ITEMS && g.visit == MLEM_VISIT_SORTED_STAGED)
            BCK(b, batch_staged(g.table, items, g.n_items, counter, g.tile, b->n_sm,
                                b->blocks_per_sm, st));
        else if (b->policy == MLEM_BATCH_ITEMS)
            BCK(b, batch_fused(g.table, items, g.n_items, counter, g.tile,
                               g.visit == MLEM_VISIT_SORTED, b->n_sm, b->blocks_per_sm, st));
        else
            BCK(b, batch_interleaved(g.table, g.tile, g.visit == MLEM_VISIT_SORTED, b->n_sm,
                                     b->blocks_per_sm, st));
    }
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        mlem_ctx* c = b->ctx[i];
        if (c->n_long)
            BCK(b, long_rows_pass(csr_view(c), c->long_segs, c->n_long_segs, c->n_long, c->x, c->Bp,
                                  eff_tile(b, i), c->sino, c->f_long, c->update, b->n_sm, st));
    }
    TRY(bmark(b, pe, 1));
    TRY(bmark(b, pe, 2));
    for (mlem_ctx* c : b->ctx) BCK(b, apply_update(c->x, c->update, c->norm, c->C, c->Bp, true, st));
    TRY(bmark(b, pe, 3));
    if (stats)
        for (mlem_ctx* c : b->ctx)
            BCK(b, image_stats(c->x, c->C, c->Bp, c->B, c->stats_scratch, c->stats_slot,
                               c->hist_sums, c->hist_zeros, c->hist_subn, st));
    TRY(bmark(b, pe, 4));
    return MLEM_OK;
}

int batch_reset_slots(mlem_batch* b) {
    for (mlem_ctx* c : b->ctx) BCK(b, cudaMemsetAsync(c->stats_slot, 0, 4, b->stream));
    return MLEM_OK;
}

void batch_drop_graph(mlem_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_iters = 0;
}

int batch_capture(mlem_batch* b, int n) {
    batch_drop_graph(b);
    BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int s = batch_reset_slots(b);
    for (int i = 0; i < n && s == MLEM_OK; ++i) s = batch_enqueue(b, true);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (s != MLEM_OK) { if (g) cudaGraphDestroy(g); return s; }
    if (e != cudaSuccess) return bfail(b, MLEM_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bfail(b, MLEM_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
    b->graph_iters = n;
    b->graph_dirty = false;
    return MLEM_OK;
}

// Average ms of `reps` iterations (after one warm-up) with the current schedule.
int batch_time(mlem_batch* b, int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms) {
    TRY(batch_enqueue(b, false));
    BCK(b, cudaEventRecord(e0, b->stream));
    for (int i = 0; i < reps; ++i) TRY(batch_enqueue(b, false));
    BCK(b, cudaEventRecord(e1, b->stream));
    BCK(b, cudaEventSynchronize(e1));
    float t = 0.0f;
    BCK(b, cudaEventElapsedTime(&t, e0, e1));
    *ms = t / reps;
    return MLEM_OK;
}

void batch_free(mlem_batch* b) {
    batch_drop_graph(b);
    dev_free(b->items_d);
    dev_free(b->counter);
}

}  // namespace

extern "C" {

const char* mlem_batch_last_error(const mlem_batch* b) {
    return b ? b->err.c_str() : global_error().c_str();
}

int mlem_batch_create(mlem_batch** out, mlem_ctx* const* ctxs, uint32_t n_ctx) {
    if (!out || !ctxs) return bfail(nullptr, MLEM_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n_ctx == 0 || n_ctx > MLEM_BATCH_MAX_MATRICES)
        return bfail(nullptr, MLEM_ERR_INVALID, "a batch holds 1..%d contexts (got %u)",
                     MLEM_BATCH_MAX_MATRICES, n_ctx);
    for (uint32_t i = 0; i < n_ctx; ++i) {
        const mlem_ctx* c = ctxs[i];
        if (!c) return bfail(nullptr, MLEM_ERR_INVALID, "context %u is null", i);
        for (uint32_t j = 0; j < i; ++j)
            if (ctxs[j] == c) return bfail(nullptr, MLEM_ERR_INVALID, "context %u repeats %u", i, j);
        if (c->device != ctxs[0]->device)
            return bfail(nullptr, MLEM_ERR_INVALID, "context %u is on device %d, not %d", i,
                         c->device, ctxs[0]->device);
        if (c->flags & MLEM_FLAG_EXACT)
            return bfail(nullptr, MLEM_ERR_INVALID,
                         "context %u was created with MLEM_FLAG_EXACT (bit-exact kernels)", i);
        if (c->mirrored)
            return bfail(nullptr, MLEM_ERR_INVALID,
                         "context %u was created with MLEM_FLAG_MIRROR_KERNELS (a batch runs the "
                         "one-pass kernels over full matrices)", i);
        if (!c->B || !c->images_ready)
            return bfail(nullptr, MLEM_ERR_STATE, "context %u: sinograms and images not set", i);
    }
    mlem_batch* b = new mlem_batch();
    b->ctx.assign(ctxs, ctxs + n_ctx);
    b->tiles.assign(n_ctx, 0);
    b->visits.assign(n_ctx, -1);
    b->device = ctxs[0]->device;
    b->n_sm = ctxs[0]->n_sm;
    b->stream = ctxs[0]->stream;
    int s = MLEM_OK;
    auto bail = [&](int status) {
        batch_free(b);
        global_error() = b->err;
        delete b;
        return status;
    };
    if (cudaSetDevice(b->device) != cudaSuccess)
        return bail(bfail(b, MLEM_ERR_CUDA, "cudaSetDevice(%d) failed", b->device));
    b->pre_file.resize(n_ctx);
    b->pre_sorted.resize(n_ctx);
    b->pre_active.resize(n_ctx);
    b->n_active.assign(n_ctx, 0);
    b->has_active.assign(n_ctx, 0);
    b->gen_seen.assign(n_ctx, ~0ull);  // read every context's list at the first refresh
    for (uint32_t i = 0; i < n_ctx; ++i) {
        mlem_ctx* c = ctxs[i];
        std::vector<uint64_t>& pre = b->pre_file[i];
        pre.resize((size_t)c->R + 1);
        std::vector<uint32_t> order(c->row_order ? c->R : 0);
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpy(pre.data(), c->row_ptr, ((size_t)c->R + 1) * 8, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && c->row_order)
            e = cudaMemcpy(order.data(), c->row_order, (size_t)c->R * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess)
            return bail(bfail(b, MLEM_ERR_CUDA, "row offsets of context %u: %s", i,
                              cudaGetErrorString(e)));
        if (c->n_long) {  // rows above the long-row limit run in their own kernels: no item cost
            uint64_t prev = pre[0];
            for (uint32_t r = 0; r < c->R; ++r) {
                const uint64_t end = pre[r + 1];
                const uint64_t len = end - prev;
                prev = end;
                pre[r + 1] = pre[r] + (len > kLongRowElems ? 0 : len);
            }
        }
        if (c->row_order) {  // element prefix in sorted order (for the sorted visits)
            std::vector<uint64_t>& ps = b->pre_sorted[i];
            ps.resize((size_t)c->R + 1);
            ps[0] = 0;
            for (uint32_t k = 0; k < c->R; ++k) ps[k + 1] = ps[k] + (pre[order[k] + 1] - pre[order[k]]);
        }
    }
    if (cudaMalloc(&b->counter, kMaxGroups * kCounterStride * sizeof(unsigned int)) != cudaSuccess) {
        cudaGetLastError();
        return bail(bfail(b, MLEM_ERR_NOMEM, "batch descriptors: cudaMalloc failed"));
    }
    s = batch_refresh(b, 1);
    if (s != MLEM_OK) return bail(s);
    *out = b;
    return MLEM_OK;
}

void mlem_batch_destroy(mlem_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    batch_free(b);
    delete b;
}

int mlem_batch_set_schedule(mlem_batch* b, int policy, uint32_t items_per_block,
                            int blocks_per_sm, int frame_tile, int visit) {
    if (!b) return bfail(nullptr, MLEM_ERR_INVALID, "null batch");
    if (policy != MLEM_BATCH_INTERLEAVED && policy != MLEM_BATCH_ITEMS)
        return bfail(b, MLEM_ERR_INVALID, "unknown batch schedule %d", policy);
    if (visit != MLEM_VISIT_FILE && visit != MLEM_VISIT_SORTED &&
        !(visit == MLEM_VISIT_SORTED_STAGED && policy == MLEM_BATCH_ITEMS))
        return bfail(b, MLEM_ERR_INVALID, "row visiting order %d is not a batch order for schedule %d",
                     visit, policy);
    if (visit != MLEM_VISIT_FILE)
        for (size_t i = 0; i < b->ctx.size(); ++i)
            if (!b->ctx[i]->row_order)
                return bfail(b, MLEM_ERR_INVALID,
                             "sorted row visiting: context %zu has no row order (MLEM_FLAG_NO_ROW_ORDER)", i);
    if (items_per_block < 1 || items_per_block > 1024)
        return bfail(b, MLEM_ERR_INVALID, "items_per_block must be 1..1024 (got %u)", items_per_block);
    if (blocks_per_sm < 1 || blocks_per_sm > 32)
        return bfail(b, MLEM_ERR_INVALID, "blocks_per_sm must be 1..32 (got %d)", blocks_per_sm);
    if (frame_tile != 0 && !tile_ok_all(b, frame_tile))
        return bfail(b, MLEM_ERR_INVALID,
                     "frame tile %d: must be 1, 2, 4, 8 or 16 and divide every context's padded "
                     "frame count", frame_tile);
    BCK(b, cudaSetDevice(b->device));
    b->policy = policy;
    b->visit = visit;
    std::fill(b->visits.begin(), b->visits.end(), -1);  // one visit for every context again
    b->items_per_block = items_per_block;
    b->blocks_per_sm = blocks_per_sm;
    if (frame_tile != 0) {  // one tile for every context again
        b->tile = frame_tile;
        std::fill(b->tiles.begin(), b->tiles.end(), 0);
    }
    b->scheduled = false;
    b->graph_dirty = true;
    return batch_refresh(b, 1);
}

int mlem_batch_get_schedule(const mlem_batch* b, int* policy, uint32_t* items_per_block,
                            int* blocks_per_sm, int* frame_tile, int* visit, uint32_t* n_items,
                            double* ms_per_iter) {
    if (!b) return bfail(nullptr, MLEM_ERR_INVALID, "null batch");
    if (policy) *policy = b->policy;
    if (visit) *visit = b->visit;
    if (items_per_block) *items_per_block = b->items_per_block;
    if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
    if (frame_tile) *frame_tile = b->tile;
    if (n_items) *n_items = (uint32_t)b->items.size();
    if (ms_per_iter) *ms_per_iter = b->ms_per_iter;
    return MLEM_OK;
}

int mlem_batch_set_tiles(mlem_batch* b, const int* tiles) {
    if (!b || !tiles) return bfail(b, MLEM_ERR_INVALID, "null argument");
    for (size_t i = 0; i < b->ctx.size(); ++i)
        if (tiles[i] != 0 && !tile_ok(tiles[i], b->ctx[i]->Bp))
            return bfail(b, MLEM_ERR_INVALID,
                         "context %zu: frame tile %d must be 1, 2, 4, 8 or 16 and divide its padded "
                         "frame count %u", i, tiles[i], b->ctx[i]->Bp);
    std::vector<int> keep = b->tiles;
    b->tiles.assign(tiles, tiles + b->ctx.size());
    if (!batch_tile_ok(b, b->tile)) {
        b->tiles = keep;
        return bfail(b, MLEM_ERR_INVALID, "the batch frame tile %d does not divide the padded frame "
                     "count of a context without a tile of its own", b->tile);
    }
    BCK(b, cudaSetDevice(b->device));
    b->scheduled = false;
    b->graph_dirty = true;
    return batch_refresh(b, 1);
}

int mlem_batch_get_tiles(const mlem_batch* b, int* tiles) {
    if (!b || !tiles) return bfail(const_cast<mlem_batch*>(b), MLEM_ERR_INVALID, "null argument");
    for (size_t i = 0; i < b->ctx.size(); ++i) tiles[i] = eff_tile(b, i);
    return MLEM_OK;
}

int mlem_batch_set_visits(mlem_batch* b, const int* visits) {
    if (!b || !visits) return bfail(b, MLEM_ERR_INVALID, "null argument");
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        const int v = visits[i];
        if (v != -1 && v != MLEM_VISIT_FILE && v != MLEM_VISIT_SORTED &&
            !(v == MLEM_VISIT_SORTED_STAGED && b->policy == MLEM_BATCH_ITEMS))
            return bfail(b, MLEM_ERR_INVALID,
                         "context %zu: row visiting order %d is not a batch order for schedule %d", i,
                         v, b->policy);
        if (v > MLEM_VISIT_FILE && !b->ctx[i]->row_order)
            return bfail(b, MLEM_ERR_INVALID,
                         "sorted row visiting: context %zu has no row order (MLEM_FLAG_NO_ROW_ORDER)", i);
    }
    BCK(b, cudaSetDevice(b->device));
    b->visits.assign(visits, visits + b->ctx.size());
    b->scheduled = false;
    b->graph_dirty = true;
    return batch_refresh(b, 1);
}

int mlem_batch_get_visits(const mlem_batch* b, int* visits) {
    if (!b || !visits) return bfail(const_cast<mlem_batch*>(b), MLEM_ERR_INVALID, "null argument");
    for (size_t i = 0; i < b->ctx.size(); ++i) visits[i] = eff_visit(b, i);
    return MLEM_OK;
}

int mlem_batch_autotune(mlem_batch* b, double* ms_per_iter) {
    if (!b) return bfail(nullptr, MLEM_ERR_INVALID, "null batch");
    BCK(b, cudaSetDevice(b->device));
    TRY(batch_refresh(b, 1));
    // Tuning runs real iterations: save the images.
    std::vector<float*> saved(b->ctx.size(), nullptr);
    auto release = [&]() {
        for (float* p : saved) dev_free(p);
    };
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        mlem_ctx* c = b->ctx[i];
        if (cudaMalloc(&saved[i], (size_t)c->C * c->Bp * 4) != cudaSuccess) {
            cudaGetLastError();
            release();
            return bfail(b, MLEM_ERR_NOMEM, "autotune: no room to save the images of context %zu", i);
        }
        if (cudaMemcpyAsync(saved[i], c->x, (size_t)c->C * c->Bp * 4, cudaMemcpyDeviceToDevice,
                            b->stream) != cudaSuccess) {
            release();
            return bfail(b, MLEM_ERR_CUDA, "autotune: saving images failed");
        }
    }
    auto restore = [&]() -> int {
        for (size_t i = 0; i < b->ctx.size(); ++i) {
            mlem_ctx* c = b->ctx[i];
            BCK(b, cudaMemcpyAsync(c->x, saved[i], (size_t)c->C * c->Bp * 4,
                                   cudaMemcpyDeviceToDevice, b->stream));
        }
        return MLEM_OK;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int s = MLEM_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        s = bfail(b, MLEM_ERR_CUDA, "event creation failed");
    uint32_t best_ipb = b->items_per_block;
    int best_bps = b->blocks_per_sm, best_tile = b->tile, best_policy = b->policy;
    int best_visit = b->visit;
    double best = 1e30;
    auto trial = [&](int policy, uint32_t ipb, int bps, int tile, int visit) -> int {
        TRY(mlem_batch_set_schedule(b, policy, ipb, bps, tile, visit));
        double ms = 0.0;
        TRY(batch_time(b, 2, e0, e1, &ms));
        TRY(restore());
        if (ms < best) {
            best = ms;
            best_policy = policy;
            best_ipb = ipb;
            best_bps = bps;
            best_tile = tile;
            best_visit = visit;
        }
        return MLEM_OK;
    };
    bool sorted_ok = true;
    for (const mlem_ctx* c : b->ctx) sorted_ok = sorted_ok && c->row_order;
    // The frame tile and the row order with the interleaved schedule first,
    // then the resident blocks, then the items schedule with that tile.
    for (int t : {16, 8, 4, 2, 1})
        for (int v : {MLEM_VISIT_FILE, MLEM_VISIT_SORTED})
            if (s == MLEM_OK && tile_ok_all(b, t) && (v == MLEM_VISIT_FILE || sorted_ok))
                s = trial(MLEM_BATCH_INTERLEAVED, best_ipb, 4, t, v);
    for (int bps : {3, 8})
        if (s == MLEM_OK) s = trial(MLEM_BATCH_INTERLEAVED, best_ipb, bps, best_tile, best_visit);
    for (uint32_t ipb : {1u, 4u, 16u, 64u})
        for (int v : {MLEM_VISIT_FILE, MLEM_VISIT_SORTED, MLEM_VISIT_SORTED_STAGED})
            if (s == MLEM_OK && (v == MLEM_VISIT_FILE || sorted_ok))
                s = trial(MLEM_BATCH_ITEMS, ipb, 4, best_tile, v);
    // Then, with that schedule, a frame tile of its own for each context,
    // heaviest first, and then a row visit of its own (contexts sharing a
    // tile and a visit share a kernel).
    std::vector<int> best_tiles(b->ctx.size(), 0), best_visits(b->ctx.size(), -1);
    if (s == MLEM_OK && b->ctx.size() > 1) {
        s = mlem_batch_set_schedule(b, best_policy, best_ipb, best_bps, best_tile, best_visit);
        std::vector<size_t> order(b->ctx.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::vector<double> cost(b->ctx.size());
        for (size_t i = 0; i < cost.size(); ++i) cost[i] = item_cost(b, i, 0, rows_of(b, i));
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t c) { return cost[a] > cost[c]; });
        for (size_t i : order)
            for (int t : {16, 8, 4, 2, 1}) {
                if (s != MLEM_OK || !tile_ok(t, b->ctx[i]->Bp)) continue;
                if (t == (best_tiles[i] ? best_tiles[i] : best_tile)) continue;
                std::vector<int> cand = best_tiles;
                cand[i] = t;
                s = mlem_batch_set_tiles(b, cand.data());
                double ms = 0.0;
                if (s == MLEM_OK) s = batch_time(b, 2, e0, e1, &ms);
                if (s == MLEM_OK) s = restore();
                if (s == MLEM_OK && ms < best) {
                    best = ms;
                    best_tiles = cand;
                }
            }
        if (s == MLEM_OK) s = mlem_batch_set_tiles(b, best_tiles.data());
        for (size_t i : order)
            for (int v : {MLEM_VISIT_FILE, MLEM_VISIT_SORTED, MLEM_VISIT_SORTED_STAGED}) {
                if (s != MLEM_OK || v == (best_visits[i] >= 0 ? best_visits[i] : best_visit)) continue;
                if (v != MLEM_VISIT_FILE && !b->ctx[i]->row_order) continue;
                if (v == MLEM_VISIT_SORTED_STAGED && best_policy != MLEM_BATCH_ITEMS) continue;
                std::vector<int> cand = best_visits;
                cand[i] = v;
                s = mlem_batch_set_visits(b, cand.data());
                double ms = 0.0;
                if (s == MLEM_OK) s = batch_time(b, 2, e0, e1, &ms);
                if (s == MLEM_OK) s = restore();
                if (s == MLEM_OK && ms < best) {
                    best = ms;
                    best_visits = cand;
                }
            }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s == MLEM_OK) s = restore();
    if (s == MLEM_OK && cudaStreamSynchronize(b->stream) != cudaSuccess)
        s = bfail(b, MLEM_ERR_CUDA, "autotune: synchronize failed");
    release();
    if (s != MLEM_OK) return s;
    TRY(mlem_batch_set_schedule(b, best_policy, best_ipb, best_bps, best_tile, best_visit));
    TRY(mlem_batch_set_tiles(b, best_tiles.data()));
    TRY(mlem_batch_set_visits(b, best_visits.data()));
    b->ms_per_iter = best;
    if (ms_per_iter) *ms_per_iter = best;
    return MLEM_OK;
}

int mlem_batch_iterate(mlem_batch* b, int n, double* const* sums) {
    if (!b) return bfail(nullptr, MLEM_ERR_INVALID, "null batch");
    if (n < 0) return bfail(b, MLEM_ERR_INVALID, "negative iteration count");
    if (n == 0) return MLEM_OK;
    BCK(b, cudaSetDevice(b->device));
    const int chunk = std::min(n, 64);
    TRY(batch_refresh(b, chunk));
    if (b->graph_dirty || !b->graph || b->graph_iters != chunk) TRY(batch_capture(b, chunk));
    int done = 0;
    while (done < n) {
        const int k = std::min(chunk, n - done);
        if (k == chunk) {
            BCK(b, cudaGraphLaunch(b->graph, b->stream));
        } else {
            TRY(batch_reset_slots(b));
            for (int i = 0; i < k; ++i) TRY(batch_enqueue(b, true));
        }
        bool any = false;
        for (size_t i = 0; sums && i < b->ctx.size(); ++i) {
            if (!sums[i]) continue;
            const mlem_ctx* c = b->ctx[i];
            BCK(b, cudaMemcpyAsync(sums[i] + (size_t)done * c->B, c->hist_sums,
                                   (size_t)k * c->B * 8, cudaMemcpyDeviceToHost, b->stream));
            any = true;
        }
        if (any) BCK(b, cudaStreamSynchronize(b->stream));
        done += k;
    }
    BCK(b, cudaStreamSynchronize(b->stream));
    return MLEM_OK;
}

int mlem_batch_profile(mlem_batch* b, int n, double* ms, double* bytes, int* launches) {
    if (!b || n <= 0) return bfail(b, MLEM_ERR_INVALID, "bad argument");
    BCK(b, cudaSetDevice(b->device));
    TRY(batch_refresh(b, 1));
    std::vector<PhaseEvents> evs((size_t)n);
    for (auto& pe : evs)
        for (auto& e : pe.ev) BCK(b, cudaEventCreate(&e));
    int s = MLEM_OK;
    for (int i = 0; i < n && s == MLEM_OK; ++i) {
        s = batch_reset_slots(b);
        if (s == MLEM_OK) s = batch_enqueue(b, true, &evs[(size_t)i]);
    }
    if (s == MLEM_OK && cudaStreamSynchronize(b->stream) != cudaSuccess)
        s = bfail(b, MLEM_ERR_CUDA, "synchronize");
    double acc[MLEM_N_PHASES] = {0, 0, 0, 0};
    for (auto& pe : evs)
        for (int p = 0; p < MLEM_N_PHASES && s == MLEM_OK; ++p) {
            float t = 0.0f;
            if (cudaEventElapsedTime(&t, pe.ev[p], pe.ev[p + 1]) != cudaSuccess)
                s = bfail(b, MLEM_ERR_CUDA, "event timing");
            acc[p] += t;
        }
    for (auto& pe : evs)
        for (auto& e : pe.ev) cudaEventDestroy(e);
    if (s != MLEM_OK) return s;
    double tb[MLEM_N_PHASES] = {0, 0, 0, 0};
    int tl[MLEM_N_PHASES] = {0, 0, 0, 0};
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        double pb[MLEM_N_PHASES];
        int pl[MLEM_N_PHASES];
        phase_bytes_for(b->ctx[i], MLEM_BK_FUSED, eff_tile(b, i), pb, pl, uses_active(b, i));
        for (int p = 0; p < MLEM_N_PHASES; ++p) {
            tb[p] += pb[p];
            tl[p] += pl[p];
        }
    }
    tl[MLEM_PHASE_PROJECT] = (int)b->groups.size();  // one kernel per (frame tile, row visit) group
    for (const mlem_ctx* c : b->ctx)
        if (c->n_long) tl[MLEM_PHASE_PROJECT] += 2;  // the long-row kernels
    for (int p = 0; p < MLEM_N_PHASES; ++p) {
        if (ms) ms[p] = acc[p] / n;
        if (bytes) bytes[p] = tb[p];
        if (launches) launches[p] = tl[p];
    }
    return MLEM_OK;
}

}  // extern "C"
