// ctx.hpp -- the device context behind the C ABI (internal), shared by
// capi.cu (contexts, iteration, tuning, subsets, device-pointer entry points)
// and capi_batch.cu (multi-matrix batches).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "kernels.h"
#include "mlem_b200.h"

struct mlem_ctx {
    int device = 0;
    int n_sm = 148;
    uint32_t R = 0, C = 0;
    uint64_t Z = 0;
    uint32_t flags = 0;
    cudaStream_t stream = nullptr;      // where work is enqueued
    cudaStream_t own_stream = nullptr;  // created with the context
    uint64_t device_bytes = 0;

    // matrix
    uint64_t* row_ptr = nullptr;
    uint2* elems = nullptr;
    uint64_t* col_ptr = nullptr;
    uint2* celems = nullptr;
    bool has_csc = false;
    // The CSC in visiting order (ensure_csc_vis; built when MLEM_BK_CSC runs
    // with a sorted visit): each column lists the visiting positions of its
    // rays (positions in row_order) ascending, with the same col_ptr.  The
    // forward pass then writes the correlations by visiting position, so a
    // column's gathers fall on neighbouring, nearly coincident rays.
    uint2* celems_vis = nullptr;
    uint32_t* row_pos = nullptr;  // visiting position of every row
    // celems_vis cut to the rays with counts (csc_active_build), refilled by
    // mlem_set_sinograms: each column's kept entries at its offset,
    // csc_act_len[col] of them; pos_keep: one bit per visiting position.  The
    // CSC method's back projection walks it while csc_act_ready (the
    // one-iteration host steps clear that); made only where it fits.
    uint2* csc_act = nullptr;
    uint32_t* csc_act_len = nullptr;
    uint32_t* pos_keep = nullptr;
    bool csc_act_ready = false;
    uint32_t max_col_len = 0, max_row_len = 0;
    float* norm = nullptr;       // column sums, device voxel order
    float* norm_nat = nullptr;   // column sums, natural voxel order
    std::vector<float> norm_host;  // natural order
    double sumnorm = 0.0;

    // Voxel order on the device.  With a known grid the columns are
    // relabelled along a Morton curve (see brick_order); perm maps a natural
    // voxel index to its device index.
    bool bricked = false;
    uint32_t grid[3] = {0, 0, 0};
    uint32_t* perm = nullptr;
    std::vector<uint32_t> perm_host, iperm_host;
    float* pscratch[2] = {nullptr, nullptr};
    size_t pscratch_floats = 0;

    // Visiting order of the row kernels (row_order_build): rays with nearby
    // entry and exit voxels next to each other.  Null with MLEM_FLAG_NO_ROW_ORDER.
    uint32_t* row_order = nullptr;
    ulonglong2* row_ranges = nullptr;  // element range of each visited row (row_ranges_build)
    // The sorted visiting list without the rows whose counts are zero in every
    // frame, rebuilt on the device whenever the sinograms change
    // (active_rows_build); the one-pass iteration walks it.  act_rows and
    // act_nnz are read back by mlem_set_sinograms.
    uint32_t* act_order = nullptr;
    ulonglong2* act_ranges = nullptr;
    uint8_t* act_tmp = nullptr;
    size_t act_tmp_bytes = 0;
    uint32_t* act_n = nullptr;
    unsigned long long* act_z = nullptr;
    bool act_ready = false;
    uint32_t act_rows = 0;
    uint64_t act_nnz = 0;
    // pinned host copy of act_n / act_z, read after mlem_step_host's final
    // synchronisation (that call does not wait for the list on its own)
    unsigned long long* act_host = nullptr;
    uint64_t sino_gen = 0;  // counts sinogram uploads (a batch rebuilds its items on change)
    unsigned int* counter = nullptr;  // work counter of the dynamically scheduled kernels

    // Rows longer than kLongRowElems, cut into segments (k_long.cu) for the
    // one-pass method; f_long holds their forward sums (n_long x Bp).
    mlem::LongSeg* long_segs = nullptr;
    uint32_t n_long_segs = 0, n_long = 0;
    float* f_long = nullptr;
    float* f_long_d = nullptr;  // the same for mlem_fused_update_d (any frame count)
    size_t f_long_d_floats = 0;

    // Ordered subsets (mlem_set_subsets): row r in subset r % n_subsets.
    // sub_norm[s * C ...]: subset column sums (device voxel order); the visiting
    // lists hold every subset's rows back to back (subset s at sub_off[s]), in
    // file order and, with a row order, in the sorted order, with their ranges.
    uint32_t n_subsets = 1;
    float* sub_norm = nullptr;
    uint32_t* sub_file = nullptr;
    ulonglong2* sub_file_ranges = nullptr;
    uint32_t* sub_sorted = nullptr;
    ulonglong2* sub_sorted_ranges = nullptr;
    std::vector<uint64_t> sub_off;
    size_t sub_bytes = 0;  // device bytes of the subset buffers
    // every subset's sorted list without its rows whose counts are zero in
    // every frame (built like act_order whenever the sinograms or the subsets
    // change; subset s at sub_off[s], its length in sub_act_n[s])
    uint32_t* sub_act_order = nullptr;
    ulonglong2* sub_act_ranges = nullptr;
    uint32_t* sub_act_n = nullptr;
    unsigned long long* sub_act_z = nullptr;
    bool sub_act_ready = false;

    // frames
    uint32_t B = 0, Bp = 0;
    std::vector<double> sumin;
    int32_t* sino = nullptr;
    float* x = nullptr;
    float* correl = nullptr;
    float* update = nullptr;
    void* stage = nullptr;  // staging for frame-major <-> interleaved copies
    size_t stage_bytes = 0;
    // mlem_stream_host: an upload and a download stream, double-buffered
    // staging of the sinograms and images, and the events between the streams
    cudaStream_t up_stream = nullptr, down_stream = nullptr;
    // The second set of per-sinogram buffers of the overlapped streaming steps
    // (mlem_stream_host with the list of rows with counts): sinogram and list,
    // and the one-iteration graph captured over them.  The two sets trade
    // places when a call ends on this one.
    int32_t* sino_alt = nullptr;
    uint32_t* act_order_alt = nullptr;
    ulonglong2* act_ranges_alt = nullptr;
    uint32_t* act_n_alt = nullptr;
    unsigned long long* act_z_alt = nullptr;
    cudaGraphExec_t graph_alt = nullptr;
    int32_t* sstage[2] = {nullptr, nullptr};
    float* istage[2] = {nullptr, nullptr};
    size_t sstage_n = 0, istage_n = 0;  // elements of each buffer
    cudaEvent_t ev_up[2] = {nullptr, nullptr}, ev_sfree[2] = {nullptr, nullptr};
    cudaEvent_t ev_img[2] = {nullptr, nullptr}, ev_dfree[2] = {nullptr, nullptr};
    bool images_ready = false;

    // statistics history
    void* stats_scratch = nullptr;
    unsigned int* stats_slot = nullptr;
    double* hist_sums = nullptr;
    unsigned long long* hist_zeros = nullptr;
    unsigned long long* hist_subn = nullptr;
    int hist_cap = 0;

    // scratch for the host-buffer reference functions
    float* tmp_r[2] = {nullptr, nullptr};
    float* tmp_c[3] = {nullptr, nullptr, nullptr};
    int32_t* tmp_sino = nullptr;
    double* tmp_d = nullptr;
    float* inits_dev = nullptr;

    // Mirrors applied in the kernels (MLEM_FLAG_MIRROR_KERNELS): the matrix
    // arrays hold the stored elements only; norm holds the full matrix's
    // column sums; f_mirror_d is the per-row sum buffer of mlem_fused_update_d.
    bool mirrored = false;
    mlem::MirrorView mirror;
    uint32_t* mirror_lut = nullptr;
    uint32_t* mirror_vox = nullptr;
    float* f_mirror_d = nullptr;
    size_t f_mirror_d_floats = 0;

    // region-blocked copy of the matrix (MLEM_BK_REGION), for one frame tile
    mlem::RegionBlocks rb;
    size_t rb_bytes = 0;

    mlem_tuning tuning{};
    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    bool graph_dirty = true;

    std::string err;
};

// Return the status of a call that failed.
#define TRY(call)                         \
    do {                                  \
        int s_ = (call);                  \
        if (s_ != MLEM_OK) return s_;     \
    } while (0)

namespace mlem {

// Events recorded at the phase boundaries of one iteration (profiling only).
struct PhaseEvents {
    cudaEvent_t ev[MLEM_N_PHASES + 1];
};

// The context's CSR as the row kernels see it (row order and ranges included).
SparseView csr_view(const mlem_ctx* c);
void dev_free(void* p);
// Algorithmic bytes and kernel launches of one iteration, per phase.
// active_rows: the context's one-pass sorted walk, which visits only the
// rows with counts (the batch kernels visit every row).
void phase_bytes_for(const mlem_ctx* c, int bk_mode, int frame_tile, double* bytes,
                     int* launches, bool active_rows = false);
// Room for the image statistics of n iterations.
int ensure_history(mlem_ctx* c, int n);

}  // namespace mlem
