// kernels.h -- host-side launchers of the sm_100a MLEM kernels.
//
// Device layouts (all in HBM, 256-byte aligned by cudaMalloc):
//   CSR  : ptr u64[R+1] (leading 0, then the CSR4 row END offsets),
//          elements {u32 column, f32 value} x Z, padded to an even count so
//          that they can be read as 16-byte pairs.
//   CSC  : ptr u64[C+1], elements {u32 row, f32 value} x Z (same padding),
//          rows ascending inside a column (stable transpose of CSR order).
//   frame-interleaved vectors for B frames: image x[C][B], sinogram s[R][B],
//   correlation c[R][B], update u[C][B]; norm[C] is shared by all frames.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace mlem {

struct SparseView {
    const uint64_t* ptr;  // n+1 offsets
    const uint4* pairs;   // elements as 16-byte pairs
    uint32_t n;           // rows (CSR) or columns (CSC)
    uint64_t nnz;
    // Row kernels visit rows in this order when non-null: the k-th row a
    // grid-stride walk reaches is order[k] (a permutation of [0, n)).  Only
    // the visiting order changes; every vector stays indexed by row.
    const uint32_t* order = nullptr;
    // With `order`: vrange[k] = {ptr[order[k]], ptr[order[k] + 1]}, the
    // element range of the k-th visited row in one load (no order -> ptr chain).
    const ulonglong2* vrange = nullptr;
    // The one-pass row walks treat a row with more elements as empty: it is
    // left to the long-row kernels (k_long.cu).  Every other kernel ignores it.
    uint64_t long_len = ~0ull;
    // When non-null, the one-pass walks (k_fused_row, k_fused_chunked,
    // k_fused_staged) visit *n_dev positions of order/vrange instead of n: a
    // visiting list built on the device (active_rows_build), n its capacity.
    const uint32_t* n_dev = nullptr;
    // k_fwproj only: write the row's outputs (correlation, projection) at its
    // visiting position instead of its row index -- the layout the CSC in
    // visiting order (mlem_ctx::celems_vis) gathers from.
    bool out_by_visit = false;
    // k_fwproj only, with out_by_visit and a device-built list (n_dev): the
    // position of row r in the full visiting order is out_pos[r].
    const uint32_t* out_pos = nullptr;
    // CSC kernels (k_bkproj_csc, k_bkproj_csc_pipe) only, when non-null:
    // column col holds len[col] entries from ptr[col] (the rest of its span
    // is unused), the layout csc_active_build writes.
    const uint32_t* len = nullptr;
};

// Entry range of column (or row) i: [ptr[i], ptr[i + 1]), or len[i] entries from ptr[i].
__device__ __forceinline__ void span_of(const SparseView& s, uint64_t i, uint64_t& b, uint64_t& e) {
    b = s.ptr[i];
    e = s.len ? b + s.len[i] : s.ptr[i + 1];
}

// Row index of visiting position v.
__host__ __device__ inline uint64_t row_at(const SparseView& s, uint64_t v) {
    return s.order ? (uint64_t)s.order[v] : v;
}

// Per-matrix launch configuration (chosen by the autotuner).
struct LaunchCfg {
    int group = 32;       // lanes cooperating on one row / column: 4, 8, 16 or 32
    int frame_tile = 1;   // frames per pass over the matrix: 1, 2, 4, 8 or 16
    int blocks_per_sm = 8;
    int sm_count = 148;
};

// Valid launch configuration (group 4..32, frame tile 1..16, 1..8 blocks/SM).
bool cfg_valid(const LaunchCfg& c);

// ---- forward projection -------------------------------------------------
// y[r][f] = sum_k v_k x[col_k][f] for frames f in [f0, f0+BT); when sino is
// non-null also c[r][f] = calcCorrel(sino, y).  y and/or c may be null.
cudaError_t fwproj(const SparseView& csr, const float* x, uint32_t B, uint32_t f0,
                   const int32_t* sino, float* c, float* y, const LaunchCfg& cfg,
                   cudaStream_t st);

// ---- back projection over the CSC copy ----------------------------------
// u[col][f] = sum_k v_k c[row_k][f]; with norm non-null, instead
// x[col][f] *= calcUpdate factor(u, norm[col]) (u not stored).
cudaError_t bkproj_csc(const SparseView& csc, const float* c, uint32_t B, uint32_t f0,
                       const float* norm, float* x, float* u, const LaunchCfg& cfg,
                       cudaStream_t st);

// ---- back projection by atomic scatter over the CSR ---------------------
// u[col][f] += v_k c[r][f] (u must be zeroed before the first call).
cudaError_t bkproj_scatter(const SparseView& csr, const float* c, uint32_t B, uint32_t f0,
                           float* u, const LaunchCfg& cfg, cudaStream_t st);

// ---- one pass per row: forward projection, correlation, scatter ---------
cudaError_t fused_row(const SparseView& csr, const float* x, uint32_t B, uint32_t f0,
                      const int32_t* sino, float* u, const LaunchCfg& cfg, cudaStream_t st);

// ---- symmetry-compressed matrices (k_sym.cu) -----------------------------
// The stored CSR (ptr R+1 with a leading 0, elements) and the mirror tables:
// lut[m * n_crystals + d] = detector d mirrored by m (bit 0 x, 1 y, 2 z).
struct SymExpand {
    const uint64_t* ptr;
    const uint2* el;
    uint32_t R;
    const uint32_t* lut;
    uint32_t n_crystals;
    uint32_t grid[3];
};
// Host: the 8 x n_crystals mirror tables (symhandler.cpp:33-114).
void sym_detector_luts(uint32_t n_layers, uint32_t n_blocks, uint32_t block_size,
                       uint32_t n_rings, std::vector<uint32_t>& lut);
// Host: the mirrors a header's flags allow, in generateSyms order.
std::vector<uint32_t> sym_mirrors(uint32_t sym);
// counts[full row] += stored row length, for mirror m (0: the stored rows).
cudaError_t sym_count(const SymExpand& s, uint32_t mirror, unsigned long long* counts,
                      cudaStream_t st);
// Copy mirror m's elements to the full rows' cursors, then advance them.
cudaError_t sym_fill(const SymExpand& s, uint32_t mirror, unsigned long long* cursor, uint2* out,
                     cudaStream_t st);

// ---- mirrors applied in the kernels (k_mirror.cu) --------------------------
// A symmetry-compressed matrix kept as stored; mirror j (0 = the identity,
// then the header's mirrors in generateSyms order) maps stored row r to full
// row lor(r, j) through lut[j * n_crystals + detector], and device voxel v to
// vox[j * C + v], or to v ^ xor_mask[j] when vox is null (power-of-two grid
// in Morton order).
struct MirrorView {
    const uint32_t* lut = nullptr;
    const uint32_t* vox = nullptr;
    uint32_t xor_mask[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t n_crystals = 0;
    uint32_t C = 0;
    uint32_t n = 1;  // mirrors including the identity, 1..8
};
// f[lor(r, j)][f0 .. f0+frame_tile) += the stored row's partial sums under
// every mirror (f zeroed by the caller; float atomics).
cudaError_t mirror_fwproj(const SparseView& csr, const MirrorView& mv, const float* x, uint32_t B,
                          uint32_t f0, int frame_tile, float* f, int sm_count, int blocks_per_sm,
                          cudaStream_t st);
// u[vox(v, j)][...] += value * c for every stored element and mirror, with
// c = calcCorrel(sino[t], y[t]) when sino is non-null, else y[t] (u zeroed
// by the caller).
cudaError_t mirror_bkproj(const SparseView& csr, const MirrorView& mv, const float* y,
                          const int32_t* sino, uint32_t B, uint32_t f0, int frame_tile, float* u,
                          int sm_count, int blocks_per_sm, cudaStream_t st);
// Full column sums from the stored matrix's: sum over j of norm[vox(w, j)].
cudaError_t mirror_norm(const float* norm_stored, const MirrorView& mv, float* norm_full,
                        cudaStream_t st);

// ---- rows too long for one warp (k_long.cu) ------------------------------
// Rows longer than kLongRowElems are cut into segments of at most
// kLongSegElems elements: elements [b, e) of row `row`, the slot-th long row.
constexpr uint64_t kLongRowElems = 4096;
constexpr uint64_t kLongSegElems = 4096;
struct LongSeg {
    uint64_t b, e;
    uint32_t slot, row;
};
// u += the one-pass contribution of the long rows: f_long (n_long x B floats)
// is zeroed, the segments' partial sums are added into it, then every
// segment scatters value x calcCorrel(count, f) into u (all B frames, in
// passes of frame_tile).
cudaError_t long_rows_pass(const SparseView& csr, const LongSeg* segs, uint32_t n_seg,
                           uint32_t n_long, const float* x, uint32_t B, int frame_tile,
                           const int32_t* sino, float* f_long, float* u, int sm_count,
                           cudaStream_t st);

// x[i] *= factor(u[i], norm[i/B]); u[i] = 0 when zero_u.
cudaError_t apply_update(float* x, float* u, const float* norm, uint32_t C, uint32_t B,
                         bool zero_u, cudaStream_t st);

// ---- ordered subsets (row r in subset r % S) -------------------------------
// x *= norm_s != 0 ? u / norm_s : (norm != 0 ? 1 : u); u = 0.
cudaError_t apply_update_subset(float* x, float* u, const float* norm_s, const float* norm,
                                uint32_t C, uint32_t B, cudaStream_t st);
// Column sums of subset s over the CSC, in ascending row order (bit-exact
// with calcColumnSums over the subset's rows).
cudaError_t subset_column_sums_exact(const SparseView& csc, uint32_t S, uint32_t s, float* norm,
                                     cudaStream_t st);
// All S subsets' column sums by atomics over the CSR: norm[s * C + col].
cudaError_t subset_column_sums_atomic(const SparseView& csr, uint32_t S, uint32_t C, float* norm,
                                      cudaStream_t st);

// ---- bit-exact kernels: the float operation order of seqcsr4mlem --------
cudaError_t fwproj_exact(const SparseView& csr, const float* x, uint32_t B, const int32_t* sino,
                         float* c, float* y, cudaStream_t st);
cudaError_t bkproj_exact(const SparseView& csc, const float* c, uint32_t B, const float* norm,
                         float* x, float* u, cudaStream_t st);
cudaError_t column_sums_exact(const SparseView& csc, float* norm, cudaStream_t st);
cudaError_t column_sums_atomic(const SparseView& csr, uint32_t C, float* norm, cudaStream_t st);

// ---- per-frame image statistics (sum in double, zeros, subnormals) -----
// Deterministic: fixed-order block tree.  `partial` needs stats_scratch_bytes.
// B is the interleave stride; the first n_out frames are written.  When
// `slot` is non-null, results go to row *slot of [n][n_out] outputs and the
// kernel then increments *slot (so one captured graph serves every
// iteration).
size_t stats_scratch_bytes(uint32_t B);
cudaError_t image_stats(const float* x, uint32_t C, uint32_t B, uint32_t n_out, void* partial,
                        unsigned int* slot, double* sums, unsigned long long* zeros,
                        unsigned long long* subnormals, cudaStream_t st);

// ---- layout helpers -------------------------------------------------------
// out[p(i)*Bp + b] = in[b*n + i] for b < B (n items per frame; pad frames
// untouched), and back: out[b*n + i] = in[p(i)*Bp + b], where p = perm
// (natural -> device order) or the identity when perm is null.
cudaError_t interleave_i32(const int32_t* in, int32_t* out, uint64_t n, uint32_t B, uint32_t Bp,
                           cudaStream_t st);
cudaError_t interleave_f32(const float* in, float* out, uint64_t n, uint32_t B, uint32_t Bp,
                           const uint32_t* perm, cudaStream_t st);
cudaError_t deinterleave_f32(const float* in, float* out, uint64_t n, uint32_t B, uint32_t Bp,
                             const uint32_t* perm, cudaStream_t st);
// Interleaved [n][B] vectors between natural and device voxel order:
// to_device: out[perm[i]*B + b] = in[i*B + b]; to_natural: out[i*B + b] = in[perm[i]*B + b].
cudaError_t permute_to_device(const float* in, float* out, const uint32_t* perm, uint64_t n,
                              uint32_t B, cudaStream_t st);
cudaError_t permute_to_natural(const float* in, float* out, const uint32_t* perm, uint64_t n,
                               uint32_t B, cudaStream_t st);
// Relabel the column (voxel) index of every element: e.x = perm[e.x].
cudaError_t remap_columns(uint2* elems, uint64_t nnz, const uint32_t* perm, cudaStream_t st);
// x[i][b] = b < B ? vals[b] : 0 for the Bp-interleaved image (vals: device, B floats).
cudaError_t fill_frames(float* x, uint64_t n, uint32_t Bp, uint32_t B, const float* vals,
                        cudaStream_t st);
// c[i] = calcCorrel(s[i], f[i]).
cudaError_t correl_elementwise(const float* f, const int32_t* s, float* c, uint64_t n,
                               cudaStream_t st);

// ---- prefix sums ----------------------------------------------------------
// out[0] = 0, out[i+1] = in[0] + ... + in[i]  (n+1 outputs).
size_t scan_scratch_bytes(uint64_t n);
// `scratch` must hold scan_scratch_bytes(n) bytes; scratch_bytes is checked
// (cudaErrorInvalidValue, nothing launched, when it is too small).
cudaError_t exclusive_scan_u64(const uint64_t* in, uint64_t* out, uint64_t n, void* scratch,
                               size_t scratch_bytes, cudaStream_t st);

// ---- deterministic CSR -> CSC transpose -----------------------------------
// col_ptr: C+1 entries; celems: Z (+ padding) 8-byte elements.  scratch is
// transpose_scratch_bytes(C) bytes.  Result is identical to a stable
// counting-sort transpose (ascending row, then in-row position).
size_t transpose_scratch_bytes(uint32_t C);
// CSR -> CSC.  Each column lists its rows ascending.  With row_key (and its
// inverse key_row), row r is stored as row_key[r] and the columns list those
// keys ascending: with the visiting positions of the row order as keys, a
// column lists its rays in visiting order.
cudaError_t transpose(const SparseView& csr, uint32_t C, uint64_t* col_ptr, uint2* celems,
                      void* scratch, uint32_t* max_col_len, cudaStream_t st,
                      const uint32_t* row_key = nullptr, const uint32_t* key_row = nullptr);
// pos[order[v]] = v for a permutation order of [0, n).
cudaError_t invert_permutation(const uint32_t* order, uint32_t* pos, uint64_t n, cudaStream_t st);

// ---- row visiting order (k_order.cu) -------------------------------------------
// order[k]: rows sorted by a key that interleaves the bits of the device
// column indices of each row's first and last element (a ray's entry and
// exit voxels for a geometric matrix, which the device voxel order makes
// spatially coherent), so rows visited together share image lines in L1.
// `order` holds csr.n entries; temporary memory is allocated and freed here.
cudaError_t row_order_build(const SparseView& csr, uint32_t C, uint32_t* order, cudaStream_t st);
// vrange[k] = {ptr[order[k]], ptr[order[k] + 1]} for k < csr.n.
cudaError_t row_ranges_build(const SparseView& csr, const uint32_t* order, ulonglong2* vrange,
                             cudaStream_t st);
// The sorted visiting list (csr.order, csr.vrange, csr.n < 2^31) without the
// rows whose counts are zero in all Bp frames of sino ([R][Bp]): their
// calcCorrel is 0 in every frame, so they add nothing to the update and their
// forward sums are never used.  Writes act_order / act_ranges (csr.n
// capacity), *act_n = rows kept, *act_z = their elements; tmp:
// active_rows_tmp_bytes(csr.n) bytes.  The list keeps the visiting order.
size_t active_rows_tmp_bytes(uint32_t n);
cudaError_t active_rows_build(const SparseView& csr, const int32_t* sino, uint32_t Bp,
                              void* tmp, size_t tmp_bytes, uint32_t* act_order,
                              ulonglong2* act_ranges, uint32_t* act_n, unsigned long long* act_z,
                              cudaStream_t st);

// The CSC in visiting order (csc_vis: ptr[C+1], entries {visiting position,
// value}) cut to the entries whose rays have a count in some frame: bit k & 31
// of keep[k >> 5] ((csr.n + 31) / 32 words) flags visiting position k
// (csr.order, as active_rows_build decides), dst (csc_vis.nnz capacity, same
// offsets) gets each column's kept
// entries in their order from ptr[col], len[col] their number.  The other
// entries meet calcCorrel 0 in every frame and add +0 to the column's sum.
cudaError_t csc_active_build(const SparseView& csr, const int32_t* sino, uint32_t Bp,
                             const SparseView& csc_vis, uint32_t* keep, uint2* dst, uint32_t* len,
                             cudaStream_t st);

// ---- matrix validation: every column < C and offsets non-decreasing ------
cudaError_t validate_csr(const SparseView& csr, uint32_t C, unsigned int* bad_flag,
                         cudaStream_t st);

// ---- synthetic Siddon generator on the device -----------------------------
struct SiddonSpec {
    uint32_t nx, ny, nz, n_rows, min_count, max_count;
    double radius_scale, min_len;
    uint64_t seed;
};
cudaError_t siddon_counts(const SiddonSpec& s, uint64_t* counts, cudaStream_t st);
// The device voxel order of a grid (capi.cu): perm[natural index] = device
// index, the Morton code of (ix, iy, iz) with x lowest (ranked when a
// dimension is not a power of two).
void voxel_permutation(uint32_t nx, uint32_t ny, uint32_t nz, std::vector<uint32_t>& perm);
cudaError_t siddon_fill(const SiddonSpec& s, const uint64_t* row_ptr, uint2* elems,
                        cudaStream_t st);
// out[r] = sequential double sum of v_k * x[col_k] (bit-identical to the host).
cudaError_t project_f64(const SparseView& csr, const float* x, double* out, cudaStream_t st);

// ---- region-blocked method (k_region.cu) -----------------------------------
// Rows cut into segments, one per region (aligned block of RS = 2^rlog device
// voxels), segments ordered by region.  Two region-major copies of the
// elements, {word, value} with word = (segment index inside the region <<
// rlog) | voxel index inside the region:
//   el_fw: segment-major (the rows' element order inside each segment);
//   el_bk: per block of SB = 2^sblog consecutive segments of a region,
//          voxel-major.
// Both are stored per block in span tiles: gpw spans of 16 consecutive
// elements, element k of every span of a tile side by side (one coalesced
// warp load per step); blocks are padded to whole tiles with value-0 copies.
// seg_row[s]: row of segment s (region order).
struct RegionView {
    const uint32_t* reg_order;    // nreg regions, most elements first
    const uint64_t* reg_seg_ptr;  // nreg+1 segment ranges
    const uint64_t* reg_el_ptr;   // nreg+1 element ranges
    const uint32_t* reg_blk_ptr;  // nreg+1 block ranges
    const uint64_t* blk_el_ptr;   // nblk+1 element ranges of the segment-major copy
    const uint64_t* bk_el_ptr;    // nblk+1 element ranges of the voxel-major copy
    const uint32_t* seg_row;
    const uint2* el_fw;
    const uint2* el_bk;
    uint32_t nreg;
    int rlog, sblog;
};

struct RegionBlocks {
    uint32_t* reg_order = nullptr;
    uint64_t* reg_seg_ptr = nullptr;
    uint64_t* reg_el_ptr = nullptr;
    uint32_t* reg_blk_ptr = nullptr;
    uint64_t* blk_el_ptr = nullptr;
    uint64_t* bk_el_ptr = nullptr;
    uint32_t* seg_row = nullptr;
    uint2* el_fw = nullptr;
    uint2* el_bk = nullptr;
    uint32_t nreg = 0, nblk = 0;
    uint64_t nseg = 0, nel = 0;  // nel: elements of the segment-major copy, padding included
    uint64_t nel_bk = 0;         // the same for the voxel-major copy (run-aligned spans)
    int rlog = 0, sblog = 0;
    uint32_t gpw = 0;            // lane groups per warp the copies are interleaved for
    RegionView view() const {
        return RegionView{reg_order, reg_seg_ptr, reg_el_ptr, reg_blk_ptr, blk_el_ptr, bk_el_ptr,
                          seg_row,   el_fw,       el_bk,      nreg,        rlog,       sblog};
    }
};

// Shared memory of one image / update tile (RS x BT floats) at most.
constexpr size_t kRegionTileBytes = 65536;
// Region size (log2 voxels), segment block size (log2) and lane groups per
// warp for a frame tile and C voxels.
void region_params(int frame_tile, uint32_t C, int* rlog, int* sblog, uint32_t* gpw);
// failed_line (nullable) receives the k_region.cu line of a failing step.
cudaError_t region_build(const SparseView& csr, uint32_t C, int rlog, int sblog, uint32_t gpw,
                         RegionBlocks* out, size_t* bytes, int* failed_line, cudaStream_t st);
void region_free(RegionBlocks* rb);
// fw[row][f] += segment partial projections (fw zeroed by the caller).
cudaError_t region_fwproj(const RegionBlocks& rb, const float* x, uint32_t B, uint32_t f0,
                          uint32_t C, float* fw, const LaunchCfg& cfg, cudaStream_t st);
// x[col][f] *= calcUpdate factor((A^T c)[col][f], norm[col]) for the frames of the tile.
cudaError_t region_bkproj_update(const RegionBlocks& rb, const float* c, uint32_t B, uint32_t f0,
                                 uint32_t C, const float* norm, float* x, const LaunchCfg& cfg,
                                 cudaStream_t st);
// f[i] = calcCorrel(s[i], f[i]).
cudaError_t correl_inplace(float* f, const int32_t* s, uint64_t n, cudaStream_t st);

// ---- multi-matrix batches (k_batch.cu) ---------------------------------------
// One matrix of a batch: its CSR and interleaved images / sinograms / update
// vector (stride Bp).
struct BatchMat {
    SparseView csr;
    const float* x;
    const int32_t* sino;
    float* u;
    uint32_t Bp;
    uint32_t pad;
};
// Rows [row0, row1) of matrix `mat` (pad: 0).
struct BatchItem {
    uint32_t mat;
    uint32_t row0, row1;
    uint32_t pad;
};
// The matrices of a batch, passed by value as the kernels' parameter (it
// lives in the constant bank, like a single-matrix kernel's arguments, and
// takes no registers): matrix i owns virtual rows [row_base[i], row_base[i+1]).
constexpr uint32_t kBatchTableMax = 64;
struct BatchTable {
    BatchMat mats[kBatchTableMax];
    uint64_t row_base[kBatchTableMax + 1];
    uint32_t n;
};
static_assert(sizeof(BatchTable) <= 32764, "kernel parameter space (CUDA >= 12.1)");

// Items schedule: every item does u[mat] += A^T correl(A x) over its rows,
// all frames of its matrix in passes of frame_tile (1, 2, 4, 8 or 16;
// divides every Bp).  `counter` (one uint) is reset on the stream first.
// sorted: every matrix of the table is visited in its sorted order (their
// views carry order and vrange); else every one in file order.
cudaError_t batch_fused(const BatchTable& t, const BatchItem* items, uint32_t n_items,
                        unsigned int* counter, int frame_tile, bool sorted, int sm_count,
                        int blocks_per_sm, cudaStream_t st);
// The items schedule with the staged row walk (staged_dev.cuh): every matrix
// in its sorted order; at most 4 resident CTAs per SM.
cudaError_t batch_staged(const BatchTable& t, const BatchItem* items, uint32_t n_items,
                         unsigned int* counter, int frame_tile, int sm_count, int blocks_per_sm,
                         cudaStream_t st);
// One matrix in chunks (MLEM_VISIT_SORTED_CHUNKED): CTAs take chunks of
// chunk_rows consecutive visiting positions from `counter` (reset here on the
// stream), and do every frame tile of a chunk's rows back to back -- each CTA
// stays on neighbouring rows for many steps (L1 reuse of their voxels) while
// the grid as a whole moves through one window of the order.
// ctas_per_sm: 1, 2 or 4 resident CTAs of 1024, 512 or 256 threads (the
// CTAs of one SM share its L1, a bigger CTA puts more neighbouring rows on it).
// ---- backward-pass one-pass kernels (k_adjoint.cu), one frame ----------------
// kOpRatio  : u += A^T calcCorrel(s, A x); rows[r] = (A x)_r (0 for a row
//             without a count, which is skipped)
// kOpAdjoint: u += A^T df, df_r = -(A x)_r (s_r / rows_r) / rows_r where s_r
//             and rows_r are nonzero, else 0 (x is the adjoint image here)
constexpr int kOpRatio = 0, kOpAdjoint = 1;
cudaError_t adjoint_pass(int op, const SparseView& csr, const float* x, const int32_t* sino,
                         float* rows, float* u, unsigned int* counter, int sm_count,
                         cudaStream_t st);

cudaError_t fused_chunked(const SparseView& csr, const float* x, uint32_t B, int frame_tile,
                          const int32_t* sino, float* u, uint32_t chunk_rows, int ctas_per_sm,
                          unsigned int* counter, int sm_count, cudaStream_t st);
// The same chunked walk with each warp's rows pipelined: the next row's
// elements staged in shared memory by cp.async, ranges and counts loaded
// ahead (k_staged.cu).  ctas_per_sm: 1..4 CTAs of 256 threads.
cudaError_t fused_staged(const SparseView& csr, const float* x, uint32_t B, int frame_tile,
                         const int32_t* sino, float* u, uint32_t chunk_rows, int ctas_per_sm,
                         unsigned int* counter, int sm_count, cudaStream_t st);
// Interleaved schedule: the same work in grid-stride order over the virtual
// row space.
cudaError_t batch_interleaved(const BatchTable& t, int frame_tile, bool sorted, int sm_count,
                              int blocks_per_sm, cudaStream_t st);

}  // namespace mlem
