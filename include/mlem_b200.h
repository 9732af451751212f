/*
 * mlem_b200.h -- C ABI of the B200-native MLEM reconstructor.
 *
 * Drop-in boundary for the hot path of the reference tools seqcsr4mlem /
 * openmpcsr4mlem (gupta-apoorva/mlem):
 *   calcColumnSums once, then per iteration calcFwProj -> calcCorrel ->
 *   calcBkProj -> calcUpdate (mlem_seq/seqcsr4mlem.cpp:37-189),
 * over the CSR4 system matrix of helper_files_common/csr4matrix.cpp:32-157.
 *
 * Conventions
 *   - Every function returns an int status (MLEM_OK == 0); no C++ exception
 *     crosses the ABI.  Where the reference throws std::runtime_error
 *     (csr4matrix.cpp:41-136, vector.hpp:35-44) or asserts on a size
 *     mismatch (seqcsr4mlem.cpp:39,73,96,110,125) these functions return
 *     MLEM_ERR_FORMAT / MLEM_ERR_IO / MLEM_ERR_INVALID and record a message,
 *     readable with mlem_last_error(ctx) (or mlem_global_error() when no
 *     context exists yet).
 *   - A context owns one matrix on one GPU: the CSR copy, the CSC copy built
 *     once on the device, the column sums, and the state of B frames
 *     (sinograms and images).  A context is not thread-safe.
 *   - Host pointers are caller-owned and only read (or written) during the
 *     call.  Host frame arrays are frame-major: sinograms [B][R], images
 *     [B][C].
 *   - The *_d functions take caller-owned DEVICE pointers and a cudaStream_t
 *     (passed as void*) and only enqueue work; their frame layout is
 *     interleaved: x[C][B], y[R][B].
 *   - Element layout (CSR4 and the device copies): 8 bytes {uint32 index,
 *     float32 value}, little-endian (helper_files_common/matrixelement.hpp
 *     :37-46).  Row offsets: the R uint64 row END offsets of the file
 *     (no leading zero).
 */
#ifndef MLEM_B200_H
#define MLEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MLEM_B200_VERSION 1

/* ---- status codes ----------------------------------------------------- */
#define MLEM_OK 0
#define MLEM_ERR_INVALID 1   /* bad argument or size mismatch */
#define MLEM_ERR_CUDA 2      /* CUDA runtime error (message has the name) */
#define MLEM_ERR_IO 3        /* cannot open / read / write a file */
#define MLEM_ERR_FORMAT 4    /* not a valid CSR4 file or vector file */
#define MLEM_ERR_NOMEM 5     /* device or host allocation failed */
#define MLEM_ERR_STATE 6     /* call out of order (e.g. iterate before sinograms) */
#define MLEM_ERR_MATRIX 7    /* matrix content invalid (column >= C, offsets decreasing) */
#define MLEM_NO_CHECKPOINT 8 /* mlem_checkpoint_read: no complete checkpoint present */

/* ---- context flags ------------------------------------------------------ */
#define MLEM_FLAG_EXACT 0x1u    /* bit-exact kernels: the float operation order of seqcsr4mlem */
#define MLEM_FLAG_NO_CSC 0x2u   /* do not build the CSC copy (atomic back projection only) */
#define MLEM_FLAG_CHECKED 0x4u  /* accepted for compatibility: offsets and column indices are always validated */
#define MLEM_FLAG_NATURAL_LAYOUT 0x8u /* keep the natural voxel order on the device (no Morton layout) */
#define MLEM_FLAG_NO_ROW_ORDER 0x10u  /* visit rows in file order (no entry/exit-voxel sort of the rows) */
#define MLEM_FLAG_EXPAND_SYMMETRY 0x20u /* mlem_create_from_file: regenerate the elements a
                                           symmetry-compressed file omits (mlem_create_symmetric);
                                           without it the symmetry flags are ignored, as the
                                           reference's MLEM ignores them */
#define MLEM_FLAG_MIRROR_KERNELS 0x40u /* with mlem_create_symmetric or a symmetry-compressed
                                          file: keep only the stored elements on the device and
                                          apply the mirrors inside the projection kernels
                                          (MLEM_BK_MIRRORED): the full matrix's results with
                                          about 1/|mirrors| of its device memory.  mlem_info.nnz,
                                          mlem_get_csr and mlem_get_csc give the stored elements;
                                          the column sums are the full matrix's.  Not with
                                          MLEM_FLAG_EXACT, ordered subsets, batches,
                                          mlem_bkproj_update_d or mlem_project_f64 (they
                                          return MLEM_ERR_INVALID / MLEM_ERR_STATE) */

/* ---- back-projection strategies ---------------------------------------- */
#define MLEM_BK_AUTO 0    /* the autotuner's choice (CSC when not tuned) */
#define MLEM_BK_CSC 1     /* gather over the device CSC copy, fused with calcUpdate (deterministic) */
#define MLEM_BK_ATOMIC 2  /* atomic scatter over the CSR (reference GPU drivers' method) */
#define MLEM_BK_FUSED 3   /* one pass per row: fwproj, correl and atomic scatter together */
#define MLEM_BK_REGION 4  /* region-blocked copy: shared-memory image/update tiles per region */
#define MLEM_BK_MIRRORED 5 /* mirrors applied in the kernels: a forward pass into per-row sums,
                              then a scatter (contexts made with MLEM_FLAG_MIRROR_KERNELS only) */

typedef struct mlem_ctx mlem_ctx;

typedef struct {
    uint32_t n_rows;      /* LORs */
    uint32_t n_cols;      /* voxels */
    uint64_t nnz;
    uint32_t n_frames;    /* B of the current sinograms (0 before mlem_set_sinograms) */
    uint32_t flags;
    int device;
    int has_csc;
    uint32_t max_col_len;
    uint32_t max_row_len;
    uint64_t device_bytes; /* device memory held by the context */
    uint64_t nnz_with_counts;  /* elements of the rows with a nonzero count in some frame of the
                                  current sinograms (0 before mlem_set_sinograms) */
    uint32_t rows_with_counts; /* those rows: the rest have calcCorrel 0 in every frame and are
                                  not walked by the one-pass iteration with a sorted visit
                                  (0 without a row order, in the bit-exact mode and with
                                  MLEM_FLAG_MIRROR_KERNELS, which walk every row) */
} mlem_info;

/* Launch configuration chosen by the autotuner (or set by the caller).
 * MLEM_BK_REGION builds its region-blocked copy of the matrix (about the
 * size of the CSR) when it is first selected for a frame tile.  MLEM_BK_CSC
 * with MLEM_VISIT_SORTED builds, when first selected, a second CSC in which
 * each column lists its rays by their position in the sorted row order
 * (another Z x 8 bytes + R x 4): the forward pass stores the correlations
 * by that position and the back projection gathers neighbouring rays.  It
 * stays deterministic (each column summed in ascending position); with
 * MLEM_VISIT_FILE the CSC lists rows ascending, as calcBkProj adds them.
 * With sinograms set, that CSC is also copied cut to the rays with a count in
 * some frame (another Z x 8 bytes + C x 4 + R / 8, made only while 2 GiB of
 * the device stay free beside it), and the back projection walks those
 * entries only, leaving out terms that are +0.  mlem_set_sinograms refills
 * the copy, as does selecting the method; mlem_step_host and
 * mlem_stream_host, one iteration per sinogram, walk the whole CSC in
 * visiting order instead (the copy takes about as long as the back
 * projection saves in six iterations).  Either way the sums are a fixed
 * function of the matrix, the sinograms and the entry point, the same from
 * run to run. */
typedef struct {
    int bk_mode;        /* MLEM_BK_CSC, MLEM_BK_ATOMIC, MLEM_BK_FUSED or MLEM_BK_REGION */
    int group;          /* lanes per row/column: 4, 8, 16 or 32 */
    int frame_tile;     /* frames per pass over the matrix: 1, 2, 4, 8 or 16 */
    int blocks_per_sm;  /* 1..8 blocks of 256 threads per SM (chunked visit: 1, 2 or 4 CTAs
                           of 1024, 512 or 256 threads; staged visit: 1..4 CTAs of 256) */
    int visit;          /* row visiting order: MLEM_VISIT_FILE, _SORTED, _SORTED_CHUNKED or
                           _SORTED_STAGED */
    double ms_per_iter; /* measured by mlem_autotune; 0 when set by hand */
} mlem_tuning;

/* Row visiting orders (mlem_tuning.visit).  The sorted orders need the row
 * order built at creation (not MLEM_FLAG_NO_ROW_ORDER); results change only
 * by the order of the scatter atomics (MLEM_BK_CSC: of the column sums). */
#define MLEM_VISIT_FILE 0           /* file order, grid stride */
#define MLEM_VISIT_SORTED 1         /* rows sorted by entry/exit voxel, grid stride */
#define MLEM_VISIT_SORTED_CHUNKED 2 /* sorted; CTAs take chunks of neighbouring rows from a counter
                                       (one-pass method, group 32) */
#define MLEM_VISIT_SORTED_STAGED 3  /* as chunked, each warp's rows pipelined: elements staged in
                                       shared memory by asynchronous copies rows ahead (one-pass
                                       method, group 32) */

/* ---- errors ------------------------------------------------------------- */
const char* mlem_last_error(const mlem_ctx* ctx);
const char* mlem_global_error(void);
const char* mlem_status_string(int status);
int mlem_version(void);

/* ---- context lifecycle -------------------------------------------------- */
/* Replaces Csr4Matrix + mapRows (csr4matrix.cpp:32-224): uploads the CSR4
 * arrays (row_end = the file's R row END offsets) to `device`, builds the
 * CSC copy (unless MLEM_FLAG_NO_CSC) and computes the column sums. */
int mlem_create(mlem_ctx** out, const uint64_t* row_end, const void* elems, uint32_t n_rows,
                uint32_t n_cols, uint64_t nnz, uint32_t flags, int device);

/* Same, with the voxel grid (nx, ny, nz; nx*ny*nz == n_cols): the device
 * then stores the image along a Morton (Z-order) curve over the whole grid,
 * which keeps a ray's voxels in few cache lines (every 2x2x2 cube in one
 * 32-byte sector).  Only the device layout changes; every
 * host- and device-pointer interface keeps the natural voxel order
 * ix + nx*(iy + ny*iz) (helper_files_common/scannerconfig.cpp getVoxelNr)
 * and every result is unchanged.  grid == NULL: natural order. */
int mlem_create_grid(mlem_ctx** out, const uint64_t* row_end, const void* elems, uint32_t n_rows,
                     uint32_t n_cols, uint64_t nnz, const uint32_t grid[3], uint32_t flags,
                     int device);

/* Same, from a CSR4 file (the command-line driver's path; the grid comes
 * from the file's scanner block). */
int mlem_create_from_file(mlem_ctx** out, const char* csr4_path, uint32_t flags, int device);

/* Scanner symmetries of a symmetry-compressed CSR4 matrix (header flags @5:
 * x = 1, y = 2, z = 4, csr4matrix.cpp:62-65) and the geometry they act on:
 * rows are LORs d1 * n_crystals + d2 (n_rows = n_crystals^2, n_crystals =
 * block_size * n_blocks * n_layers * n_rings) and columns voxels
 * ix + nx * (iy + ny * iz) of the grid (n_cols = nx * ny * nz). */
typedef struct {
    uint32_t sym;
    uint32_t n_layers, n_blocks, block_size, n_rings;
    uint32_t grid[3];
} mlem_symmetry;
/* A context on the full matrix of a symmetry-compressed one: for every
 * symmetry the flags allow (all combinations of x, y and z mirrors but the
 * identity, x outermost, in the order of visualizematrix/symhandler.hpp:
 * generateSyms), every stored row r adds its elements, with mirrored voxels,
 * to row transformLor(r) (symhandler.hpp/.cpp: detector mirror tables).  In a
 * full row the stored elements come first, then each symmetry's in that
 * order, source rows ascending.  The expansion runs on the device; the stored
 * arrays are read only during the call.  With sym == 0 this is mlem_create_grid. */
int mlem_create_symmetric(mlem_ctx** out, const uint64_t* row_end, const void* elems,
                          uint32_t n_rows, uint32_t n_cols, uint64_t nnz,
                          const mlem_symmetry* sym, uint32_t flags, int device);

/* Synthetic Siddon matrix generated on the device (bit-identical to the host
 * generator of mlem_b200/gen); the reference relies on an external generator. */
int mlem_create_siddon(mlem_ctx** out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t n_rows,
                       uint32_t min_count, uint32_t max_count, double radius_scale,
                       double min_len, uint64_t seed, uint32_t flags, int device);

void mlem_destroy(mlem_ctx* ctx);
int mlem_get_info(const mlem_ctx* ctx, mlem_info* out);
/* Enqueue the context's work on `stream` (a cudaStream_t of the context's
 * device; NULL restores the context's own stream).  Lets a caller order the
 * reconstruction with its own work and time it with its own events. */
int mlem_set_stream(mlem_ctx* ctx, void* stream);
/* Number of kernels one iteration launches with the current tuning and
 * frame count (the iteration, plus the two image-statistics kernels). */
int mlem_kernels_per_iteration(const mlem_ctx* ctx, int* n);

/* Copy the device CSR back: row_end[R] (END offsets), elems[Z]. */
int mlem_get_csr(mlem_ctx* ctx, uint64_t* row_end, void* elems);
/* Copy the device CSC: col_ptr[C+1] (leading 0), elems[Z] {row, value}. */
int mlem_get_csc(mlem_ctx* ctx, uint64_t* col_ptr, void* elems);

/* ---- the reference's five functions, on host buffers ------------------ */
/* seqcsr4mlem.cpp:37-49 calcColumnSums -> norm[C] (bit-exact). */
int mlem_calc_column_sums(mlem_ctx* ctx, float* norm);
/* seqcsr4mlem.cpp:52-66 initImage: float(sum_double(sino) / sum_double(norm)). */
int mlem_init_value(mlem_ctx* ctx, const int32_t* sino, uint64_t sino_len, float* initial);
/* seqcsr4mlem.cpp:69-91 calcFwProj: fwproj[R] = A image[C]. */
int mlem_calc_fwproj(mlem_ctx* ctx, const float* image, float* fwproj);
/* seqcsr4mlem.cpp:94-105 calcCorrel: correl[R] = fwproj != 0 ? sino / fwproj : 0. */
int mlem_calc_correl(mlem_ctx* ctx, const float* fwproj, const int32_t* sino, uint64_t sino_len,
                     float* correl);
/* seqcsr4mlem.cpp:108-120 calcBkProj: update[C] = A^T correl[R]. */
int mlem_calc_bkproj(mlem_ctx* ctx, const float* correl, float* update);
/* seqcsr4mlem.cpp:123-134 calcUpdate: image *= norm != 0 ? update / norm : update. */
int mlem_calc_update(mlem_ctx* ctx, const float* update, const float* norm, float* image);

/* ---- device-resident reconstruction (seqcsr4mlem.cpp:137-189 mlem) ------ */
/* Upload B sinograms [B][R] (int32).  Each must have exactly R entries
 * (the reference asserts this in calcCorrel, seqcsr4mlem.cpp:96). */
int mlem_set_sinograms(mlem_ctx* ctx, const int32_t* sino, uint32_t n_frames);
/* initImage for every frame (seqcsr4mlem.cpp:52-66); `initial` (nullable)
 * receives the B initial values. */
int mlem_init_images(mlem_ctx* ctx, float* initial);
/* Set the B images [B][C] (restart from a checkpoint, mpicsr4mlem.cpp:536-553). */
int mlem_set_images(mlem_ctx* ctx, const float* images);
/* Run n iterations.  image_sums (nullable) receives [n][B] double image
 * sums after each iteration; zeros / subnormals (nullable) the per-iteration
 * zero and subnormal counts [n][B] that seqcsr4mlem prints (:172-185).
 * The iteration is replayed from a captured CUDA graph. */
int mlem_iterate(mlem_ctx* ctx, int n_iter, double* image_sums, uint64_t* zeros,
                 uint64_t* subnormals);
/* Download the B images [B][C]. */
int mlem_get_images(mlem_ctx* ctx, float* images);
/* One iteration end to end on host buffers: upload the B sinograms and the B
 * images, iterate once on the device, download the images. */
int mlem_step_host(mlem_ctx* ctx, const int32_t* sino, float* images_inout, uint32_t n_frames);
/* n iterations on host buffers, each with sinograms of its own: iteration k
 * uses sinos[k] ([B][R] int32, B = the context's frame count) and, when
 * images is non-null and images[k] non-null, writes the B images after it to
 * images[k] ([B][C] float32).  Iteration 0 starts from the context's images
 * (mlem_init_images, mlem_set_images or an earlier call), iteration k + 1
 * from iteration k's, which stay on the device.  The upload of sinos[k + 1]
 * runs on a copy stream of its own during iteration k and the download of
 * images[k] on another during iteration k + 1; with page-locked host buffers
 * (cudaHostAlloc, cudaHostRegister) they overlap the kernels.  Where the
 * iteration walks the list of rows with counts (a sorted row order, no
 * ordered subsets, not MLEM_FLAG_EXACT or MLEM_FLAG_MIRROR_KERNELS), the copy
 * stream also rebuilds that list for sinos[k + 1] during iteration k, in a
 * second set of sinogram and list buffers (R x Bp x 4 + R x 20 bytes, made on
 * first use) with a captured iteration of its own.  Every copy has ended when
 * the call returns.  Afterwards the context holds sinos[n - 1] as its
 * sinograms (the initImage sums of mlem_set_sinograms are kept). */
int mlem_stream_host(mlem_ctx* ctx, const int32_t* const* sinos, float* const* images,
                     uint32_t n);

/* Phases of one iteration, as timed by mlem_profile_phases. */
#define MLEM_PHASE_PROJECT 0     /* forward projection + calcCorrel (or the one-pass kernel) */
#define MLEM_PHASE_BACKPROJECT 1 /* back projection (+ calcUpdate for the CSC method) */
#define MLEM_PHASE_UPDATE 2      /* calcUpdate for the scatter methods */
#define MLEM_PHASE_STATS 3       /* per-iteration image sum / zero / subnormal census */
#define MLEM_N_PHASES 4

/* Run n iterations with CUDA events around every phase on the context's
 * stream.  ms[p]: average device time of phase p per iteration; bytes[p]:
 * the algorithmic bytes phase p moves per iteration (each matrix element,
 * offset and vector entry counted once per pass); launches[p]: kernels per
 * iteration.  Changes the images like mlem_iterate. */
int mlem_profile_phases(mlem_ctx* ctx, int n_iter, double* ms, double* bytes, int* launches);
/* The rates the L2 serves to random addresses on `device`, measured with
 * four small kernels over a 64 MB scratch array (allocated and freed here):
 * rates[0] float gathers of 4 bytes per second, rates[1] gathers of 64-byte
 * rows (16 floats) per second, rates[2] float reductions (red.global.add) of
 * 4 bytes per second, rates[3] reductions of 64-byte rows per second.  The
 * one-pass iteration gathers and reduces at such addresses; its measured
 * bound.  No counterpart in the reference. */
int mlem_measure_l2_rates(int device, double* rates);

/* ---- tuning --------------------------------------------------------------- */
int mlem_get_tuning(const mlem_ctx* ctx, mlem_tuning* out);
int mlem_set_tuning(mlem_ctx* ctx, const mlem_tuning* t);
/* Time every valid configuration for the current B on the device and keep
 * the fastest (deterministic_only != 0 restricts to MLEM_BK_CSC).  The
 * image state is restored afterwards. */
int mlem_autotune(mlem_ctx* ctx, int deterministic_only, mlem_tuning* best);

/* ---- ordered subsets (OSEM) ---------------------------------------------
 * No counterpart in the reference (its thesis names OSEM as future work).
 * Rows are split into n_subsets interleaved subsets (row r in subset
 * r % n_subsets) and every iteration of mlem_iterate / mlem_step_host runs
 * them in order 0, 1, ...: the one-pass forward projection, correlation and
 * back projection over the subset's rows, then
 *   x *= norm_s != 0 ? u / norm_s : (norm != 0 ? 1 : u)
 * with norm_s the subset's column sums (bit-exact sums over the CSC, in row
 * order; atomic without a CSC), so a voxel the subset does not see keeps its
 * value and one subset is the reference's calcUpdate.  The image statistics
 * are taken after each full iteration.  Needs the one-pass method
 * (MLEM_BK_FUSED, any row visit; mlem_autotune then tries only it); not in
 * the bit-exact mode.  n_subsets 1 turns subsets off.  mlem_set_norm_d does
 * not change the subset column sums. */
int mlem_set_subsets(mlem_ctx* ctx, uint32_t n_subsets);
int mlem_get_subsets(const mlem_ctx* ctx, uint32_t* n_subsets);
/* Column sums of subset s (natural voxel order, C floats); n_subsets >= 2. */
int mlem_subset_column_sums(mlem_ctx* ctx, uint32_t s, float* out);

/* ---- device-pointer entry points (torch extension, custom drivers) ------ */
/* y[R][B] = A x[C][B]. */
int mlem_fwproj_d(mlem_ctx* ctx, const float* x, float* y, uint32_t n_frames, void* stream);
/* x[C][B] = A^T y[R][B]. */
int mlem_bkproj_d(mlem_ctx* ctx, const float* y, float* x, uint32_t n_frames, void* stream);
/* correl[R][B] = calcCorrel(sino[R][B], A x[C][B])  (fused). */
int mlem_fwproj_correl_d(mlem_ctx* ctx, const float* x, const int32_t* sino, float* correl,
                         uint32_t n_frames, void* stream);
/* update[C][B] = A^T calcCorrel(sino[R][B], A x[C][B]) in one pass over the
 * matrix (the one-pass kernels, with the context's row visit when it is tuned
 * to MLEM_BK_FUSED, else sorted rows in chunks): the partial update of a row
 * shard (mlem_mpi/fusedmpimlem.cpp:205-225) or the numerator of calcUpdate.
 * sino NULL: the context's own sinograms (mlem_set_sinograms with n_frames
 * frames, a power of two up to 16 so that none is padded); the sorted visits
 * then leave out the rows whose counts are zero in every frame, as an
 * iteration does.  Summation order varies from run to run (float atomics).
 * Not in the bit-exact mode; must not run concurrently with the context's
 * own iterations. */
int mlem_fused_update_d(mlem_ctx* ctx, const float* x, const int32_t* sino, float* update,
                        uint32_t n_frames, void* stream);
/* x[C][B] *= calcUpdate factor(A^T correl[R][B], norm)  (fused, CSC). */
int mlem_bkproj_update_d(mlem_ctx* ctx, const float* correl, float* x, uint32_t n_frames,
                         void* stream);
/* x[C][B] *= calcUpdate factor(update[C][B], norm): the update step of a
 * row-sharded reconstruction after the update vectors of all shards have
 * been summed (the single exchange of mlem_mpi/fusedmpimlem.cpp:227). */
int mlem_apply_update_d(mlem_ctx* ctx, const float* update, float* x, uint32_t n_frames,
                        void* stream);
/* The two one-pass kernels of the unrolled MLEM's backward pass (one frame,
 * device pointers, natural voxel order; no counterpart in the reference):
 *   mlem_ratio_rows_d:    update = A^T calcCorrel(sino, A x) as
 *                         mlem_fused_update_d, and rows[R] = A x for the
 *                         rows with a nonzero count (0 for the others);
 *   mlem_adjoint_update_d: update = A^T df with
 *                         df_r = -(A du)_r * (sino_r / rows_r) / rows_r where
 *                         sino_r and rows_r are nonzero, else 0 -- the
 *                         adjoint of calcCorrel and both projections.
 * Each is one pass over the matrix; rows without counts are skipped before
 * their elements are read.  Summation order varies from run to run.  Not in
 * the bit-exact mode nor with MLEM_FLAG_MIRROR_KERNELS; must not run
 * concurrently with the context's own iterations or mlem_fused_update_d. */
int mlem_ratio_rows_d(mlem_ctx* ctx, const float* x, const int32_t* sino, float* rows,
                      float* update, void* stream);
int mlem_adjoint_update_d(mlem_ctx* ctx, const float* du, const int32_t* sino, const float* rows,
                          float* update, void* stream);
/* Device pointer of the context's column sums (float[C]). */
int mlem_norm_d(mlem_ctx* ctx, const float** norm);
/* Replace the column sums with norm[C] (device pointer): a row shard uses the
 * column sums of the whole matrix (mlem_mpi/mpicsr4mlem.cpp:266). */
int mlem_set_norm_d(mlem_ctx* ctx, const float* norm, void* stream);
/* Sequential double projection out[R] = A x (bit-identical to the host
 * generator's; used for synthetic sinogram means).  Host buffers. */
int mlem_project_f64(mlem_ctx* ctx, const float* x, double* out);

/* ---- matrix-free iteration (prototype) ------------------------------------
 * No counterpart in the reference, which reads a stored CSR4 matrix from an
 * external generator (README.md:35-36).  For the synthetic Siddon geometry
 * (mlem_create_siddon's parameters) the matrix is never stored: every ray is
 * kept as a small descriptor of the generator's accepted line (entry point,
 * direction, alpha range inside the grid: 104 bytes instead of about 8 bytes
 * per element) and traced again, in double, in every pass.  One iteration is
 * one pass per ray: forward projection, calcCorrel and the scatter of the
 * traced elements, then calcUpdate.  The traced lengths equal the generator's
 * up to rounding (a voxel cut by a lane's interval boundary is traced as two
 * pieces), so results agree with a stored-matrix context of the same
 * geometry within the float tolerance, not bit for bit.  Rays whose count is
 * zero are skipped.  One frame; images in natural voxel order.  A walk whose
 * interval held more elements than its bound returns MLEM_ERR_CUDA (the bound
 * follows from the grid's diagonal, so this does not happen). */
typedef struct mlem_mf mlem_mf;
int mlem_mf_create_siddon(mlem_mf** out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t n_rows,
                          uint32_t min_count, uint32_t max_count, double radius_scale,
                          double min_len, uint64_t seed, int device);
void mlem_mf_destroy(mlem_mf* mf);
int mlem_mf_set_stream(mlem_mf* mf, void* stream);
/* Column sums (traced once at creation), natural voxel order, float[C]. */
int mlem_mf_column_sums(mlem_mf* mf, float* norm);
/* Upload the int32[R] sinogram (host buffer). */
int mlem_mf_set_sinogram(mlem_mf* mf, const int32_t* sino);
/* initImage (seqcsr4mlem.cpp:52-66); init_value (may be NULL) receives the value. */
int mlem_mf_init_image(mlem_mf* mf, float* init_value);
int mlem_mf_iterate(mlem_mf* mf, int n_iter);
int mlem_mf_get_image(mlem_mf* mf, float* image);
/* Device bytes held (descriptors, vectors, voxel order) and the per-lane element bound. */
int mlem_mf_info(const mlem_mf* mf, uint64_t* device_bytes, uint32_t* lane_capacity);

/* ---- allocation-free iteration ------------------------------------------- */
/* No counterpart in the reference.  Every other entry point keeps working
 * vectors in device memory the library allocates.  This one is for callers
 * that cannot let a library call cudaMalloc: programs that run inside a fixed
 * device-memory budget handed out by a framework or scheduler, or that run
 * while another component owns the device allocator.  It runs one MLEM
 * iteration (calcFwProj, calcCorrel, calcBkProj, calcUpdate,
 * mlem_seq/seqcsr4mlem.cpp:164-167) on caller-owned DEVICE buffers and calls
 * no cudaMalloc, cudaFree or allocating library routine:
 *   row_ptr  uint64[R+1]: row offsets WITH a leading 0 (the CSR4 row END
 *            offsets shifted by one); elems: n_elems 8-byte {uint32 column,
 *            float32 value} elements; sino int32[R]; norm float32[C] (the
 *            column sums); image float32[C], updated in place.
 * Its only working vector, the back-projection update, is a fixed
 * MLEM_NOALLOC_MAX_VOXELS-float array in the library's static device memory:
 * every GPU that loads the library holds those 4 MiB until exit.  Images with
 * more voxels are rejected (MLEM_ERR_INVALID).  All calls on a device share the
 * array and each call clears it first, so calls that overlap on the GPU
 * (several streams or host threads) race and must be serialised by the
 * caller.  The first call on a device (and the first after its context is
 * created again) does a one-time set-up: it looks up the array's device
 * address (cudaGetSymbolAddress, with that device current); make that first
 * call before any stream capture begins.  The call enqueues on `stream`, then
 * waits for the stream to finish and reads the kernels' error word back.  It
 * checks the matrix as it goes: a row whose offsets decrease or pass n_elems
 * is skipped, and so is an element whose column is >= n_cols; either gives
 * MLEM_ERR_MATRIX after the iteration (the other rows are applied).  Natural
 * voxel order; one frame. */
#define MLEM_NOALLOC_MAX_VOXELS 1048576
int mlem_iterate_noalloc_d(const uint64_t* row_ptr, const void* elems, uint64_t n_elems,
                           uint32_t n_rows, uint32_t n_cols, const int32_t* sino,
                           const float* norm, float* image, void* stream);

/* ---- uneven multi-matrix batches ----------------------------------------
 * No counterpart in the reference, which reconstructs one matrix per process
 * (seqcsr4mlem.cpp:137-189).  A batch iterates several contexts (different
 * scanner matrices, different frame counts) together on one GPU.  Each
 * iteration runs ONE kernel over the rows of all matrices, then a per-matrix
 * calcUpdate and the image statistics; up to 64 iterations are captured as
 * one graph.  Every row does the one-pass fwproj + correl + scatter for all
 * frames of its matrix, in passes of one frame tile shared by the batch.  Two
 * schedules share the rows out:
 *   MLEM_BATCH_INTERLEAVED -- the rows of all matrices form one virtual row
 *     space that the warps walk in grid-stride order, so every warp gets an
 *     equal share of every matrix and a small matrix fills the tail of a
 *     large one;
 *   MLEM_BATCH_ITEMS -- the rows are cut into work items of about equal cost
 *     (full items of the costliest matrix first, ragged remainders last,
 *     heaviest first) that persistent blocks take from a shared counter.
 *
 * All contexts must live on the same device, be created without
 * MLEM_FLAG_EXACT, and have sinograms and images set.  The batch enqueues on
 * the first context's stream and waits for the others'; the contexts stay
 * usable (mlem_get_images, ...) and must outlive the batch.  Results equal
 * each context's own MLEM_BK_FUSED iterations up to float rounding (the
 * scatter order differs). */
typedef struct mlem_batch mlem_batch;
#define MLEM_BATCH_MAX_MATRICES 64
#define MLEM_BATCH_INTERLEAVED 0
#define MLEM_BATCH_ITEMS 1
int mlem_batch_create(mlem_batch** out, mlem_ctx* const* ctxs, uint32_t n_ctx);
void mlem_batch_destroy(mlem_batch* b);
const char* mlem_batch_last_error(const mlem_batch* b);
/* policy: MLEM_BATCH_INTERLEAVED or MLEM_BATCH_ITEMS; items_per_block (1..1024,
 * items schedule): about that many items for every resident block
 * (blocks_per_sm x SMs); frame_tile in {1,2,4,8,16} dividing every context's
 * padded frame count (0 keeps the current tile); visit: MLEM_VISIT_FILE or
 * MLEM_VISIT_SORTED for every matrix, or MLEM_VISIT_SORTED_STAGED with the
 * items schedule (sorted needs every context's row order; with the items
 * schedule a sorted item is a run of neighbouring rows; staged pipelines each
 * warp's rows of an item through shared memory, at most 4 blocks per SM).
 * Every context takes the batch's visit again (see mlem_batch_set_visits). */
int mlem_batch_set_schedule(mlem_batch* b, int policy, uint32_t items_per_block,
                            int blocks_per_sm, int frame_tile, int visit);
/* A frame tile for each context (n_ctx entries): 0 follows the batch's tile,
 * else 1, 2, 4, 8 or 16 dividing that context's padded frame count.  The
 * contexts that share a tile share one kernel per iteration (heaviest group
 * first).  mlem_batch_set_schedule with a non-zero frame_tile sets every
 * context back to the batch's tile. */
int mlem_batch_set_tiles(mlem_batch* b, const int* tiles);
/* The frame tile each context runs with (n_ctx entries). */
int mlem_batch_get_tiles(const mlem_batch* b, int* tiles);
/* A row visit for each context (n_ctx entries): -1 follows the batch's visit,
 * else MLEM_VISIT_FILE, MLEM_VISIT_SORTED or, with the items schedule,
 * MLEM_VISIT_SORTED_STAGED (the sorted visits need the context's row order).
 * The contexts that share a frame tile and a visit share one kernel per
 * iteration. */
int mlem_batch_set_visits(mlem_batch* b, const int* visits);
/* The row visit each context runs with (n_ctx entries). */
int mlem_batch_get_visits(const mlem_batch* b, int* visits);
/* Current schedule; any pointer may be NULL.  n_items: 0 for the interleaved
 * schedule.  ms_per_iter: from the last autotune, else 0. */
int mlem_batch_get_schedule(const mlem_batch* b, int* policy, uint32_t* items_per_block,
                            int* blocks_per_sm, int* frame_tile, int* visit, uint32_t* n_items,
                            double* ms_per_iter);
/* Time real iterations over schedules, frame tiles, row visits and resident
 * blocks, then a tile and a visit per context, and keep the fastest; the
 * images are restored afterwards. */
int mlem_batch_autotune(mlem_batch* b, double* ms_per_iter);
/* n iterations of every context.  sums may be NULL, or hold n_ctx pointers
 * (each NULL or n x n_frames doubles, iteration-major) for the image sums. */
int mlem_batch_iterate(mlem_batch* b, int n, double* const* sums);
/* Like mlem_profile_phases for the whole batch: ms[0] = the multi-matrix
 * kernel, ms[2] = the calcUpdate launches, ms[3] = the statistics, averaged
 * over n iterations; bytes[] are the algorithmic bytes of each phase summed
 * over the contexts. */
int mlem_batch_profile(mlem_batch* b, int n, double* ms, double* bytes, int* launches);

/* ---- host IO: the reference's file formats ------------------------------ */
typedef struct {
    uint32_t n_rows, n_cols;
    uint64_t nnz;
    uint8_t version, flags;
    uint32_t scan_config_bytes;
    uint32_t grid[3];
    float voxel_size[3];
    uint64_t file_size;
    uint64_t data_offset; /* byte offset of the row END offsets */
    uint32_t n_layers, n_blocks, block_size, n_rings; /* detector of the scanner block */
} mlem_csr4_header;

/* Parse and validate a CSR4 header like csr4matrix.cpp:32-138, with 64-bit
 * size arithmetic. */
int mlem_csr4_read_header(const char* path, mlem_csr4_header* out);
/* Read the row END offsets [R] and elements [Z] of a CSR4 file. */
int mlem_csr4_read(const char* path, uint64_t* row_end, void* elems);
/* Write a CSR4 file with the minimal 60-byte scanner block. */
int mlem_csr4_write(const char* path, const uint64_t* row_end, const void* elems,
                    uint32_t n_rows, uint32_t n_cols, const uint32_t grid[3]);
/* vector.hpp:33-53: element count = file size / elem_size (error if not a
 * multiple).  Call with buf == NULL to query the count. */
int mlem_vector_read(const char* path, uint32_t elem_size, void* buf, uint64_t capacity,
                     uint64_t* count);
/* vector.hpp:77-87 writeToFile, or :102-114 writeToFileSync when sync != 0. */
int mlem_vector_write(const char* path, const void* buf, uint32_t elem_size, uint64_t count,
                      int sync);
/* mpicsr4mlem.cpp:95-122 checkPointNow: img.chkpt (float32[C], fsync'd) and
 * iter.chkpt (int32 next iteration) in `dir`. */
int mlem_checkpoint_write(const char* dir, const float* image, uint32_t n_cols, int32_t next_iter);
/* mpicsr4mlem.cpp:133-154 restore + :536-550: MLEM_NO_CHECKPOINT unless both
 * files exist; the image must have exactly n_cols floats. */
int mlem_checkpoint_read(const char* dir, float* image, uint32_t n_cols, int32_t* next_iter);
/* mpicsr4mlem.cpp:656-660: remove both checkpoint files. */
int mlem_checkpoint_remove(const char* dir);

/* mpicsr4mlem.cpp:202-234 partition(): nnz-balanced contiguous row ranges
 * for n_ranks (starts/ends: n_ranks entries each). */
int mlem_partition_rows(const uint64_t* row_end, uint32_t n_rows, int n_ranks, uint32_t* starts,
                        uint32_t* ends);

#ifdef __cplusplus
}
#endif

#endif /* MLEM_B200_H */
