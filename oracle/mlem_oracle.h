/*
 * mlem_oracle.h -- CPU restatement of the reference MLEM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity checker for the CUDA path in
 * mlem_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product never links or calls it.
 *
 * Every function restates one function of the reference's sequential MLEM
 * (mlem_seq/seqcsr4mlem.cpp) with the same operation order and the same
 * float/double types, so that, compiled with -ffp-contract=off on x86-64, it
 * reproduces the reference binary bit for bit.  The f64 variants are the
 * FP64 oracle: the same iteration with every quantity in double.
 *
 * Matrix layout is the CSR4 on-disk layout (helper_files_common/csr4matrix.cpp
 * :32-157): R uint64 row END offsets (no leading zero) and Z 8-byte elements
 * {uint32 column, float value} (helper_files_common/matrixelement.hpp:37-46).
 */
#ifndef MLEM_ORACLE_H
#define MLEM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t index; /* column (CSR) or row (CSC) */
    float value;
} oracle_elem;

/* mlem_seq/seqcsr4mlem.cpp:37-49 calcColumnSums: norm[c] = sum of column c, float, row order. */
void oracle_column_sums(uint32_t R, uint32_t C, const uint64_t* row_end,
                        const oracle_elem* e, float* norm);

/* mlem_seq/seqcsr4mlem.cpp:52-66 initImage: float(sum_double(sino) / sum_double(norm)). */
float oracle_init_value(uint32_t C, const float* norm, uint64_t S, const int32_t* sino,
                        double* sumnorm_out, double* sumin_out);

/* mlem_seq/seqcsr4mlem.cpp:69-91 calcFwProj: f[r] = float dot product in element order. */
void oracle_fwproj(uint32_t R, const uint64_t* row_end, const oracle_elem* e,
                   const float* x, float* f);

/* mlem_seq/seqcsr4mlem.cpp:94-105 calcCorrel: c = f != 0 ? (float)s / f : 0. */
void oracle_correl(uint64_t R, const float* f, const int32_t* s, float* c);

/* mlem_seq/seqcsr4mlem.cpp:108-120 calcBkProj: u[col] += v * c[row] in row order. */
void oracle_bkproj(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                   const float* c, float* u);

/* mlem_seq/seqcsr4mlem.cpp:123-134 calcUpdate: x *= norm != 0 ? u / norm : u. */
void oracle_update(uint32_t C, const float* u, const float* norm, float* x);

/*
 * mlem_seq/seqcsr4mlem.cpp:137-189 mlem() plus the FTZ mode main() sets at :194.
 * Runs calcColumnSums, initImage (skipped when start_image != NULL: the restart
 * path of mlem_mpi/mpicsr4mlem.cpp:536-553) and n_iter iterations.
 * image_sums (may be NULL) receives the per-iteration float image sum the
 * reference prints (:172-185).  Returns 0, or -1 on a size mismatch
 * (the reference asserts there).
 */
int oracle_mlem(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                const int32_t* sino, uint64_t S, int n_iter, int ftz,
                const float* start_image, float* image, float* image_sums);

/*
 * Ordered subsets (OSEM, Hudson & Larkin 1994), which the reference names as
 * future work but does not implement: row r belongs to subset r % n_subsets,
 * and every iteration runs the subsets in order 0, 1, ...  A sub-iteration is
 * the reference iteration restricted to the subset's rows (seqcsr4mlem.cpp:
 * 69-120 visiting only those rows, in ascending order), followed by the update
 *   x *= norm_s != 0 ? u / norm_s : (norm != 0 ? 1 : u)
 * with norm_s the subset's column sums (calcColumnSums over the subset's rows,
 * seqcsr4mlem.cpp:37-49): a voxel the subset does not see keeps its value,
 * and with one subset this is calcUpdate (seqcsr4mlem.cpp:123-134), so
 * oracle_osem(..., 1, ...) equals oracle_mlem bit for bit.  The initial image
 * is initImage over the full column sums.  image_sums (may be NULL) gets the
 * float image sum after each full iteration.
 */
int oracle_osem(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                const int32_t* sino, uint64_t S, int n_iter, uint32_t n_subsets, int ftz,
                const float* start_image, float* image, float* image_sums);

/* Column sums over the rows of subset s (r % n_subsets == s), in row order. */
void oracle_subset_column_sums(uint32_t R, uint32_t C, const uint64_t* row_end,
                               const oracle_elem* e, uint32_t n_subsets, uint32_t s,
                               float* norm);

/*
 * The full matrix of a symmetry-compressed CSR4 matrix, as the reference's
 * matrix viewer regenerates it (visualizematrix/dispcsr4spy.cpp:123-140 with
 * symhandler.hpp/.cpp): for each mirror the flags allow (sym bits x = 1,
 * y = 2, z = 4; generateSyms order, x outermost, identity excluded) and each
 * stored row r, the elements of r with voxels mirrored (transformVoxel) go to
 * row transformLor(r).  Full row t holds its stored elements first, then each
 * mirror's contributions, source rows ascending.  Rows are LORs
 * d1 * n_crystals + d2; columns voxels of the nx x ny x nz grid.  Returns the
 * full element count; row_end_out (R) and e_out receive the matrix when
 * non-NULL.
 */
uint64_t oracle_expand_symmetries(uint32_t R, const uint64_t* row_end, const oracle_elem* e,
                                  uint32_t sym, uint32_t n_layers, uint32_t n_blocks,
                                  uint32_t block_size, uint32_t n_rings, uint32_t nx,
                                  uint32_t ny, uint32_t nz, uint64_t* row_end_out,
                                  oracle_elem* e_out);

/* FP64 oracle: the same iteration with double norm, projections, ratios and image. */
int oracle_mlem_f64(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                    const int32_t* sino, uint64_t S, int n_iter, double* image);

/* oracle_mlem_f64 on n_threads host threads (OpenMP): row blocks of about
 * equal element counts, private double column sums and update vectors added in
 * thread order.  Equal to oracle_mlem_f64 up to the order of double additions
 * in the column sums and the back projection. */
int oracle_mlem_f64_threads(uint32_t R, uint32_t C, const uint64_t* row_end,
                            const oracle_elem* e, const int32_t* sino, uint64_t S, int n_iter,
                            int n_threads, double* image);

/*
 * Relaxed FP64 MLEM used by the gradient checks:
 *   x_{k+1} = x_k * ratio_k ^ omega_k,  ratio_k = calcUpdate's factor
 * (u/norm, or u where norm == 0), u = A^T (s / A x_k) with the calcCorrel
 * zero rule.  omega_k == 1 gives the reference iteration.
 */
void oracle_mlem_relaxed_f64(uint32_t R, uint32_t C, const uint64_t* row_end,
                             const oracle_elem* e, const int32_t* sino, const double* x0,
                             const double* omega, int K, double* xK);

/* Sequential double projection sum_k (double)v_k * x[col_k], no FMA (sinogram means). */
void oracle_project_f64(uint32_t R, const uint64_t* row_end, const oracle_elem* e,
                        const float* x, double* out);

/* Analytic gradient of the Poisson negative log-likelihood: A^T (1 - s / A x), double. */
void oracle_poisson_grad_f64(uint32_t R, uint32_t C, const uint64_t* row_end,
                             const oracle_elem* e, const int32_t* s, const double* x,
                             double* grad);

/*
 * Stable CPU transpose CSR -> CSC: col_ptr has C+1 entries starting at 0;
 * within a column, entries are in ascending row order, and entries of the
 * same (row, column) keep their in-row order.  This is the order in which
 * calcBkProj (seqcsr4mlem.cpp:116-119) adds into update[col].
 */
void oracle_transpose(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                      uint64_t* col_ptr, oracle_elem* ce);

/* mlem_mpi/mpicsr4mlem.cpp:202-234 partition(): nnz-balanced contiguous row ranges.
 * starts/ends receive n_ranks entries each. */
void oracle_partition(uint32_t R, const uint64_t* row_end, int n_ranks,
                      uint32_t* starts, uint32_t* ends);

#ifdef __cplusplus
}
#endif

#endif /* MLEM_ORACLE_H */
