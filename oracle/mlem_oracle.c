/*
 * mlem_oracle.c -- CPU restatement of the reference MLEM hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker).  See mlem_oracle.h for the
 * contract; every function cites the reference function it restates.
 * Build with -ffp-contract=off so no multiply-add is fused: the reference is
 * compiled for x86-64 without FMA, and bit-exact agreement depends on that.
 */
#include "mlem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#if defined(__x86_64__) || defined(__i386__)
#include <xmmintrin.h>
#define ORACLE_HAVE_MXCSR 1
#endif

static inline uint64_t row_begin(const uint64_t* row_end, uint32_t r) {
    /* helper_files_common/csr4matrix.hpp:138-140: row r starts at row_end[r-1]. */
    return r == 0 ? 0 : row_end[r - 1];
}

void oracle_column_sums(uint32_t R, uint32_t C, const uint64_t* row_end,
                        const oracle_elem* e, float* norm) {
    /* seqcsr4mlem.cpp:41 zero-fill, then :44-47 scatter-add in row order. */
    memset(norm, 0, (size_t)C * sizeof(float));
    for (uint32_t r = 0; r < R; ++r)
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            norm[e[k].index] += e[k].value;
}

float oracle_init_value(uint32_t C, const float* norm, uint64_t S, const int32_t* sino,
                        double* sumnorm_out, double* sumin_out) {
    /* seqcsr4mlem.cpp:55-60 */
    double sumnorm = 0.0;
    for (uint32_t i = 0; i < C; ++i) sumnorm += norm[i];
    double sumin = 0.0;
    for (uint64_t i = 0; i < S; ++i) sumin += sino[i];
    if (sumnorm_out) *sumnorm_out = sumnorm;
    if (sumin_out) *sumin_out = sumin;
    return (float)(sumin / sumnorm);
}

void oracle_fwproj(uint32_t R, const uint64_t* row_end, const oracle_elem* e,
                   const float* x, float* f) {
    /* seqcsr4mlem.cpp:76-90: float accumulator, multiply then add. */
    for (uint32_t r = 0; r < R; ++r) {
        float res = 0.0f;
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            res += e[k].value * x[e[k].index];
        f[r] = res;
    }
}

void oracle_correl(uint64_t R, const float* f, const int32_t* s, float* c) {
    /* seqcsr4mlem.cpp:98-99: the int count is converted to float before the divide. */
    for (uint64_t i = 0; i < R; ++i)
        c[i] = (f[i] != 0.0) ? ((float)s[i] / f[i]) : 0.0f;
}

void oracle_bkproj(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                   const float* c, float* u) {
    /* seqcsr4mlem.cpp:113 zero-fill, :116-119 scatter in row order. */
    memset(u, 0, (size_t)C * sizeof(float));
    for (uint32_t r = 0; r < R; ++r)
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            u[e[k].index] += e[k].value * c[r];
}

void oracle_update(uint32_t C, const float* u, const float* norm, float* x) {
    /* seqcsr4mlem.cpp:127-128 */
    for (uint32_t i = 0; i < C; ++i)
        x[i] *= (norm[i] != 0.0) ? (u[i] / norm[i]) : u[i];
}

int oracle_mlem(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                const int32_t* sino, uint64_t S, int n_iter, int ftz,
                const float* start_image, float* image, float* image_sums) {
    if (S != R) return -1; /* seqcsr4mlem.cpp:96 asserts fwproj.size() == input.size() */
#ifdef ORACLE_HAVE_MXCSR
    unsigned int saved = _mm_getcsr();
    if (ftz) _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON); /* seqcsr4mlem.cpp:194 */
#else
    (void)ftz;
#endif
    float* fw = (float*)malloc((size_t)R * sizeof(float) + 1);
    float* cr = (float*)malloc((size_t)R * sizeof(float) + 1);
    float* up = (float*)malloc((size_t)C * sizeof(float) + 1);
    float* norm = (float*)malloc((size_t)C * sizeof(float) + 1);
    int rc = 0;
    if (!fw || !cr || !up || !norm) { rc = -2; goto done; }

    oracle_column_sums(R, C, row_end, e, norm);
    if (start_image) {
        memcpy(image, start_image, (size_t)C * sizeof(float));
    } else {
        float init = oracle_init_value(C, norm, S, sino, NULL, NULL);
        for (uint32_t i = 0; i < C; ++i) image[i] = init;
    }
    for (int it = 0; it < n_iter; ++it) {
        oracle_fwproj(R, row_end, e, image, fw);
        oracle_correl(R, fw, sino, cr);
        oracle_bkproj(R, C, row_end, e, cr, up);
        oracle_update(C, up, norm, image);
        if (image_sums) {
            float s = 0.0f; /* seqcsr4mlem.cpp:174-176 */
            for (uint32_t i = 0; i < C; ++i) s += image[i];
            image_sums[it] = s;
        }
    }
done:
    free(fw); free(cr); free(up); free(norm);
#ifdef ORACLE_HAVE_MXCSR
    _mm_setcsr(saved);
#endif
    return rc;
}

void oracle_subset_column_sums(uint32_t R, uint32_t C, const uint64_t* row_end,
                               const oracle_elem* e, uint32_t n_subsets, uint32_t s,
                               float* norm) {
    /* seqcsr4mlem.cpp:41-47 over the subset's rows, ascending. */
    memset(norm, 0, (size_t)C * sizeof(float));
    for (uint32_t r = s; r < R; r += n_subsets)
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            norm[e[k].index] += e[k].value;
}

int oracle_osem(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                const int32_t* sino, uint64_t S, int n_iter, uint32_t n_subsets, int ftz,
                const float* start_image, float* image, float* image_sums) {
    if (S != R) return -1;
    if (n_subsets == 0) return -3;
#ifdef ORACLE_HAVE_MXCSR
    unsigned int saved = _mm_getcsr();
    if (ftz) _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON); /* seqcsr4mlem.cpp:194 */
#else
    (void)ftz;
#endif
    float* fw = (float*)malloc((size_t)R * sizeof(float) + 1);
    float* up = (float*)malloc((size_t)C * sizeof(float) + 1);
    float* norm = (float*)malloc((size_t)C * sizeof(float) + 1);
    float* nsub = (float*)malloc((size_t)C * n_subsets * sizeof(float) + 1);
    int rc = 0;
    if (!fw || !up || !norm || !nsub) { rc = -2; goto done; }

    oracle_column_sums(R, C, row_end, e, norm);
    for (uint32_t s = 0; s < n_subsets; ++s)
        oracle_subset_column_sums(R, C, row_end, e, n_subsets, s, nsub + (size_t)s * C);
    if (start_image) {
        memcpy(image, start_image, (size_t)C * sizeof(float));
    } else {
        float init = oracle_init_value(C, norm, S, sino, NULL, NULL);
        for (uint32_t i = 0; i < C; ++i) image[i] = init;
    }
    for (int it = 0; it < n_iter; ++it) {
        for (uint32_t s = 0; s < n_subsets; ++s) {
            const float* ns = nsub + (size_t)s * C;
            /* calcFwProj + calcCorrel (seqcsr4mlem.cpp:76-99) on the subset's rows */
            for (uint32_t r = s; r < R; r += n_subsets) {
                float res = 0.0f;
                for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                    res += e[k].value * image[e[k].index];
                fw[r] = (res != 0.0) ? ((float)sino[r] / res) : 0.0f;
            }
            /* calcBkProj (seqcsr4mlem.cpp:113-119) on the subset's rows */
            memset(up, 0, (size_t)C * sizeof(float));
            for (uint32_t r = s; r < R; r += n_subsets)
                for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                    up[e[k].index] += e[k].value * fw[r];
            for (uint32_t i = 0; i < C; ++i)
                image[i] *= (ns[i] != 0.0) ? (up[i] / ns[i]) : ((norm[i] != 0.0) ? 1.0f : up[i]);
        }
        if (image_sums) {
            float sum = 0.0f; /* seqcsr4mlem.cpp:174-176 */
            for (uint32_t i = 0; i < C; ++i) sum += image[i];
            image_sums[it] = sum;
        }
    }
done:
    free(fw); free(up); free(norm); free(nsub);
#ifdef ORACLE_HAVE_MXCSR
    _mm_setcsr(saved);
#endif
    return rc;
}

/* symhandler.cpp:33-114 initLUTs: crystal c = v + layer * per_layer + ring * per_ring. */
static uint32_t sym_detector(uint32_t c, uint32_t m, uint32_t n_layers, uint32_t n_blocks,
                             uint32_t block_size, uint32_t n_rings) {
    const uint32_t per_layer = block_size * n_blocks, per_ring = per_layer * n_layers;
    /* lut 7 = z(y(x)), 3 = y(x), 5 = z(x), 6 = z(y): apply x, then y, then z */
    if (m & 1u) {
        uint32_t v = c % per_layer, rest = c - v;
        c = (per_layer - v + block_size - 1) % per_layer + rest;
    }
    if (m & 2u) {
        uint32_t v = c % per_layer, rest = c - v;
        c = (per_layer - v + block_size * (n_blocks / 2 + 1) - 1) % per_layer + rest;
    }
    if (m & 4u) {
        uint32_t ring = c / per_ring, v = c % per_ring;
        c = v + (n_rings - 1 - ring) * per_ring;
    }
    return c;
}

static uint32_t sym_lor(uint32_t r, uint32_t m, uint32_t nc, uint32_t n_layers, uint32_t n_blocks,
                        uint32_t block_size, uint32_t n_rings) {
    /* symhandler.hpp transformLor: mirror both detectors, smaller one first */
    uint32_t d1 = sym_detector(r / nc, m, n_layers, n_blocks, block_size, n_rings);
    uint32_t d2 = sym_detector(r % nc, m, n_layers, n_blocks, block_size, n_rings);
    return d1 < d2 ? d1 * nc + d2 : d2 * nc + d1;
}

static uint32_t sym_voxel(uint32_t v, uint32_t m, uint32_t nx, uint32_t ny, uint32_t nz) {
    /* symhandler.hpp transformVoxel */
    uint32_t slice = nx * ny, z = v / slice, y = (v % slice) / nx, x = v % nx;
    if (m & 1u) x = nx - 1 - x;
    if (m & 2u) y = ny - 1 - y;
    if (m & 4u) z = nz - 1 - z;
    return z * slice + y * nx + x;
}

uint64_t oracle_expand_symmetries(uint32_t R, const uint64_t* row_end, const oracle_elem* e,
                                  uint32_t sym, uint32_t n_layers, uint32_t n_blocks,
                                  uint32_t block_size, uint32_t n_rings, uint32_t nx,
                                  uint32_t ny, uint32_t nz, uint64_t* row_end_out,
                                  oracle_elem* e_out) {
    const uint32_t nc = block_size * n_blocks * n_layers * n_rings;
    uint32_t mirrors[8], nm = 0;
    for (uint32_t x = 0; x <= (sym & 1u); ++x) /* generateSyms, symhandler.hpp:37-51 */
        for (uint32_t y = 0; y <= ((sym >> 1) & 1u); ++y)
            for (uint32_t z = 0; z <= ((sym >> 2) & 1u); ++z)
                if (x || y || z) mirrors[nm++] = x | (y << 1) | (z << 2);
    uint64_t* len = (uint64_t*)calloc((size_t)R + 1, sizeof(uint64_t));
    if (!len) return 0;
    for (uint32_t r = 0; r < R; ++r) len[r] = row_end[r] - row_begin(row_end, r);
    uint64_t* full = (uint64_t*)calloc((size_t)R + 1, sizeof(uint64_t));
    if (!full) { free(len); return 0; }
    for (uint32_t r = 0; r < R; ++r) full[r] += len[r];
    for (uint32_t i = 0; i < nm; ++i)
        for (uint32_t r = 0; r < R; ++r)
            full[sym_lor(r, mirrors[i], nc, n_layers, n_blocks, block_size, n_rings)] += len[r];
    uint64_t total = 0;
    for (uint32_t r = 0; r < R; ++r) total += full[r];
    if (row_end_out && e_out) {
        uint64_t* cur = full; /* reused as the write cursor of each full row */
        uint64_t acc = 0;
        for (uint32_t r = 0; r < R; ++r) {
            uint64_t n = cur[r];
            cur[r] = acc;
            acc += n;
            row_end_out[r] = acc;
        }
        for (uint32_t r = 0; r < R; ++r)
            for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k) e_out[cur[r]++] = e[k];
        for (uint32_t i = 0; i < nm; ++i)
            for (uint32_t r = 0; r < R; ++r) {
                uint32_t t = sym_lor(r, mirrors[i], nc, n_layers, n_blocks, block_size, n_rings);
                for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k) {
                    oracle_elem q = e[k];
                    q.index = sym_voxel(q.index, mirrors[i], nx, ny, nz);
                    e_out[cur[t]++] = q;
                }
            }
    }
    free(len);
    free(full);
    return total;
}

int oracle_mlem_f64(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                    const int32_t* sino, uint64_t S, int n_iter, double* image) {
    if (S != R) return -1;
    double* fw = (double*)malloc((size_t)R * sizeof(double) + 1);
    double* up = (double*)malloc((size_t)C * sizeof(double) + 1);
    double* norm = (double*)calloc((size_t)C + 1, sizeof(double));
    if (!fw || !up || !norm) { free(fw); free(up); free(norm); return -2; }
    for (uint32_t r = 0; r < R; ++r)
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            norm[e[k].index] += (double)e[k].value;
    double sumnorm = 0.0, sumin = 0.0;
    for (uint32_t i = 0; i < C; ++i) sumnorm += norm[i];
    for (uint64_t i = 0; i < S; ++i) sumin += sino[i];
    for (uint32_t i = 0; i < C; ++i) image[i] = sumin / sumnorm;
    for (int it = 0; it < n_iter; ++it) {
        for (uint32_t r = 0; r < R; ++r) {
            double res = 0.0;
            for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                res += (double)e[k].value * image[e[k].index];
            fw[r] = (res != 0.0) ? (double)sino[r] / res : 0.0;
        }
        memset(up, 0, (size_t)C * sizeof(double));
        for (uint32_t r = 0; r < R; ++r)
            for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                up[e[k].index] += (double)e[k].value * fw[r];
        for (uint32_t i = 0; i < C; ++i)
            image[i] *= (norm[i] != 0.0) ? (up[i] / norm[i]) : up[i];
    }
    free(fw); free(up); free(norm);
    return 0;
}

/*
 * The FP64 oracle above on several host threads, for matrices where the serial
 * loop takes minutes.  Rows are cut into n_threads contiguous blocks of about
 * equal element counts; each thread sums its rows' column sums and back
 * projection into a private double vector, and the vectors are added in
 * thread order.  The forward projection of a row is the same sequential
 * double sum as oracle_mlem_f64's; the column sums and back projection differ
 * from it only by the order of double additions (a few units in the last
 * place), and a fixed thread count gives the same image on every run.
 */
int oracle_mlem_f64_threads(uint32_t R, uint32_t C, const uint64_t* row_end,
                            const oracle_elem* e, const int32_t* sino, uint64_t S, int n_iter,
                            int n_threads, double* image) {
    if (S != R) return -1;
    if (n_threads < 1) n_threads = 1;
    if ((uint32_t)n_threads > R && R > 0) n_threads = (int)R;
    const int T = n_threads;
    double* fw = (double*)malloc((size_t)R * sizeof(double) + 1);
    double* norm = (double*)calloc((size_t)C + 1, sizeof(double));
    double* priv = (double*)malloc((size_t)T * (C + 1) * sizeof(double));
    uint32_t* cut = (uint32_t*)malloc((size_t)(T + 1) * sizeof(uint32_t));
    if (!fw || !norm || !priv || !cut) {
        free(fw); free(norm); free(priv); free(cut);
        return -2;
    }
    /* block t holds rows [cut[t], cut[t+1]): the first row whose END offset
     * reaches t/T of the elements starts block t */
    const uint64_t Z = R ? row_end[R - 1] : 0;
    cut[0] = 0;
    cut[T] = R;
    for (int t = 1; t < T; ++t) {
        const uint64_t want = Z / (uint64_t)T * (uint64_t)t;
        uint32_t lo = cut[t - 1], hi = R;
        while (lo < hi) {
            uint32_t mid = lo + (hi - lo) / 2;
            if (row_end[mid] < want) lo = mid + 1; else hi = mid;
        }
        cut[t] = lo;
    }
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        double* p = priv + (size_t)t * (C + 1);
        memset(p, 0, (size_t)C * sizeof(double));
        for (uint32_t r = cut[t]; r < cut[t + 1]; ++r)
            for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                p[e[k].index] += (double)e[k].value;
    }
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t i = 0; i < (int64_t)C; ++i) {
        double s = 0.0;
        for (int t = 0; t < T; ++t) s += priv[(size_t)t * (C + 1) + i];
        norm[i] = s;
    }
    double sumnorm = 0.0, sumin = 0.0;
    for (uint32_t i = 0; i < C; ++i) sumnorm += norm[i];
    for (uint64_t i = 0; i < S; ++i) sumin += sino[i];
    for (uint32_t i = 0; i < C; ++i) image[i] = sumin / sumnorm;
    for (int it = 0; it < n_iter; ++it) {
#pragma omp parallel for num_threads(T) schedule(static, 1)
        for (int t = 0; t < T; ++t) {
            for (uint32_t r = cut[t]; r < cut[t + 1]; ++r) {
                double res = 0.0;
                for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                    res += (double)e[k].value * image[e[k].index];
                fw[r] = (res != 0.0) ? (double)sino[r] / res : 0.0;
            }
            double* p = priv + (size_t)t * (C + 1);
            memset(p, 0, (size_t)C * sizeof(double));
            for (uint32_t r = cut[t]; r < cut[t + 1]; ++r)
                for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                    p[e[k].index] += (double)e[k].value * fw[r];
        }
#pragma omp parallel for num_threads(T) schedule(static)
        for (int64_t i = 0; i < (int64_t)C; ++i) {
            double u = 0.0;
            for (int t = 0; t < T; ++t) u += priv[(size_t)t * (C + 1) + i];
            image[i] *= (norm[i] != 0.0) ? (u / norm[i]) : u;
        }
    }
    free(fw); free(norm); free(priv); free(cut);
    return 0;
}

void oracle_mlem_relaxed_f64(uint32_t R, uint32_t C, const uint64_t* row_end,
                             const oracle_elem* e, const int32_t* sino, const double* x0,
                             const double* omega, int K, double* xK) {
    double* fw = (double*)malloc((size_t)R * sizeof(double) + 1);
    double* up = (double*)malloc((size_t)C * sizeof(double) + 1);
    double* norm = (double*)calloc((size_t)C + 1, sizeof(double));
    for (uint32_t r = 0; r < R; ++r)
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            norm[e[k].index] += (double)e[k].value;
    memcpy(xK, x0, (size_t)C * sizeof(double));
    for (int it = 0; it < K; ++it) {
        for (uint32_t r = 0; r < R; ++r) {
            double res = 0.0;
            for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                res += (double)e[k].value * xK[e[k].index];
            fw[r] = (res != 0.0) ? (double)sino[r] / res : 0.0;
        }
        memset(up, 0, (size_t)C * sizeof(double));
        for (uint32_t r = 0; r < R; ++r)
            for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
                up[e[k].index] += (double)e[k].value * fw[r];
        for (uint32_t i = 0; i < C; ++i) {
            double ratio = (norm[i] != 0.0) ? (up[i] / norm[i]) : up[i];
            xK[i] *= (ratio > 0.0) ? pow(ratio, omega[it]) : 0.0;
        }
    }
    free(fw); free(up); free(norm);
}

void oracle_project_f64(uint32_t R, const uint64_t* row_end, const oracle_elem* e,
                        const float* x, double* out) {
    for (uint32_t r = 0; r < R; ++r) {
        double s = 0.0;
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            s += (double)e[k].value * (double)x[e[k].index];
        out[r] = s;
    }
}

void oracle_poisson_grad_f64(uint32_t R, uint32_t C, const uint64_t* row_end,
                             const oracle_elem* e, const int32_t* s, const double* x,
                             double* grad) {
    memset(grad, 0, (size_t)C * sizeof(double));
    for (uint32_t r = 0; r < R; ++r) {
        double ax = 0.0;
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            ax += (double)e[k].value * x[e[k].index];
        /* d/dx [Ax - s log Ax] = A^T (1 - s / Ax); rows with Ax == 0 contribute A^T 1. */
        double w = (ax != 0.0) ? 1.0 - (double)s[r] / ax : 1.0;
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k)
            grad[e[k].index] += (double)e[k].value * w;
    }
}

void oracle_transpose(uint32_t R, uint32_t C, const uint64_t* row_end, const oracle_elem* e,
                      uint64_t* col_ptr, oracle_elem* ce) {
    memset(col_ptr, 0, ((size_t)C + 1) * sizeof(uint64_t));
    uint64_t Z = R ? row_end[R - 1] : 0;
    for (uint64_t k = 0; k < Z; ++k) col_ptr[e[k].index + 1] += 1;
    for (uint32_t c = 0; c < C; ++c) col_ptr[c + 1] += col_ptr[c];
    uint64_t* cursor = (uint64_t*)malloc(((size_t)C + 1) * sizeof(uint64_t));
    memcpy(cursor, col_ptr, ((size_t)C + 1) * sizeof(uint64_t));
    for (uint32_t r = 0; r < R; ++r)
        for (uint64_t k = row_begin(row_end, r); k < row_end[r]; ++k) {
            uint64_t slot = cursor[e[k].index]++;
            ce[slot].index = r;
            ce[slot].value = e[k].value;
        }
    free(cursor);
}

void oracle_partition(uint32_t R, const uint64_t* row_end, int n_ranks,
                      uint32_t* starts, uint32_t* ends) {
    /* mpicsr4mlem.cpp:206-224, including its float comparison of the running sum. */
    uint64_t Z = R ? row_end[R - 1] : 0;
    float avg = (float)Z / (float)n_ranks;
    int idx = 0;
    uint64_t sum = 0;
    for (int i = 0; i < n_ranks; ++i) { starts[i] = 0; ends[i] = 0; }
    starts[0] = 0;
    for (uint32_t r = 0; r < R; ++r) {
        sum += row_end[r] - row_begin(row_end, r);
        if ((float)sum > avg * (float)(idx + 1) && idx + 1 < n_ranks) {
            ends[idx] = r + 1;
            idx += 1;
            starts[idx] = r + 1;
        }
    }
    /* ranks the threshold never reached get empty ranges at the end */
    for (int i = idx + 1; i < n_ranks; ++i) starts[i] = R;
    for (int i = idx; i < n_ranks; ++i) ends[i] = R;
}
