/*
 * siddon_host.c -- host build of the synthetic Siddon matrix generator
 * (libmlem_gen.so).  The CUDA library builds the same rows on the device from
 * the same siddon_core.h; both must agree bit for bit.
 *
 * Compiled with -ffp-contract=off (no fused multiply-add), OpenMP over rows.
 */
#include <stdint.h>
#include <stdlib.h>

#include "siddon_core.h"

#define GEN_API __attribute__((visibility("default")))

static siddon_geom make_geom(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t min_count,
                             uint32_t max_count, double radius_scale, double min_len,
                             uint64_t seed) {
    siddon_geom g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.pad_ = 0;
    g.min_count = min_count;
    g.max_count = max_count;
    g.radius_scale = radius_scale;
    g.min_len = min_len;
    g.seed = seed;
    return g;
}

/* Number of elements of every row; returns the total. */
GEN_API uint64_t mlem_gen_siddon_counts(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t R,
                                        uint32_t min_count, uint32_t max_count,
                                        double radius_scale, double min_len, uint64_t seed,
                                        uint32_t* counts) {
    siddon_geom g = make_geom(nx, ny, nz, min_count, max_count, radius_scale, min_len, seed);
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : total)
    for (int64_t r = 0; r < (int64_t)R; ++r) {
        counts[r] = sd_row(&g, (uint32_t)r, 0);
        total += counts[r];
    }
    return total;
}

/* Fill the CSR4 element array (8 bytes per element: uint32 voxel, float32 length)
 * given the row END offsets produced from the counts. */
GEN_API int mlem_gen_siddon_fill(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t R,
                                 uint32_t min_count, uint32_t max_count,
                                 double radius_scale, double min_len, uint64_t seed,
                                 const uint64_t* row_end, void* elems) {
    siddon_geom g = make_geom(nx, ny, nz, min_count, max_count, radius_scale, min_len, seed);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t r = 0; r < (int64_t)R; ++r) {
        uint64_t begin = r == 0 ? 0 : row_end[r - 1];
        uint32_t expect = (uint32_t)(row_end[r] - begin);
        /* count first: never write past the slot the counts pass reserved */
        if (sd_row(&g, (uint32_t)r, 0) != expect) { bad = 1; continue; }
        sd_row(&g, (uint32_t)r, (uint32_t*)elems + 2 * begin);
    }
    return bad ? -1 : 0;
}

/* Sequential double projection of one image through every row,
 * out[r] = sum_k (double)value_k * (double)x[column_k] in element order with
 * no fused multiply-add: the sinogram means of the synthetic workloads.  The
 * CUDA library computes the same sums on the device bit for bit. */
GEN_API void mlem_gen_project_f64(uint32_t R, const uint64_t* row_end, const void* elems,
                                  const float* x, double* out) {
    const uint32_t* e = (const uint32_t*)elems;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t r = 0; r < (int64_t)R; ++r) {
        uint64_t begin = r == 0 ? 0 : row_end[r - 1];
        double s = 0.0;
        for (uint64_t k = begin; k < row_end[r]; ++k) {
            union { uint32_t u; float f; } cv;
            cv.u = e[2 * k + 1];
            s += (double)cv.f * (double)x[e[2 * k]];
        }
        out[r] = s;
    }
}
