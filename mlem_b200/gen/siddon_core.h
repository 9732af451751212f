/*
 * siddon_core.h -- synthetic PET system-matrix rows by Siddon ray marching.
 *
 * The reference ships no matrix generator (its README points to an external
 * one), so the synthetic workloads are defined here.  One row = one line of
 * response (LOR) between two points drawn uniformly on the lateral surface of
 * a cylinder around the voxel grid; its elements are {voxel index, float32
 * intersection length} for every voxel the line crosses, in ray order
 * (Siddon 1985, in the incremental form of Jacobs et al. 1998: step to the
 * nearest of the next x/y/z plane crossings).
 *
 * This header is compiled for the host (gcc, -ffp-contract=off) and for the
 * GPU (nvcc).  Every floating-point step is an IEEE-754 double operation with
 * round-to-nearest and no fused multiply-add (explicit __d*_rn intrinsics on
 * the device), and the random numbers come from a counter-based integer hash,
 * so both builds produce bit-identical matrices.
 *
 * Geometry (unit voxels): voxel (ix,iy,iz) covers [ix,ix+1)x[iy,iy+1)x[iz,iz+1),
 * its index is ix + nx*(iy + ny*iz), the grid spans [0,nx]x[0,ny]x[0,nz].
 * The cylinder's axis is the grid's z axis through (nx/2, ny/2); its radius is
 * radius_scale * max(nx,ny)/2 and endpoint z is uniform in [0, nz].  A LOR
 * whose element count falls outside [min_count, max_count] (a miss has count
 * 0) is redrawn; after SIDDON_MAX_ATTEMPTS draws the last non-empty one is
 * kept, and a row whose every draw missed stays empty.  The count window is
 * how a workload's "about lo-hi elements per row" is honoured.  Segments
 * shorter than min_len are dropped, so every stored value lies in
 * [min_len, sqrt(3)].
 */
#ifndef MLEM_SIDDON_CORE_H
#define MLEM_SIDDON_CORE_H

#include <stdint.h>

#if defined(__CUDACC__)
#define SD_FN __host__ __device__ __forceinline__
#else
#define SD_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define SD_MUL(a, b) __dmul_rn((a), (b))
#define SD_ADD(a, b) __dadd_rn((a), (b))
#define SD_SUB(a, b) __dsub_rn((a), (b))
#define SD_DIV(a, b) __ddiv_rn((a), (b))
#define SD_SQRT(a) __dsqrt_rn(a)
#define SD_FLOOR(a) floor(a)
#define SD_CEIL(a) ceil(a)
#else
#include <math.h>
#define SD_MUL(a, b) ((a) * (b))
#define SD_ADD(a, b) ((a) + (b))
#define SD_SUB(a, b) ((a) - (b))
#define SD_DIV(a, b) ((a) / (b))
#define SD_SQRT(a) sqrt(a)
#define SD_FLOOR(a) floor(a)
#define SD_CEIL(a) ceil(a)
#endif

#define SIDDON_MAX_ATTEMPTS 64
#define SIDDON_DEFAULT_MIN_LEN 1.0e-4

typedef struct {
    uint32_t nx, ny, nz;
    uint32_t min_count;  /* accepted element-count window of a row */
    uint32_t max_count;
    uint32_t pad_;
    double radius_scale; /* cylinder radius / grid half-width; 1.2 for the standard workloads */
    double min_len;      /* shortest stored segment, in voxel units */
    uint64_t seed;
} siddon_geom;

/* splitmix64 output function (Steele, Lea, Flood 2014). */
SD_FN uint64_t sd_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* k-th uniform double in [0,1) of stream `key` (53 random bits). */
SD_FN double sd_uniform(uint64_t key, uint32_t k) {
    uint64_t h = sd_mix64(key ^ sd_mix64(0xD1B54A32D192ED03ull * (uint64_t)(k + 1)));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

SD_FN uint64_t sd_stream(uint64_t seed, uint32_t row, uint32_t attempt, uint32_t endpoint) {
    return sd_mix64(seed ^ sd_mix64(((uint64_t)row << 8) | ((uint64_t)attempt << 1) | endpoint));
}

/* Uniform point on the cylinder surface: uniform angle by rejection from the
 * square (no trigonometry, so host and device agree), uniform z. */
SD_FN void sd_endpoint(const siddon_geom* g, uint64_t key, double* p) {
    double half = 0.5 * (double)(g->nx > g->ny ? g->nx : g->ny);
    double radius = SD_MUL(g->radius_scale, half);
    double u = 1.0, v = 0.0, q = 1.0;
    for (uint32_t t = 0; t < 64; ++t) {
        double a = SD_SUB(SD_MUL(2.0, sd_uniform(key, 2 * t)), 1.0);
        double b = SD_SUB(SD_MUL(2.0, sd_uniform(key, 2 * t + 1)), 1.0);
        double qq = SD_ADD(SD_MUL(a, a), SD_MUL(b, b));
        if (qq > 1.0e-12 && qq <= 1.0) { u = a; v = b; q = qq; break; }
    }
    double s = SD_DIV(radius, SD_SQRT(q));
    p[0] = SD_ADD(0.5 * (double)g->nx, SD_MUL(u, s));
    p[1] = SD_ADD(0.5 * (double)g->ny, SD_MUL(v, s));
    p[2] = SD_MUL((double)g->nz, sd_uniform(key, 200));
}

/*
 * Trace one LOR (p0 -> p1).  When `out` is non-null the elements are written
 * there as interleaved 32-bit words {voxel index, float32 length bits}, the
 * CSR4 element layout (capacity nx+ny+nz+4 elements).  Returns the number of
 * elements.
 */
SD_FN uint32_t sd_f32_bits(float f) {
    union { float f; uint32_t u; } cv;
    cv.f = f;
    return cv.u;
}

SD_FN uint32_t sd_trace(const siddon_geom* g, const double* p0, const double* p1,
                        uint32_t* out) {
    const double n[3] = {(double)g->nx, (double)g->ny, (double)g->nz};
    double d[3];
    double amin = 0.0, amax = 1.0;
    for (int i = 0; i < 3; ++i) {
        d[i] = SD_SUB(p1[i], p0[i]);
        if (d[i] != 0.0) {
            double lo = SD_DIV(SD_SUB(0.0, p0[i]), d[i]);
            double hi = SD_DIV(SD_SUB(n[i], p0[i]), d[i]);
            if (lo > hi) { double t = lo; lo = hi; hi = t; }
            if (lo > amin) amin = lo;
            if (hi < amax) amax = hi;
        } else if (p0[i] < 0.0 || p0[i] > n[i]) {
            return 0;
        }
    }
    if (!(amin < amax)) return 0;
    double len2 = SD_ADD(SD_ADD(SD_MUL(d[0], d[0]), SD_MUL(d[1], d[1])), SD_MUL(d[2], d[2]));
    double L = SD_SQRT(len2);

    int32_t idx[3], step[3];
    double anext[3];
    for (int i = 0; i < 3; ++i) {
        double pos = SD_ADD(p0[i], SD_MUL(amin, d[i]));
        int32_t k;
        if (d[i] > 0.0) { k = (int32_t)SD_FLOOR(pos); step[i] = 1; }
        else if (d[i] < 0.0) { k = (int32_t)SD_CEIL(pos) - 1; step[i] = -1; }
        else { k = (int32_t)SD_FLOOR(pos); step[i] = 0; }
        int32_t hiidx = (int32_t)(i == 0 ? g->nx : (i == 1 ? g->ny : g->nz)) - 1;
        if (k < 0) k = 0;
        if (k > hiidx) k = hiidx;
        idx[i] = k;
        if (step[i] > 0) anext[i] = SD_DIV(SD_SUB((double)(k + 1), p0[i]), d[i]);
        else if (step[i] < 0) anext[i] = SD_DIV(SD_SUB((double)k, p0[i]), d[i]);
        else anext[i] = 2.0; /* never crosses a plane of this axis: beyond amax <= 1 */
    }

    uint32_t count = 0;
    double cur = amin;
    uint32_t max_steps = g->nx + g->ny + g->nz + 4;
    for (uint32_t it = 0; it < max_steps; ++it) {
        int ax = 0;
        double an = anext[0];
        if (anext[1] < an) { an = anext[1]; ax = 1; }
        if (anext[2] < an) { an = anext[2]; ax = 2; }
        int last = 0;
        if (an >= amax) { an = amax; last = 1; }
        double len = SD_MUL(SD_SUB(an, cur), L);
        if (len >= g->min_len) {
            if (out) {
                out[2 * count] = (uint32_t)idx[0] +
                                 g->nx * ((uint32_t)idx[1] + g->ny * (uint32_t)idx[2]);
                out[2 * count + 1] = sd_f32_bits((float)len);
            }
            ++count;
        }
        if (last) break;
        idx[ax] += step[ax];
        int32_t hiidx = (int32_t)(ax == 0 ? g->nx : (ax == 1 ? g->ny : g->nz)) - 1;
        if (idx[ax] < 0 || idx[ax] > hiidx) break;
        if (step[ax] > 0) anext[ax] = SD_DIV(SD_SUB((double)(idx[ax] + 1), p0[ax]), d[ax]);
        else anext[ax] = SD_DIV(SD_SUB((double)idx[ax], p0[ax]), d[ax]);
        if (an > cur) cur = an;
    }
    return count;
}

/* Row generator: draws LORs for `row` until one has an accepted element
 * count, then traces it once more into `out` (when non-null). */
SD_FN uint32_t sd_row(const siddon_geom* g, uint32_t row, uint32_t* out) {
    int32_t keep = -1;
    for (uint32_t a = 0; a < SIDDON_MAX_ATTEMPTS; ++a) {
        double p0[3], p1[3];
        sd_endpoint(g, sd_stream(g->seed, row, a, 0), p0);
        sd_endpoint(g, sd_stream(g->seed, row, a, 1), p1);
        uint32_t c = sd_trace(g, p0, p1, 0);
        if (c > 0) keep = (int32_t)a;
        if (c > 0 && c >= g->min_count && c <= g->max_count) break;
    }
    if (keep < 0) return 0;
    double p0[3], p1[3];
    sd_endpoint(g, sd_stream(g->seed, row, (uint32_t)keep, 0), p0);
    sd_endpoint(g, sd_stream(g->seed, row, (uint32_t)keep, 1), p1);
    return sd_trace(g, p0, p1, out);
}

SD_FN uint32_t sd_row_capacity(const siddon_geom* g) { return g->nx + g->ny + g->nz + 4; }

#endif /* MLEM_SIDDON_CORE_H */
