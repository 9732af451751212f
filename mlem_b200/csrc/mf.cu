// mf.cu -- matrix-free MLEM on the synthetic Siddon geometry (prototype).
//
// The stored-matrix path streams every element {voxel, length} from HBM once
// per iteration (8 bytes each, 6.2 GB on the 128x128x64 workload).  Here the
// matrix is never stored: a ray (one LOR, one row) is kept as a 104-byte
// descriptor -- entry point, direction, its inverse, the alpha range inside
// the grid and the length -- and its elements are traced again in every pass
// (Siddon 1985 in the incremental form of Jacobs et al. 1998, the generator
// of mlem_b200/gen/siddon_core.h).
//
// A warp traces one ray: lane j walks the j-th of 32 equal alpha intervals
// of the ray (a voxel cut by an interval boundary gives two elements, one per
// lane) once, keeping its elements in its own shared-memory slots; the
// forward sum (four gathers in flight per lane), calcCorrel and the scatter
// replay those slots.  Each lane's interval starts in double from the
// generator's accepted line (entry point, direction and alpha range computed
// with the generator's own code) and steps in float in the interval's local
// parameter, so the traced lengths equal the stored ones to about 1e-6.
// Rays whose counts are zero are skipped, as calcCorrel makes their
// contribution 0.  The kernel is bound by instruction issue (the walk), not
// by memory.
//
// The descriptors are sorted like the stored rows (Morton interleave of the
// entry and exit voxels), and voxels use the stored path's Morton device
// order.  One frame; the summation order of the atomics varies run to run.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "mlem_b200.h"
#include "host/errors.hpp"
#include "siddon_core.h"

using namespace mlem;

struct MfRay {
    double p0[3];    // entry-draw endpoint (the line's origin, alpha = 0)
    double d[3];     // direction p1 - p0
    double invd[3];  // 1 / d (0 on an axis the line does not move along)
    double a0, a1;   // alpha range inside the grid (a0 == a1: the ray misses it)
    double L;        // |d|: element length = alpha span * L
    uint32_t row;    // the ray's row (sinogram index)
    uint32_t pad;
};

struct MfGrid {
    int32_t n[3];
    const uint32_t* perm;  // natural -> device voxel (ranked Morton), non-power-of-two grids
    int pow2;              // device index = dil[ix] | dil[nx + iy] | dil[nx + ny + iz]
};

struct mlem_mf {
    int device = 0;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    uint32_t R = 0, C = 0;
    uint32_t grid[3] = {0, 0, 0};
    uint32_t cap = 0;  // elements a lane's interval can hold
    MfRay* rays = nullptr;
    uint32_t* perm = nullptr;
    uint32_t* dil = nullptr;  // nx + ny + nz Morton parts (power-of-two grids)
    bool pow2 = false;
    std::vector<uint32_t> perm_host;
    float* norm = nullptr;
    float* x = nullptr;
    float* u = nullptr;
    int32_t* sino = nullptr;
    unsigned int* flag = nullptr;
    std::vector<float> norm_nat;
    double sumnorm = 0.0, sumin = 0.0;
    bool have_sino = false, have_image = false;
    uint64_t device_bytes = 0;
};

namespace {

constexpr int kMfThreads = 256;
constexpr int kMfWarps = kMfThreads / 32;
// Slot t of lane j sits at word j + kMfStride * t of its warp's arrays: the
// walk's writes (one slot of every lane) and the gathers' reads (eight slots
// of four neighbouring lanes, bank (j + 4 t) mod 32) hit 32 different banks.
constexpr int kMfStride = 36;

__device__ __forceinline__ uint32_t mf_voxel(const MfGrid& g, const uint32_t* dil, const int32_t (&i)[3]) {
    if (g.pow2) return dil[i[0]] | dil[g.n[0] + i[1]] | dil[g.n[0] + g.n[1] + i[2]];
    return g.perm[(uint32_t)i[0] + (uint32_t)g.n[0] * ((uint32_t)i[1] + (uint32_t)g.n[1] * (uint32_t)i[2])];
}

// Per-axis state of a walk, in the lane's local parameter t = alpha - A
// (t <= 1/32 of the ray): voxel index, step, and the next plane crossing at
// t = (dist + k) * dt, with dist the distance from the start point to the
// first plane ahead, k the planes crossed since, dt = |1 / d|.  The start is
// found in double; the steps are float products of small numbers, so a
// crossing is placed to about 1e-6 voxel (float accumulation of dt would
// drift by the step count).
struct MfAxis {
    int32_t i, step, n, k;
    float dist, dt, tn;
    __device__ __forceinline__ void start(double p0, double d, double invd, double A, int32_t n_) {
        n = n_;
        k = 0;
        const double pos = __dadd_rn(p0, __dmul_rn(A, d));
        int32_t v;
        double gap;
        if (d > 0.0) { v = (int32_t)floor(pos); step = 1; }
        else if (d < 0.0) { v = (int32_t)ceil(pos) - 1; step = -1; }
        else { v = (int32_t)floor(pos); step = 0; }
        i = v < 0 ? 0 : (v >= n ? n - 1 : v);
        if (step > 0) gap = __dsub_rn((double)(i + 1), pos);
        else if (step < 0) gap = __dsub_rn(pos, (double)i);
        else gap = 0.0;
        dist = (float)gap;
        dt = step ? (float)fabs(invd) : 0.0f;
        tn = step ? __fmul_rn(dist, dt) : 4.0f;  // 4 > any t (t <= 1): never crossed
    }
    // cross the next plane; false when the walk leaves the grid
    __device__ __forceinline__ bool advance() {
        i += step;
        if (i < 0 || i >= n) return false;
        ++k;
        tn = __fmul_rn(__fadd_rn(dist, (float)k), dt);
        return true;
    }
};

__device__ __forceinline__ uint32_t mf_voxel3(const MfGrid& g, const uint32_t* dil, int32_t x,
                                              int32_t y, int32_t z) {
    if (g.pow2) return dil[x] | dil[g.n[0] + y] | dil[g.n[0] + g.n[1] + z];
    return g.perm[(uint32_t)x + (uint32_t)g.n[0] * ((uint32_t)y + (uint32_t)g.n[1] * (uint32_t)z)];
}

// The elements of a ray inside a lane's interval, from the axis states at
// its start, T = its length in alpha, L = |d|: counted (WRITE false) or
// written to vox[0 .. count) / lens[0 .. count).  At most `cap` elements; a
// longer walk sets *over and stops (the bound of the interval length keeps
// it unreached).
template <bool WRITE>
__device__ __forceinline__ uint32_t mf_walk(MfAxis X, MfAxis Y, MfAxis Z, float T, float L,
                                            const MfGrid& g, const uint32_t* dil, uint32_t* vox,
                                            float* lens, uint32_t cap, bool* over) {
    if (!(T > 0.0f)) return 0;
    float cur = 0.0f;
    uint32_t cnt = 0;
    const uint32_t max_it = 3 * cap + 8;
    for (uint32_t it = 0;; ++it) {
        if (it == max_it) { *over = true; break; }
        const float t_min = fminf(X.tn, fminf(Y.tn, Z.tn));
        const bool last = t_min >= T;
        const float t = last ? T : t_min;
        const float len = __fmul_rn(__fsub_rn(t, cur), L);
        if (len > 0.0f) {
            if (cnt == cap) { *over = true; break; }
            if (WRITE) {
                vox[kMfStride * cnt] = mf_voxel3(g, dil, X.i, Y.i, Z.i);
                lens[kMfStride * cnt] = len;
            }
            ++cnt;
        }
        if (last) break;
        // the axis whose plane comes first (x before y before z on a tie)
        bool inside;
        if (X.tn == t_min) inside = X.advance();
        else if (Y.tn == t_min) inside = Y.advance();
        else inside = Z.advance();
        if (!inside) break;
        if (t > cur) cur = t;
    }
    return cnt;
}

// Lane `lane` traces its 1/32 of ray r into its own slots vox[0 .. n) /
// lens[0 .. n) (slot t of lane j at j + kMfStride t in the warp's arrays);
// returns n.
__device__ __forceinline__ uint32_t mf_trace_lane(const MfRay& r, const MfGrid& g, const uint32_t* dil,
                                                  uint32_t* vox, float* lens, uint32_t cap, int lane,
                                                  bool* over) {
    const double span = __dsub_rn(r.a1, r.a0);
    const double A = __dadd_rn(r.a0, __dmul_rn(span, (double)lane * (1.0 / 32.0)));
    const double Aend = lane == 31 ? r.a1 : __dadd_rn(r.a0, __dmul_rn(span, (double)(lane + 1) * (1.0 / 32.0)));
    MfAxis X, Y, Z;
    X.start(r.p0[0], r.d[0], r.invd[0], A, g.n[0]);
    Y.start(r.p0[1], r.d[1], r.invd[1], A, g.n[1]);
    Z.start(r.p0[2], r.d[2], r.invd[2], A, g.n[2]);
    const float T = Aend > A ? (float)__dsub_rn(Aend, A) : 0.0f, L = (float)r.L;
    return mf_walk<true>(X, Y, Z, T, L, g, dil, vox, lens, cap, over);
}

__device__ __forceinline__ void load_dil(const MfGrid& g, const uint32_t* dil_g, uint32_t* dil_s) {
    if (g.pow2)
        for (int i = threadIdx.x; i < g.n[0] + g.n[1] + g.n[2]; i += blockDim.x) dil_s[i] = dil_g[i];
    __syncthreads();
}

// One pass per ray: forward projection, calcCorrel, scatter into u.
__global__ void __launch_bounds__(kMfThreads, 4) k_mf_fused(const MfRay* __restrict__ rays, uint32_t n,
                                                         MfGrid g, const uint32_t* __restrict__ dil_g,
                                                         uint32_t cap, const float* __restrict__ x,
                                                         const int32_t* __restrict__ sino,
                                                         float* __restrict__ u,
                                                         unsigned int* __restrict__ flag) {
    extern __shared__ uint32_t smem[];
    const size_t per_warp = (size_t)kMfStride * cap;
    uint32_t* dil = smem + (size_t)kMfWarps * 2 * per_warp;
    load_dil(g, dil_g, dil);
    const int lane = threadIdx.x & 31;
    uint32_t* wvox = smem + (size_t)(threadIdx.x >> 5) * 2 * per_warp;
    float* wlens = reinterpret_cast<float*>(wvox + per_warp);
    // the gathers and the scatter read the slots across lanes: lane i takes
    // slot r0 + (i & 7) of lane 4 q + (i >> 3) in step q, so one instruction
    // covers about 32 consecutive elements of the ray (four neighbouring
    // intervals), and its sectors are shared as in the stored walk
    const int sub = lane & 7, grp = lane >> 3;
    const uint64_t ph = l2_evict_last();
    bool over = false;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = warp; k < n; k += nwarps) {
        if (lane < 2 && k + nwarps < n)  // the next ray's descriptor, two 128-byte lines
            asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char*>(rays + k + nwarps) + 64 * lane));
        const MfRay r = rays[k];
        const int32_t s = sino[r.row];
        if (s == 0 || !(r.a1 > r.a0)) continue;  // calcCorrel 0: nothing to scatter
        const uint32_t cnt = mf_trace_lane(r, g, dil, wvox + lane, wlens + lane, cap, lane, &over);
        __syncwarp();  // every lane's slots are written
        uint32_t mx = cnt;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(MLEM_FULL_MASK, mx, o));
        uint32_t oc[8];  // the slot counts of the lanes this lane reads from
#pragma unroll
        for (int q = 0; q < 8; ++q) oc[q] = __shfl_sync(MLEM_FULL_MASK, cnt, 4 * q + grp);
        float acc = 0.0f;
        for (uint32_t r0 = 0; r0 < mx; r0 += 8) {
            const uint32_t t = r0 + sub;
            float xv[8], lv[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t w = 4 * q + grp + kMfStride * t;
                const bool ok = t < oc[q];
                lv[q] = ok ? wlens[w] : 0.0f;
                xv[q] = ok ? ld_hot(x + wvox[w], ph) : 0.0f;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) acc = fmaf(lv[q], xv[q], acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MLEM_FULL_MASK, acc, o);
        const float c = correl_of(s, acc);
        if (c != 0.0f)
            for (uint32_t r0 = 0; r0 < mx; r0 += 8) {
                const uint32_t t = r0 + sub;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const uint32_t w = 4 * q + grp + kMfStride * t;
                    if (t < oc[q]) atomicAdd(u + wvox[w], wlens[w] * c);
                }
            }
        __syncwarp();  // the slots are read before the next ray's walk
    }
    if (over) atomicOr(flag, 1u);
}

// Column sums: every ray's lengths added into norm (device voxel order).
__global__ void __launch_bounds__(kMfThreads, 4) k_mf_colsum(const MfRay* __restrict__ rays, uint32_t n,
                                                          MfGrid g, const uint32_t* __restrict__ dil_g,
                                                          uint32_t cap, float* __restrict__ norm,
                                                          unsigned int* __restrict__ flag) {
    extern __shared__ uint32_t smem[];
    const size_t per_warp = (size_t)kMfStride * cap;
    uint32_t* dil = smem + (size_t)kMfWarps * 2 * per_warp;
    load_dil(g, dil_g, dil);
    const int lane = threadIdx.x & 31;
    uint32_t* vox = smem + (size_t)(threadIdx.x >> 5) * 2 * per_warp + lane;
    float* lens = reinterpret_cast<float*>(vox + per_warp);
    bool over = false;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = warp; k < n; k += nwarps) {
        const MfRay r = rays[k];
        if (!(r.a1 > r.a0)) continue;
        const uint32_t cnt = mf_trace_lane(r, g, dil, vox, lens, cap, lane, &over);
        for (uint32_t t = 0; t < cnt; ++t) atomicAdd(norm + vox[kMfStride * t], lens[kMfStride * t]);
        __syncwarp();
    }
    if (over) atomicOr(flag, 1u);
}

__device__ __forceinline__ uint64_t spread2(uint32_t v) {
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

// Voxel of the line at alpha a (direction-aware at a plane), clamped to the grid.
__device__ __forceinline__ void mf_voxel_at(const MfRay& r, double a, const MfGrid& g, int32_t (&i)[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double pos = r.p0[k] + a * r.d[k];
        int32_t v = r.d[k] < 0.0 ? (int32_t)ceil(pos) - 1 : (int32_t)floor(pos);
        i[k] = v < 0 ? 0 : (v >= g.n[k] ? g.n[k] - 1 : v);
    }
}

// Thread per row: the generator's accepted draw (sd_row's attempt loop), its
// descriptor and its sort key (Morton interleave of entry and exit voxels).
__global__ void k_mf_rays(siddon_geom sg, uint32_t R, MfGrid g, const uint32_t* __restrict__ dil,
                          MfRay* __restrict__ rays, uint64_t* __restrict__ key,
                          uint32_t* __restrict__ idx) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < R;
         r += (uint64_t)gridDim.x * blockDim.x) {
        int32_t keep = -1;
        for (uint32_t a = 0; a < SIDDON_MAX_ATTEMPTS; ++a) {
            double p0[3], p1[3];
            sd_endpoint(&sg, sd_stream(sg.seed, (uint32_t)r, a, 0), p0);
            sd_endpoint(&sg, sd_stream(sg.seed, (uint32_t)r, a, 1), p1);
            const uint32_t c = sd_trace(&sg, p0, p1, nullptr);
            if (c > 0) keep = (int32_t)a;
            if (c > 0 && c >= sg.min_count && c <= sg.max_count) break;
        }
        MfRay ray;
        ray.row = (uint32_t)r;
        ray.pad = 0;
        ray.a0 = ray.a1 = 0.0;
        uint64_t k = ~0ull;  // rays that miss the grid last
        double p0[3] = {0, 0, 0}, p1[3] = {0, 0, 0};
        if (keep >= 0) {
            sd_endpoint(&sg, sd_stream(sg.seed, (uint32_t)r, (uint32_t)keep, 0), p0);
            sd_endpoint(&sg, sd_stream(sg.seed, (uint32_t)r, (uint32_t)keep, 1), p1);
        }
        const double n[3] = {(double)sg.nx, (double)sg.ny, (double)sg.nz};
        double amin = 0.0, amax = 1.0;
        bool miss = keep < 0;
        for (int i = 0; i < 3; ++i) {  // the clipping of sd_trace
            ray.p0[i] = p0[i];
            ray.d[i] = SD_SUB(p1[i], p0[i]);
            ray.invd[i] = ray.d[i] != 0.0 ? SD_DIV(1.0, ray.d[i]) : 0.0;
            if (ray.d[i] != 0.0) {
                double lo = SD_DIV(SD_SUB(0.0, p0[i]), ray.d[i]);
                double hi = SD_DIV(SD_SUB(n[i], p0[i]), ray.d[i]);
                if (lo > hi) { const double t = lo; lo = hi; hi = t; }
                if (lo > amin) amin = lo;
                if (hi < amax) amax = hi;
            } else if (p0[i] < 0.0 || p0[i] > n[i]) {
                miss = true;
            }
        }
        if (!(amin < amax)) miss = true;
        ray.L = SD_SQRT(SD_ADD(SD_ADD(SD_MUL(ray.d[0], ray.d[0]), SD_MUL(ray.d[1], ray.d[1])),
                               SD_MUL(ray.d[2], ray.d[2])));
        if (!miss) {
            ray.a0 = amin;
            ray.a1 = amax;
            int32_t ie[3], ix[3];
            mf_voxel_at(ray, amin, g, ie);
            // exit voxel: the last voxel before amax
            const double back = amax - (amax - amin) * 1e-9;
            mf_voxel_at(ray, back, g, ix);
            const uint32_t va = mf_voxel(g, dil, ie), vb = mf_voxel(g, dil, ix);
            const uint32_t lo = va < vb ? va : vb, hi = va < vb ? vb : va;
            k = (spread2(hi) << 1) | spread2(lo);
        }
        rays[r] = ray;
        key[r] = k;
        idx[r] = (uint32_t)r;
    }
}

__global__ void k_mf_gather(const MfRay* __restrict__ in, const uint32_t* __restrict__ order, uint32_t n,
                            MfRay* __restrict__ out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n;
         k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = in[order[k]];
}

__global__ void k_mf_fill(float* __restrict__ x, uint32_t n, float v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        x[i] = v;
}

int mf_fail(int status, const char* what, cudaError_t e) {
    cudaGetLastError();
    return set_error(nullptr, status, "%s: %s", what, cudaGetErrorString(e));
}

#define MF_CK(what, call)                                                          \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess)                                                     \
            return mf_fail(e_ == cudaErrorMemoryAllocation ? MLEM_ERR_NOMEM : MLEM_ERR_CUDA, \
                           what, e_);                                              \
    } while (0)

template <typename T>
cudaError_t mf_alloc(mlem_mf* m, T** p, size_t count) {
    const size_t b = std::max<size_t>(count * sizeof(T), 256);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), b);
    if (e == cudaSuccess) m->device_bytes += b;
    return e;
}

MfGrid grid_of(const mlem_mf* m) {
    MfGrid g;
    for (int i = 0; i < 3; ++i) g.n[i] = (int32_t)m->grid[i];
    g.perm = m->perm;
    g.pow2 = m->pow2 ? 1 : 0;
    return g;
}

size_t mf_smem(const mlem_mf* m) {
    // per warp: 32 lanes x cap slots of a voxel and a length, then the Morton parts
    return (size_t)kMfWarps * 2 * kMfStride * m->cap * 4 + (size_t)(m->grid[0] + m->grid[1] + m->grid[2]) * 4;
}

int mf_check_flag(mlem_mf* m) {
    unsigned int f = 0;
    MF_CK("matrix-free flag", cudaMemcpyAsync(&f, m->flag, 4, cudaMemcpyDeviceToHost, m->stream));
    MF_CK("matrix-free sync", cudaStreamSynchronize(m->stream));
    if (f)
        return set_error(nullptr, MLEM_ERR_CUDA,
                         "matrix-free walk: a lane's interval held more elements than its bound");
    return MLEM_OK;
}

}  // namespace

extern "C" {

int mlem_mf_create_siddon(mlem_mf** out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t n_rows,
                          uint32_t min_count, uint32_t max_count, double radius_scale,
                          double min_len, uint64_t seed, int device) {
    if (!out) return set_error(nullptr, MLEM_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!nx || !ny || !nz) return set_error(nullptr, MLEM_ERR_INVALID, "empty voxel grid");
    const uint64_t C64 = (uint64_t)nx * ny * nz;
    if (C64 > 0xffffffffull || nx > 0x7fffffffu || ny > 0x7fffffffu || nz > 0x7fffffffu)
        return set_error(nullptr, MLEM_ERR_INVALID, "grid has more than 2^32 voxels");
    if (!(min_len > 0.0)) return set_error(nullptr, MLEM_ERR_INVALID, "min_len must be > 0");
    MF_CK("cudaSetDevice", cudaSetDevice(device));
    mlem_mf* m = new mlem_mf;
    m->device = device;
    m->R = n_rows;
    m->C = (uint32_t)C64;
    m->grid[0] = nx;
    m->grid[1] = ny;
    m->grid[2] = nz;
    // per-lane element bound: an interval of length l (<= diagonal / 32) crosses
    // at most l * sqrt(3) + 3 planes
    const double diag = std::sqrt((double)nx * nx + (double)ny * ny + (double)nz * nz);
    m->cap = (uint32_t)std::ceil(diag * std::sqrt(3.0) / 32.0) + 6;
    auto bail = [&](int s) { mlem_mf_destroy(m); return s; };
    cudaError_t e = cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(mf_fail(MLEM_ERR_CUDA, "stream", e));
    m->stream = m->own_stream;
    // device voxel order, and its per-axis parts when every dimension is a power of two
    voxel_permutation(nx, ny, nz, m->perm_host);
    m->pow2 = (nx & (nx - 1)) == 0 && (ny & (ny - 1)) == 0 && (nz & (nz - 1)) == 0;
    std::vector<uint32_t> dil(nx + ny + nz, 0);
    if (m->pow2) {
        for (uint32_t i = 0; i < nx; ++i) dil[i] = m->perm_host[i];
        for (uint32_t i = 0; i < ny; ++i) dil[nx + i] = m->perm_host[(size_t)nx * i];
        for (uint32_t i = 0; i < nz; ++i) dil[nx + ny + i] = m->perm_host[(size_t)nx * ny * i];
    }
    if ((e = mf_alloc(m, &m->perm, m->C)) != cudaSuccess ||
        (e = mf_alloc(m, &m->dil, dil.size())) != cudaSuccess ||
        (e = mf_alloc(m, &m->rays, std::max<uint32_t>(n_rows, 1))) != cudaSuccess ||
        (e = mf_alloc(m, &m->norm, m->C)) != cudaSuccess ||
        (e = mf_alloc(m, &m->x, m->C)) != cudaSuccess ||
        (e = mf_alloc(m, &m->u, m->C)) != cudaSuccess ||
        (e = mf_alloc(m, &m->sino, std::max<uint32_t>(n_rows, 1))) != cudaSuccess ||
        (e = mf_alloc(m, &m->flag, 1)) != cudaSuccess)
        return bail(mf_fail(MLEM_ERR_NOMEM, "matrix-free buffers", e));
    MfRay* tmp = nullptr;
    uint64_t *key = nullptr, *key_s = nullptr;
    uint32_t *idx = nullptr, *order = nullptr;
    void* sort_tmp = nullptr;
    auto release = [&]() {
        for (void* p : {(void*)tmp, (void*)key, (void*)key_s, (void*)idx, (void*)order, sort_tmp})
            if (p) cudaFree(p);
    };
    const uint32_t Rn = std::max<uint32_t>(n_rows, 1);
    do {
        if ((e = cudaMemcpyAsync(m->perm, m->perm_host.data(), (size_t)m->C * 4,
                                 cudaMemcpyHostToDevice, m->stream)) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(m->dil, dil.data(), dil.size() * 4, cudaMemcpyHostToDevice,
                                 m->stream)) != cudaSuccess) break;
        if ((e = cudaMalloc(&tmp, (size_t)Rn * sizeof(MfRay))) != cudaSuccess) break;
        if ((e = cudaMalloc(&key, (size_t)Rn * 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&key_s, (size_t)Rn * 8)) != cudaSuccess) break;
        if ((e = cudaMalloc(&idx, (size_t)Rn * 4)) != cudaSuccess) break;
        if ((e = cudaMalloc(&order, (size_t)Rn * 4)) != cudaSuccess) break;
        siddon_geom sg;
        sg.nx = nx; sg.ny = ny; sg.nz = nz; sg.pad_ = 0;
        sg.min_count = min_count;
        sg.max_count = max_count;
        sg.radius_scale = radius_scale;
        sg.min_len = min_len;
        sg.seed = seed;
        const MfGrid g = grid_of(m);
        if (n_rows) {
            k_mf_rays<<<kB200SMs * 16, 128, 0, m->stream>>>(sg, n_rows, g, m->dil, tmp, key, idx);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
            size_t sb = 0;
            if ((e = cub::DeviceRadixSort::SortPairs(nullptr, sb, key, key_s, idx, order, (int)n_rows,
                                                     0, 64, m->stream)) != cudaSuccess) break;
            if ((e = cudaMalloc(&sort_tmp, sb)) != cudaSuccess) break;
            if ((e = cub::DeviceRadixSort::SortPairs(sort_tmp, sb, key, key_s, idx, order,
                                                     (int)n_rows, 0, 64, m->stream)) != cudaSuccess)
                break;
            k_mf_gather<<<kB200SMs * 8, 256, 0, m->stream>>>(tmp, order, n_rows, m->rays);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
        }
        if ((e = cudaMemsetAsync(m->norm, 0, (size_t)m->C * 4, m->stream)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(m->u, 0, (size_t)m->C * 4, m->stream)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(m->flag, 0, 4, m->stream)) != cudaSuccess) break;
        const size_t smem = mf_smem(m);
        if ((e = cudaFuncSetAttribute(k_mf_colsum, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess) break;
        if ((e = cudaFuncSetAttribute(k_mf_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess) break;
        if (n_rows) {
            k_mf_colsum<<<kB200SMs * 4, kMfThreads, smem, m->stream>>>(m->rays, n_rows, g, m->dil,
                                                                       m->cap, m->norm, m->flag);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
        }
        e = cudaStreamSynchronize(m->stream);
    } while (0);
    release();
    if (e != cudaSuccess)
        return bail(mf_fail(e == cudaErrorMemoryAllocation ? MLEM_ERR_NOMEM : MLEM_ERR_CUDA,
                            "matrix-free set-up", e));
    int s = mf_check_flag(m);
    if (s != MLEM_OK) return bail(s);
    // natural-order column sums and their sequential double sum (initImage)
    std::vector<float> dev(m->C);
    e = cudaMemcpy(dev.data(), m->norm, (size_t)m->C * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bail(mf_fail(MLEM_ERR_CUDA, "column sums", e));
    m->norm_nat.resize(m->C);
    double sn = 0.0;
    for (uint32_t v = 0; v < m->C; ++v) {
        m->norm_nat[v] = dev[m->perm_host[v]];
        sn += m->norm_nat[v];
    }
    m->sumnorm = sn;
    *out = m;
    return MLEM_OK;
}

void mlem_mf_destroy(mlem_mf* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (void* p : {(void*)m->rays, (void*)m->perm, (void*)m->dil, (void*)m->norm, (void*)m->x,
                    (void*)m->u, (void*)m->sino, (void*)m->flag})
        if (p) cudaFree(p);
    if (m->own_stream) cudaStreamDestroy(m->own_stream);
    delete m;
}

int mlem_mf_set_stream(mlem_mf* m, void* stream) {
    if (!m) return set_error(nullptr, MLEM_ERR_INVALID, "null matrix-free context");
    MF_CK("cudaSetDevice", cudaSetDevice(m->device));
    MF_CK("sync", cudaStreamSynchronize(m->stream));
    m->stream = stream ? static_cast<cudaStream_t>(stream) : m->own_stream;
    return MLEM_OK;
}

int mlem_mf_column_sums(mlem_mf* m, float* norm) {
    if (!m || !norm) return set_error(nullptr, MLEM_ERR_INVALID, "null argument");
    std::copy(m->norm_nat.begin(), m->norm_nat.end(), norm);
    return MLEM_OK;
}

int mlem_mf_set_sinogram(mlem_mf* m, const int32_t* sino) {
    if (!m || !sino) return set_error(nullptr, MLEM_ERR_INVALID, "null argument");
    MF_CK("cudaSetDevice", cudaSetDevice(m->device));
    MF_CK("sinogram upload", cudaMemcpyAsync(m->sino, sino, (size_t)m->R * 4, cudaMemcpyHostToDevice,
                                             m->stream));
    double s = 0.0;
    for (uint32_t r = 0; r < m->R; ++r) s += sino[r];
    m->sumin = s;
    MF_CK("sync", cudaStreamSynchronize(m->stream));
    m->have_sino = true;
    return MLEM_OK;
}

// initImage (mlem_seq/seqcsr4mlem.cpp:52-66): float(sum of counts / sum of column sums).
int mlem_mf_init_image(mlem_mf* m, float* init_value) {
    if (!m) return set_error(nullptr, MLEM_ERR_INVALID, "null matrix-free context");
    if (!m->have_sino) return set_error(nullptr, MLEM_ERR_STATE, "set the sinogram first");
    MF_CK("cudaSetDevice", cudaSetDevice(m->device));
    const float v = (float)(m->sumin / m->sumnorm);
    k_mf_fill<<<kB200SMs * 4, 256, 0, m->stream>>>(m->x, m->C, v);
    MF_CK("image fill", cudaGetLastError());
    MF_CK("sync", cudaStreamSynchronize(m->stream));
    if (init_value) *init_value = v;
    m->have_image = true;
    return MLEM_OK;
}

int mlem_mf_iterate(mlem_mf* m, int n_iter) {
    if (!m) return set_error(nullptr, MLEM_ERR_INVALID, "null matrix-free context");
    if (!m->have_image) return set_error(nullptr, MLEM_ERR_STATE, "initialise the image first");
    if (n_iter < 0) return set_error(nullptr, MLEM_ERR_INVALID, "negative iteration count");
    MF_CK("cudaSetDevice", cudaSetDevice(m->device));
    const MfGrid g = grid_of(m);
    const size_t smem = mf_smem(m);
    // the attribute belongs to the kernel: set it for this context's grid
    MF_CK("shared memory", cudaFuncSetAttribute(k_mf_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)smem));
    for (int it = 0; it < n_iter; ++it) {
        if (m->R) {
            k_mf_fused<<<kB200SMs * 4, kMfThreads, smem, m->stream>>>(m->rays, m->R, g, m->dil, m->cap,
                                                                      m->x, m->sino, m->u, m->flag);
            MF_CK("matrix-free pass", cudaGetLastError());
        }
        MF_CK("calcUpdate", apply_update(m->x, m->u, m->norm, m->C, 1, true, m->stream));
    }
    return mf_check_flag(m);
}

int mlem_mf_get_image(mlem_mf* m, float* image) {
    if (!m || !image) return set_error(nullptr, MLEM_ERR_INVALID, "null argument");
    MF_CK("cudaSetDevice", cudaSetDevice(m->device));
    std::vector<float> dev(m->C);
    MF_CK("image download", cudaMemcpyAsync(dev.data(), m->x, (size_t)m->C * 4, cudaMemcpyDeviceToHost,
                                            m->stream));
    MF_CK("sync", cudaStreamSynchronize(m->stream));
    for (uint32_t v = 0; v < m->C; ++v) image[v] = dev[m->perm_host[v]];
    return MLEM_OK;
}

int mlem_mf_info(const mlem_mf* m, uint64_t* device_bytes, uint32_t* lane_capacity) {
    if (!m) return set_error(nullptr, MLEM_ERR_INVALID, "null matrix-free context");
    if (device_bytes) *device_bytes = m->device_bytes;
    if (lane_capacity) *lane_capacity = m->cap;
    return MLEM_OK;
}

}  // extern "C"
