// k_setup.cu -- one-time and bookkeeping kernels: prefix sums, the
// deterministic CSR -> CSC transpose, matrix validation, image statistics,
// frame-layout transposes, and the synthetic Siddon generator on the device.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "siddon_core.h"

namespace mlem {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanTile = 2 * kScanThreads;

__device__ __forceinline__ uint64_t warp_incl_scan(uint64_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t t = __shfl_up_sync(MLEM_FULL_MASK, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-level inclusive scan of a 2048-element tile; out[i+1] = inclusive
// sum within the tile; tile_sums[tile] = tile total.
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const uint64_t* __restrict__ in,
                                                             uint64_t* __restrict__ out,
                                                             uint64_t n,
                                                             uint64_t* __restrict__ tile_sums) {
    __shared__ uint64_t warp_tot[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const uint64_t i0 = base + 2 * t, i1 = i0 + 1;
    const uint64_t a = i0 < n ? in[i0] : 0, b = i1 < n ? in[i1] : 0;
    uint64_t s = warp_incl_scan(a + b, lane);
    if (lane == 31) warp_tot[w] = s;
    __syncthreads();
    if (w == 0) {
        uint64_t v = warp_tot[lane];
        v = warp_incl_scan(v, lane);
        warp_tot[lane] = v;
    }
    __syncthreads();
    const uint64_t before = (w > 0 ? warp_tot[w - 1] : 0) + s - (a + b);
    if (i0 < n) out[i0 + 1] = before + a;
    if (i1 < n) out[i1 + 1] = before + a + b;
    if (t == kScanThreads - 1) tile_sums[blockIdx.x] = before + a + b;
}

// out[i+1] += offsets[tile of i]  (offsets = exclusive scan of tile sums).
__global__ void k_scan_add(uint64_t* __restrict__ out, uint64_t n,
                           const uint64_t* __restrict__ offsets) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i + 1] += offsets[i / kScanTile];
    if (i == 0) out[0] = 0;
}

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------
// Transpose.
// ---------------------------------------------------------------------------
__global__ void k_count_cols(SparseView csr, unsigned long long* __restrict__ cnt) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < csr.nnz;
         k += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + el[k].x, 1ull);
}

// Warp per row: every element gets a slot in its column through an atomic
// cursor; the slot holds {row (or its key), position in row} until the
// columns are sorted.
__global__ void k_fill_csc(SparseView csr, const uint64_t* __restrict__ col_ptr,
                           unsigned long long* __restrict__ cursor, uint2* __restrict__ ce,
                           const uint32_t* __restrict__ row_key) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < csr.n; r += nwarps) {
        const uint64_t b = csr.ptr[r], e = csr.ptr[r + 1];
        for (uint64_t k = b + lane; k < e; k += 32) {
            const uint32_t col = el[k].x;
            const uint64_t slot = col_ptr[col] + atomicAdd(cursor + col, 1ull);
            ce[slot] = make_uint2(row_key ? row_key[r] : (uint32_t)r, (uint32_t)(k - b));
        }
    }
}

__global__ void k_col_len_max(const uint64_t* __restrict__ col_ptr, uint32_t C,
                              unsigned long long* __restrict__ out) {
    unsigned long long m = 0;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < C;
         c += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, (unsigned long long)(col_ptr[c + 1] - col_ptr[c]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(MLEM_FULL_MASK, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__device__ __forceinline__ uint64_t key_of(uint2 q) { return ((uint64_t)q.x << 32) | q.y; }
__device__ __forceinline__ uint2 entry_of(uint64_t k) {
    return make_uint2((uint32_t)(k >> 32), (uint32_t)k);
}

constexpr int kSortCap = 4096;  // keys per column sorted in shared memory (32 KB)

// Block per column: bitonic sort of the column's (row, position) keys.
__global__ void __launch_bounds__(256) k_sort_cols(const uint64_t* __restrict__ col_ptr,
                                                   uint32_t C, uint2* __restrict__ ce) {
    __shared__ uint64_t key[kSortCap];
    for (uint32_t col = blockIdx.x; col < C; col += gridDim.x) {
        const uint64_t b = col_ptr[col], len = col_ptr[col + 1] - b;
        if (len <= 1 || len > kSortCap) continue;  // block-uniform
        uint32_t N = 2;
        while (N < len) N <<= 1;
        for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
            key[i] = i < len ? key_of(ce[b + i]) : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= N; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
                    const uint32_t ixj = i ^ j;
                    if (ixj > i) {
                        const uint64_t a = key[i], c = key[ixj];
                        const bool up = (i & k) == 0;
                        if ((a > c) == up) { key[i] = c; key[ixj] = a; }
                    }
                }
                __syncthreads();
            }
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) ce[b + i] = entry_of(key[i]);
        __syncthreads();
    }
}

__global__ void k_long_load(const uint2* __restrict__ ce, uint64_t b, uint64_t len, uint64_t N,
                            uint64_t* __restrict__ tmp) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x)
        tmp[i] = i < len ? key_of(ce[b + i]) : ~0ull;
}

__global__ void k_bitonic_step(uint64_t* __restrict__ tmp, uint64_t N, uint64_t j, uint64_t k) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ixj = i ^ j;
        if (ixj > i) {
            const uint64_t a = tmp[i], c = tmp[ixj];
            const bool up = (i & k) == 0;
            if ((a > c) == up) { tmp[i] = c; tmp[ixj] = a; }
        }
    }
}

__global__ void k_long_store(const uint64_t* __restrict__ tmp, uint2* __restrict__ ce, uint64_t b,
                             uint64_t len) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
         i += (uint64_t)gridDim.x * blockDim.x)
        ce[b + i] = entry_of(tmp[i]);
}

__global__ void k_list_long(const uint64_t* __restrict__ col_ptr, uint32_t C,
                            uint32_t* __restrict__ list, unsigned int* __restrict__ count) {
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < C;
         c += (uint64_t)gridDim.x * blockDim.x)
        if (col_ptr[c + 1] - col_ptr[c] > (uint64_t)kSortCap) list[atomicAdd(count, 1u)] = (uint32_t)c;
}

// {row (or key), position} -> {row (or key), value}.
__global__ void k_materialize(SparseView csr, uint2* __restrict__ ce,
                              const uint32_t* __restrict__ key_row) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < csr.nnz;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint2 q = ce[s];
        const uint32_t r = key_row ? key_row[q.x] : q.x;
        ce[s] = make_uint2(q.x, el[csr.ptr[r] + q.y].y);
    }
}

__global__ void k_invert(const uint32_t* __restrict__ order, uint32_t* __restrict__ pos, uint64_t n) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x)
        pos[order[v]] = (uint32_t)v;
}

__global__ void k_validate(SparseView csr, uint32_t C, unsigned int* __restrict__ bad) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = tid; r < csr.n; r += stride)
        if (csr.ptr[r] > csr.ptr[r + 1]) atomicOr(bad, 1u);
    if (tid == 0 && csr.ptr[csr.n] != csr.nnz) atomicOr(bad, 2u);
    for (uint64_t k = tid; k < csr.nnz; k += stride)
        if (el[k].x >= C) atomicOr(bad, 4u);
}

// ---------------------------------------------------------------------------
// Image statistics: per frame, double sum, zero count, subnormal count.
// Thread-per-column over a group of V frames; fixed-order reductions.
// ---------------------------------------------------------------------------
constexpr int kStatsThreads = 256;
constexpr int kStatsBlocks = 2 * kB200SMs;

template <int V>
__global__ void __launch_bounds__(kStatsThreads) k_stats(const float* __restrict__ x, uint32_t C,
                                                         uint32_t B, double* __restrict__ ps,
                                                         unsigned long long* __restrict__ pz,
                                                         unsigned long long* __restrict__ pn) {
    __shared__ double ss[kStatsThreads / 32][V];
    __shared__ unsigned long long sz[kStatsThreads / 32][V], sn[kStatsThreads / 32][V];
    const uint32_t g = blockIdx.y;  // frames [g*V, g*V+V)
    double s[V];
    unsigned long long z[V], n[V];
#pragma unroll
    for (int i = 0; i < V; ++i) { s[i] = 0.0; z[i] = 0; n[i] = 0; }
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < C;
         c += (uint64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const float v = x[c * B + (uint64_t)g * V + i];
            const uint32_t bits = __float_as_uint(v) & 0x7fffffffu;
            s[i] += (double)v;
            z[i] += bits == 0;
            n[i] += bits != 0 && bits < 0x00800000u;
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < V; ++i) {
        for (int o = 16; o > 0; o >>= 1) {
            s[i] += __shfl_xor_sync(MLEM_FULL_MASK, s[i], o);
            z[i] += __shfl_xor_sync(MLEM_FULL_MASK, z[i], o);
            n[i] += __shfl_xor_sync(MLEM_FULL_MASK, n[i], o);
        }
        if (lane == 0) { ss[w][i] = s[i]; sz[w][i] = z[i]; sn[w][i] = n[i]; }
    }
    __syncthreads();
    if (threadIdx.x < V) {
        double a = 0.0;
        unsigned long long b = 0, c = 0;
        for (int k = 0; k < kStatsThreads / 32; ++k) {
            a += ss[k][threadIdx.x]; b += sz[k][threadIdx.x]; c += sn[k][threadIdx.x];
        }
        const uint64_t o = (uint64_t)blockIdx.x * B + (uint64_t)g * V + threadIdx.x;
        ps[o] = a; pz[o] = b; pn[o] = c;
    }
}

// One warp per frame: lanes take the block partials in a fixed stride, then a
// fixed butterfly combines the lanes -- the same order on every call.
__global__ void k_stats_final(const double* __restrict__ ps, const unsigned long long* __restrict__ pz,
                              const unsigned long long* __restrict__ pn, uint32_t nblocks,
                              uint32_t B, uint32_t n_out, unsigned int* __restrict__ slot,
                              double* __restrict__ sums, unsigned long long* __restrict__ zeros,
                              unsigned long long* __restrict__ subn) {
    const uint64_t row = slot ? *slot : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t f = w; f < n_out; f += nw) {
        double a = 0.0;
        unsigned long long b = 0, c = 0;
        for (uint32_t k = lane; k < nblocks; k += 32) {
            a += ps[(uint64_t)k * B + f]; b += pz[(uint64_t)k * B + f]; c += pn[(uint64_t)k * B + f];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(MLEM_FULL_MASK, a, o);
            b += __shfl_xor_sync(MLEM_FULL_MASK, b, o);
            c += __shfl_xor_sync(MLEM_FULL_MASK, c, o);
        }
        if (lane == 0) {
            if (sums) sums[row * n_out + f] = a;
            if (zeros) zeros[row * n_out + f] = b;
            if (subn) subn[row * n_out + f] = c;
        }
    }
    __syncthreads();
    if (slot && threadIdx.x == 0) *slot = (unsigned int)row + 1;
}

__global__ void k_fill_frames(float* __restrict__ x, uint64_t n, uint32_t Bp, uint32_t B,
                              const float* __restrict__ vals) {
    const uint64_t total = n * Bp;
    for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < total;
         o += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = (uint32_t)(o % Bp);
        x[o] = b < B ? vals[b] : 0.0f;
    }
}

__global__ void k_correl(const float* __restrict__ f, const int32_t* __restrict__ s,
                         float* __restrict__ c, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        c[i] = correl_of(s[i], f[i]);
}

template <typename T>
__global__ void k_interleave(const T* __restrict__ in, T* __restrict__ out, uint64_t n, uint32_t B,
                             uint32_t Bp, const uint32_t* __restrict__ perm) {
    const uint64_t total = n * B;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < total;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = j / n, i = j - b * n;
        const uint64_t d = perm ? perm[i] : i;
        out[d * Bp + b] = in[j];
    }
}

template <typename T>
__global__ void k_deinterleave(const T* __restrict__ in, T* __restrict__ out, uint64_t n,
                               uint32_t B, uint32_t Bp, const uint32_t* __restrict__ perm) {
    const uint64_t total = n * B;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < total;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = j / n, i = j - b * n;
        const uint64_t d = perm ? perm[i] : i;
        out[j] = in[d * Bp + b];
    }
}

template <bool TO_DEVICE>
__global__ void k_permute(const float* __restrict__ in, float* __restrict__ out,
                          const uint32_t* __restrict__ perm, uint64_t n, uint32_t B) {
    const uint64_t total = n * B;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < total;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = j / B, b = j - i * B;
        const uint64_t d = (uint64_t)perm[i] * B + b;
        if (TO_DEVICE) out[d] = in[j];
        else out[j] = in[d];
    }
}

__global__ void k_remap_columns(uint2* __restrict__ el, uint64_t nnz,
                                const uint32_t* __restrict__ perm) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz;
         k += (uint64_t)gridDim.x * blockDim.x)
        el[k].x = perm[el[k].x];
}

// ---------------------------------------------------------------------------
// Synthetic Siddon generator (thread per row), bit-identical to the host build.
// ---------------------------------------------------------------------------
__device__ __forceinline__ siddon_geom geom_of(const SiddonSpec& s) {
    siddon_geom g;
    g.nx = s.nx; g.ny = s.ny; g.nz = s.nz; g.pad_ = 0;
    g.min_count = s.min_count; g.max_count = s.max_count;
    g.radius_scale = s.radius_scale; g.min_len = s.min_len; g.seed = s.seed;
    return g;
}

__global__ void k_siddon_counts(SiddonSpec s, uint64_t* __restrict__ counts) {
    const siddon_geom g = geom_of(s);
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < s.n_rows;
         r += (uint64_t)gridDim.x * blockDim.x)
        counts[r] = sd_row(&g, (uint32_t)r, nullptr);
}

__global__ void k_siddon_fill(SiddonSpec s, const uint64_t* __restrict__ row_ptr,
                              uint2* __restrict__ elems) {
    const siddon_geom g = geom_of(s);
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < s.n_rows;
         r += (uint64_t)gridDim.x * blockDim.x)
        sd_row(&g, (uint32_t)r, reinterpret_cast<uint32_t*>(elems + row_ptr[r]));
}

__global__ void k_project_f64(SparseView csr, const float* __restrict__ x, double* __restrict__ out) {
    const uint2* el = reinterpret_cast<const uint2*>(csr.pairs);
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < csr.n;
         r += (uint64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint64_t k = csr.ptr[r]; k < csr.ptr[r + 1]; ++k) {
            const uint2 q = el[k];
            s = __dadd_rn(s, __dmul_rn((double)__uint_as_float(q.y), (double)x[q.x]));
        }
        out[r] = s;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Scan.
// ---------------------------------------------------------------------------
size_t scan_scratch_bytes(uint64_t n) {
    size_t total = 256;
    uint64_t m = n;
    while (true) {
        const uint64_t tiles = std::max<uint64_t>(1, ceil_div(m, kScanTile));
        total += align256(tiles * 8) + align256((tiles + 1) * 8);
        if (tiles <= 1) break;
        m = tiles;
    }
    return total;
}

// Three-phase scan: tile-local scans, a (recursive) scan of the tile sums,
// then every output adds the prefix of the tiles before it.
static cudaError_t scan_impl(const uint64_t* in, uint64_t* out, uint64_t n, char* scratch,
                             cudaStream_t st) {
    if (n == 0) return cudaMemsetAsync(out, 0, 8, st);
    const uint64_t tiles = ceil_div(n, kScanTile);
    uint64_t* sums = reinterpret_cast<uint64_t*>(scratch);
    uint64_t* offs = reinterpret_cast<uint64_t*>(scratch + align256(tiles * 8));
    char* next = scratch + align256(tiles * 8) + align256((tiles + 1) * 8);
    k_scan_tile<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, sums);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    err = tiles > 1 ? scan_impl(sums, offs, tiles, next, st) : cudaMemsetAsync(offs, 0, 8, st);
    if (err != cudaSuccess) return err;
    k_scan_add<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(out, n, offs);
    return cudaGetLastError();
}

cudaError_t exclusive_scan_u64(const uint64_t* in, uint64_t* out, uint64_t n, void* scratch,
                               size_t scratch_bytes, cudaStream_t st) {
    if (scratch_bytes < scan_scratch_bytes(n)) return cudaErrorInvalidValue;
    return scan_impl(in, out, n, static_cast<char*>(scratch), st);
}

// ---------------------------------------------------------------------------
// Transpose.
// ---------------------------------------------------------------------------
size_t transpose_scratch_bytes(uint32_t C) {
    return align256(((size_t)C + 1) * 8)            // counts / cursor
           + align256(((size_t)C + 1) * 4)          // long-column list
           + 256                                    // counters
           + scan_scratch_bytes((uint64_t)C);
}

cudaError_t invert_permutation(const uint32_t* order, uint32_t* pos, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_invert<<<kB200SMs * 8, 256, 0, st>>>(order, pos, n);
    return cudaGetLastError();
}

cudaError_t transpose(const SparseView& csr, uint32_t C, uint64_t* col_ptr, uint2* ce,
                      void* scratch, uint32_t* max_col_len, cudaStream_t st,
                      const uint32_t* row_key, const uint32_t* key_row) {
    char* p = static_cast<char*>(scratch);
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(p);
    p += align256(((size_t)C + 1) * 8);
    uint32_t* long_list = reinterpret_cast<uint32_t*>(p);
    p += align256(((size_t)C + 1) * 4);
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(p);  // [0]=max len, [1]=n long
    p += 256;
    void* scan_scratch = p;

    cudaError_t err;
#define MLEM_TRY(x) do { if ((err = (x)) != cudaSuccess) return err; } while (0)
    MLEM_TRY(cudaMemsetAsync(cnt, 0, ((size_t)C + 1) * 8, st));
    MLEM_TRY(cudaMemsetAsync(counters, 0, 256, st));
    const int grid = kB200SMs * 8;
    if (csr.nnz) {
        k_count_cols<<<grid, 256, 0, st>>>(csr, cnt);
        MLEM_TRY(cudaGetLastError());
    }
    MLEM_TRY(exclusive_scan_u64(reinterpret_cast<const uint64_t*>(cnt), col_ptr, C, scan_scratch,
                                scan_scratch_bytes(C), st));
    if (csr.nnz == 0) {
        if (max_col_len) *max_col_len = 0;
        return cudaStreamSynchronize(st);
    }
    MLEM_TRY(cudaMemsetAsync(cnt, 0, ((size_t)C + 1) * 8, st));
    k_fill_csc<<<grid, 256, 0, st>>>(csr, col_ptr, cnt, ce, row_key);
    MLEM_TRY(cudaGetLastError());
    k_col_len_max<<<kB200SMs * 2, 256, 0, st>>>(col_ptr, C, counters);
    MLEM_TRY(cudaGetLastError());
    k_list_long<<<kB200SMs * 2, 256, 0, st>>>(col_ptr, C, long_list,
                                              reinterpret_cast<unsigned int*>(counters + 1));
    MLEM_TRY(cudaGetLastError());
    k_sort_cols<<<kB200SMs * 6, 256, 0, st>>>(col_ptr, C, ce);
    MLEM_TRY(cudaGetLastError());

    unsigned long long host_counters[2] = {0, 0};
    MLEM_TRY(cudaMemcpyAsync(host_counters, counters, 16, cudaMemcpyDeviceToHost, st));
    MLEM_TRY(cudaStreamSynchronize(st));
    const uint64_t max_len = host_counters[0];
    const uint32_t n_long = (uint32_t)(host_counters[1] & 0xffffffffu);
    if (max_col_len) *max_col_len = (uint32_t)std::min<uint64_t>(max_len, 0xffffffffu);
    if (n_long) {
        // Columns too long for shared memory: global bitonic sort, one column at a time.
        std::vector<uint32_t> cols(n_long);
        std::vector<uint64_t> hptr(2);
        MLEM_TRY(cudaMemcpy(cols.data(), long_list, n_long * 4, cudaMemcpyDeviceToHost));
        uint64_t N = 2;
        while (N < max_len) N <<= 1;
        uint64_t* tmp = nullptr;
        MLEM_TRY(cudaMalloc(&tmp, N * 8));
        for (uint32_t c : cols) {
            MLEM_TRY(cudaMemcpy(hptr.data(), col_ptr + c, 16, cudaMemcpyDeviceToHost));
            const uint64_t b = hptr[0], len = hptr[1] - hptr[0];
            uint64_t n2 = 2;
            while (n2 < len) n2 <<= 1;
            const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(n2, 256), kB200SMs * 8);
            k_long_load<<<g, 256, 0, st>>>(ce, b, len, n2, tmp);
            for (uint64_t k = 2; k <= n2; k <<= 1)
                for (uint64_t j = k >> 1; j > 0; j >>= 1) k_bitonic_step<<<g, 256, 0, st>>>(tmp, n2, j, k);
            k_long_store<<<g, 256, 0, st>>>(tmp, ce, b, len);
            if ((err = cudaGetLastError()) != cudaSuccess) { cudaFree(tmp); return err; }
        }
        MLEM_TRY(cudaStreamSynchronize(st));
        cudaFree(tmp);
    }
    k_materialize<<<grid, 256, 0, st>>>(csr, ce, key_row);
    MLEM_TRY(cudaGetLastError());
    return cudaStreamSynchronize(st);
#undef MLEM_TRY
}

cudaError_t validate_csr(const SparseView& csr, uint32_t C, unsigned int* bad_flag,
                         cudaStream_t st) {
    cudaError_t err = cudaMemsetAsync(bad_flag, 0, sizeof(unsigned int), st);
    if (err != cudaSuccess) return err;
    k_validate<<<kB200SMs * 4, 256, 0, st>>>(csr, C, bad_flag);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Statistics and layouts.
// ---------------------------------------------------------------------------
size_t stats_scratch_bytes(uint32_t B) { return (size_t)kStatsBlocks * B * 24 + 256; }

cudaError_t image_stats(const float* x, uint32_t C, uint32_t B, uint32_t n_out, void* partial,
                        unsigned int* slot, double* sums, unsigned long long* zeros,
                        unsigned long long* subnormals, cudaStream_t st) {
    double* ps = static_cast<double*>(partial);
    unsigned long long* pz = reinterpret_cast<unsigned long long*>(ps + (size_t)kStatsBlocks * B);
    unsigned long long* pn = pz + (size_t)kStatsBlocks * B;
    int V = 1;
    for (int v : {16, 8, 4, 2}) if (B % v == 0) { V = v; break; }
    dim3 grid(kStatsBlocks, B / V);
    switch (V) {
        case 16: k_stats<16><<<grid, kStatsThreads, 0, st>>>(x, C, B, ps, pz, pn); break;
        case 8: k_stats<8><<<grid, kStatsThreads, 0, st>>>(x, C, B, ps, pz, pn); break;
        case 4: k_stats<4><<<grid, kStatsThreads, 0, st>>>(x, C, B, ps, pz, pn); break;
        case 2: k_stats<2><<<grid, kStatsThreads, 0, st>>>(x, C, B, ps, pz, pn); break;
        default: k_stats<1><<<grid, kStatsThreads, 0, st>>>(x, C, B, ps, pz, pn); break;
    }
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    k_stats_final<<<1, 512, 0, st>>>(ps, pz, pn, kStatsBlocks, B, n_out, slot, sums, zeros,
                                     subnormals);
    return cudaGetLastError();
}

static unsigned elementwise_grid(uint64_t n) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, 256), kB200SMs * 16));
}

cudaError_t interleave_i32(const int32_t* in, int32_t* out, uint64_t n, uint32_t B, uint32_t Bp,
                           cudaStream_t st) {
    if (n * B == 0) return cudaSuccess;
    k_interleave<int32_t><<<elementwise_grid(n * B), 256, 0, st>>>(in, out, n, B, Bp, nullptr);
    return cudaGetLastError();
}

cudaError_t interleave_f32(const float* in, float* out, uint64_t n, uint32_t B, uint32_t Bp,
                           const uint32_t* perm, cudaStream_t st) {
    if (n * B == 0) return cudaSuccess;
    k_interleave<float><<<elementwise_grid(n * B), 256, 0, st>>>(in, out, n, B, Bp, perm);
    return cudaGetLastError();
}

cudaError_t deinterleave_f32(const float* in, float* out, uint64_t n, uint32_t B, uint32_t Bp,
                             const uint32_t* perm, cudaStream_t st) {
    if (n * B == 0) return cudaSuccess;
    k_deinterleave<float><<<elementwise_grid(n * B), 256, 0, st>>>(in, out, n, B, Bp, perm);
    return cudaGetLastError();
}

cudaError_t permute_to_device(const float* in, float* out, const uint32_t* perm, uint64_t n,
                              uint32_t B, cudaStream_t st) {
    if (n * B == 0) return cudaSuccess;
    k_permute<true><<<elementwise_grid(n * B), 256, 0, st>>>(in, out, perm, n, B);
    return cudaGetLastError();
}

cudaError_t permute_to_natural(const float* in, float* out, const uint32_t* perm, uint64_t n,
                               uint32_t B, cudaStream_t st) {
    if (n * B == 0) return cudaSuccess;
    k_permute<false><<<elementwise_grid(n * B), 256, 0, st>>>(in, out, perm, n, B);
    return cudaGetLastError();
}

cudaError_t remap_columns(uint2* elems, uint64_t nnz, const uint32_t* perm, cudaStream_t st) {
    if (nnz == 0) return cudaSuccess;
    k_remap_columns<<<elementwise_grid(nnz), 256, 0, st>>>(elems, nnz, perm);
    return cudaGetLastError();
}

cudaError_t fill_frames(float* x, uint64_t n, uint32_t Bp, uint32_t B, const float* vals,
                        cudaStream_t st) {
    if (n * Bp == 0) return cudaSuccess;
    k_fill_frames<<<elementwise_grid(n * Bp), 256, 0, st>>>(x, n, Bp, B, vals);
    return cudaGetLastError();
}

cudaError_t correl_elementwise(const float* f, const int32_t* s, float* c, uint64_t n,
                               cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_correl<<<elementwise_grid(n), 256, 0, st>>>(f, s, c, n);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Generator.
// ---------------------------------------------------------------------------
cudaError_t siddon_counts(const SiddonSpec& s, uint64_t* counts, cudaStream_t st) {
    if (s.n_rows == 0) return cudaSuccess;
    k_siddon_counts<<<elementwise_grid(s.n_rows), 256, 0, st>>>(s, counts);
    return cudaGetLastError();
}

cudaError_t siddon_fill(const SiddonSpec& s, const uint64_t* row_ptr, uint2* elems,
                        cudaStream_t st) {
    if (s.n_rows == 0) return cudaSuccess;
    k_siddon_fill<<<elementwise_grid(s.n_rows), 256, 0, st>>>(s, row_ptr, elems);
    return cudaGetLastError();
}

cudaError_t project_f64(const SparseView& csr, const float* x, double* out, cudaStream_t st) {
    if (csr.n == 0) return cudaSuccess;
    k_project_f64<<<elementwise_grid(csr.n), 256, 0, st>>>(csr, x, out);
    return cudaGetLastError();
}

}  // namespace mlem
