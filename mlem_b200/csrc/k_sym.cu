// k_sym.cu -- expansion of a symmetry-compressed CSR4 matrix on the device.
//
// A scanner whose geometry is mirror-symmetric lets a matrix generator store
// only part of the LOR x voxel elements: the header flags (csr4matrix.cpp:
// 62-65) say which mirrors (x: the yz plane, y: the xz plane, z: the xy plane)
// were used, and the omitted elements are the stored ones with both the LOR's
// detectors and the voxel mirrored.  The reference regenerates them only in
// its matrix viewer (visualizematrix/dispcsr4spy.cpp:123-140 with the tables
// of symhandler.cpp:33-114); its MLEM drivers ignore the flags.  Here the
// expansion builds the full CSR once, in the order
//   full row t = [stored elements of row t] ++ for each mirror s (the order of
//   symhandler.hpp generateSyms): the elements of every stored row r with
//   lor(r, s) == t, ascending r, voxels mirrored
// so that the result is deterministic:
//   1. count: full row lengths, one launch per mirror (u64 atomics);
//   2. exclusive scan of the lengths -> full row offsets;
//   3. fill: one launch per mirror, a warp per stored row copies its elements
//      to the row's cursor (plus the length of the other source row of the
//      same full row, when that one comes first), then advance: every cursor
//      moves past the mirror's contributions.
// A mirrored LOR is (T(d1), T(d2)) with the smaller detector first
// (symhandler.hpp transformLor); the only other stored row reaching the same
// full row under the same mirror is the swapped LOR d2 * n + d1.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace mlem {

namespace {

struct SymGeom {
    uint32_t n_crystals;
    uint32_t nx, ny, nz;
    uint32_t mirror;  // bit 0: x, bit 1: y, bit 2: z (0: the stored elements themselves)
};

__device__ __forceinline__ uint32_t mirror_voxel(uint32_t v, const SymGeom& g) {
    const uint32_t slice = g.nx * g.ny;
    uint32_t z = v / slice;
    const uint32_t rem = v - z * slice;
    uint32_t y = rem / g.nx;
    uint32_t x = rem - y * g.nx;
    if (g.mirror & 1u) x = g.nx - 1 - x;
    if (g.mirror & 2u) y = g.ny - 1 - y;
    if (g.mirror & 4u) z = g.nz - 1 - z;
    return z * slice + y * g.nx + x;
}

// Full row of stored row r under the mirror (the row itself for mirror 0).
__device__ __forceinline__ uint32_t mirror_lor(uint32_t r, const uint32_t* __restrict__ lut,
                                               const SymGeom& g) {
    if (g.mirror == 0) return r;
    const uint32_t d1 = lut[r / g.n_crystals], d2 = lut[r % g.n_crystals];
    return d1 < d2 ? d1 * g.n_crystals + d2 : d2 * g.n_crystals + d1;
}

__global__ void k_sym_count(const uint64_t* __restrict__ ptr, uint32_t R,
                            const uint32_t* __restrict__ lut, SymGeom g,
                            unsigned long long* __restrict__ counts) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < R;
         r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t n = ptr[r + 1] - ptr[r];
        if (n) atomicAdd(counts + mirror_lor((uint32_t)r, lut, g), (unsigned long long)n);
    }
}

__global__ void k_sym_fill(const uint64_t* __restrict__ ptr, const uint2* __restrict__ el,
                           uint32_t R, const uint32_t* __restrict__ lut, SymGeom g,
                           const unsigned long long* __restrict__ cursor, uint2* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < R; r += nw) {
        const uint64_t b = ptr[r], e = ptr[r + 1];
        if (b == e) continue;  // warp-uniform
        const uint32_t t = mirror_lor((uint32_t)r, lut, g);
        uint64_t off = cursor[t];
        if (g.mirror) {  // the swapped LOR reaches the same full row; the smaller row goes first
            const uint32_t d1 = (uint32_t)r / g.n_crystals, d2 = (uint32_t)r % g.n_crystals;
            const uint64_t partner = (uint64_t)d2 * g.n_crystals + d1;
            if (partner < r) off += ptr[partner + 1] - ptr[partner];
        }
        for (uint64_t k = b + lane; k < e; k += 32) {
            const uint2 q = el[k];
            out[off + (k - b)] = make_uint2(g.mirror ? mirror_voxel(q.x, g) : q.x, q.y);
        }
    }
}

__global__ void k_sym_advance(const uint64_t* __restrict__ ptr, uint32_t R,
                              const uint32_t* __restrict__ lut, SymGeom g,
                              unsigned long long* __restrict__ cursor) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < R;
         r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t n = ptr[r + 1] - ptr[r];
        if (n) atomicAdd(cursor + mirror_lor((uint32_t)r, lut, g), (unsigned long long)n);
    }
}

SymGeom geom_of(const SymExpand& s, uint32_t mirror) {
    return SymGeom{s.n_crystals, s.grid[0], s.grid[1], s.grid[2], mirror};
}

}  // namespace

void sym_detector_luts(uint32_t n_layers, uint32_t n_blocks, uint32_t block_size,
                       uint32_t n_rings, std::vector<uint32_t>& lut) {
    // symhandler.cpp:33-114: a crystal is v + layer * per_layer + ring * per_ring
    // with v in [0, per_layer); the x and y mirrors turn v around the layer,
    // the z mirror swaps rings; the combined mirrors are compositions.
    const uint32_t per_layer = block_size * n_blocks;
    const uint32_t per_ring = per_layer * n_layers;
    const uint32_t n = per_ring * n_rings;
    lut.assign(8ull * n, 0u);
    uint32_t* L[8];
    for (int i = 0; i < 8; ++i) L[i] = lut.data() + (size_t)i * n;
    for (uint32_t i = 0; i < n; ++i) L[0][i] = i;
    const uint32_t xoff = block_size - 1;
    const uint32_t yoff = block_size * (n_blocks / 2 + 1) - 1;
    for (uint32_t r = 0; r < n_rings; ++r)
        for (uint32_t l = 0; l < n_layers; ++l)
            for (uint32_t v = 0; v < per_layer; ++v) {
                const uint32_t base = l * per_layer + r * per_ring;
                L[1][v + base] = (per_layer - v + xoff) % per_layer + base;
                L[2][v + base] = (per_layer - v + yoff) % per_layer + base;
            }
    for (uint32_t r = 0; r < n_rings; ++r)
        for (uint32_t v = 0; v < per_ring; ++v) L[4][v + r * per_ring] = v + (n_rings - 1 - r) * per_ring;
    for (uint32_t i = 0; i < n; ++i) {
        L[3][i] = L[2][L[1][i]];
        L[5][i] = L[4][L[1][i]];
        L[6][i] = L[4][L[2][i]];
        L[7][i] = L[4][L[2][L[1][i]]];
    }
}

std::vector<uint32_t> sym_mirrors(uint32_t sym) {
    // symhandler.hpp generateSyms: x outermost, then y, then z; no identity
    std::vector<uint32_t> out;
    for (uint32_t x = 0; x <= (sym & 1u); ++x)
        for (uint32_t y = 0; y <= ((sym >> 1) & 1u); ++y)
            for (uint32_t z = 0; z <= ((sym >> 2) & 1u); ++z)
                if (x | y | z) out.push_back(x | (y << 1) | (z << 2));
    return out;
}

cudaError_t sym_count(const SymExpand& s, uint32_t mirror, unsigned long long* counts,
                      cudaStream_t st) {
    if (s.R == 0) return cudaSuccess;
    const int grid = (int)std::min<uint64_t>((s.R + 255) / 256, (uint64_t)kB200SMs * 16);
    k_sym_count<<<grid, 256, 0, st>>>(s.ptr, s.R, s.lut + (size_t)mirror * s.n_crystals,
                                      geom_of(s, mirror), counts);
    return cudaGetLastError();
}

cudaError_t sym_fill(const SymExpand& s, uint32_t mirror, unsigned long long* cursor, uint2* out,
                     cudaStream_t st) {
    if (s.R == 0) return cudaSuccess;
    const uint32_t* lut = s.lut + (size_t)mirror * s.n_crystals;
    const SymGeom g = geom_of(s, mirror);
    const int wgrid = (int)std::min<uint64_t>(((uint64_t)s.R * 32 + 255) / 256, (uint64_t)kB200SMs * 16);
    k_sym_fill<<<wgrid, 256, 0, st>>>(s.ptr, s.el, s.R, lut, g, cursor, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int grid = (int)std::min<uint64_t>((s.R + 255) / 256, (uint64_t)kB200SMs * 16);
    k_sym_advance<<<grid, 256, 0, st>>>(s.ptr, s.R, lut, g, cursor);
    return cudaGetLastError();
}

}  // namespace mlem
