// shim.cpp -- C entry points over the reference's own SymHandler
// (visualizematrix/symhandler.hpp/.cpp, compiled unmodified beside this file
// with visualizematrix/scannerconfig.cpp and vector3d.cpp).  TEST
// INFRASTRUCTURE: tests/golden/make_sym_golden.py loads the library to record
// the reference's mirror tables, which pin the oracle's expansion of
// symmetry-compressed matrices (oracle_expand_symmetries).
//
// A scanner is described as the CSR4 scanner block describes it
// (csr4matrix.cpp:100-138): n_layers layers, n_blocks blocks of block_size
// crystals (block_size - 1 gaps), n_rings rings (n_rings - 1 gaps), and the
// voxel grid.  Mirror masks are x | y << 1 | z << 2.
#include <cstdint>
#include <cstdlib>

#include "scannerconfig.hpp"
#include "symhandler.hpp"

namespace {
struct RefSym {
    ScannerConfig cfg;
    SymHandler* sym = nullptr;
};

SymConfig of_mask(uint32_t m) { return SymConfig(m & 1u, (m >> 1) & 1u, (m >> 2) & 1u); }
}  // namespace

extern "C" {

void* refsym_create(uint32_t n_layers, uint32_t n_blocks, uint32_t block_size, uint32_t n_rings,
                    uint32_t nx, uint32_t ny, uint32_t nz) {
    RefSym* h = new RefSym;
    for (uint32_t i = 0; i < n_layers; ++i) h->cfg.addLayer(LayerConfig(1.0f, 1.0f, 1.0f, 1.0f, 0.0f));
    h->cfg.setNBlocks(n_blocks);
    for (uint32_t i = 1; i < block_size; ++i) h->cfg.addBlockGap(0.0f);
    for (uint32_t i = 1; i < n_rings; ++i) h->cfg.addRingGap(0.0f);
    h->cfg.setGridDim(IVec3(nx, ny, nz));
    h->sym = new SymHandler(h->cfg);
    return h;
}

void refsym_destroy(void* p) {
    RefSym* h = static_cast<RefSym*>(p);
    delete h->sym;
    delete h;
}

// generateSyms(SymConfig of `sym`) as masks, in the reference's order; returns the count.
int refsym_generate(void* p, uint32_t sym, uint32_t* out) {
    std::vector<SymConfig> v = static_cast<RefSym*>(p)->sym->generateSyms(of_mask(sym));
    for (size_t i = 0; i < v.size(); ++i)
        out[i] = (uint32_t)v[i].x | ((uint32_t)v[i].y << 1) | ((uint32_t)v[i].z << 2);
    return (int)v.size();
}

void refsym_transform_lors(void* p, uint32_t mask, uint64_t n, const uint32_t* in, uint32_t* out) {
    const SymHandler* s = static_cast<RefSym*>(p)->sym;
    const SymConfig c = of_mask(mask);
    for (uint64_t i = 0; i < n; ++i) out[i] = (uint32_t)s->transformLor((int)in[i], c);
}

void refsym_transform_voxels(void* p, uint32_t mask, uint64_t n, const uint32_t* in,
                             uint32_t* out) {
    const SymHandler* s = static_cast<RefSym*>(p)->sym;
    const SymConfig c = of_mask(mask);
    for (uint64_t i = 0; i < n; ++i) out[i] = (uint32_t)s->transformVoxel((int)in[i], c);
}

void refsym_transform_detectors(void* p, uint32_t mask, uint64_t n, const uint32_t* in,
                                uint32_t* out) {
    const SymHandler* s = static_cast<RefSym*>(p)->sym;
    const SymConfig c = of_mask(mask);
    for (uint64_t i = 0; i < n; ++i) out[i] = (uint32_t)s->transformDetector((int)in[i], c);
}
}
