"""Record the reference's own mirror tables for symmetry-compressed matrices.

Run from the repository root after `make -C oracle REFDIR=<reference tree>`,
which compiles the matrix viewer's SymHandler (visualizematrix/symhandler.cpp
with scannerconfig.cpp and vector3d.cpp, unmodified) behind the C shim
oracle/ref_sym/shim.cpp into oracle/_ref/libref_sym.so:

    python tests/golden/make_sym_golden.py

Writes tests/golden/sym_ref.npz.  For each scanner case it holds the
reference's generateSyms order for every header flag set (sym 0..7, masks
x | y << 1 | z << 2, padded with 0) and its transformLor / transformVoxel
results per mirror mask:
* "a" (1 layer, 4 blocks of 3, 2 rings; grid 8x8x4) and "b" (2 layers,
  3 blocks of 2 -- an odd block count --, 3 rings; grid 5x6x3): every LOR
  and every voxel;
* "c" (1 layer, 32 blocks of 16, 4 rings: 2,048 crystals; grid 128x128x64,
  the bench's mirrored workload): every detector, and a seeded sample of
  LORs and voxels.
tests/test_symmetry_oracle.py checks the oracle's expansion against these
tables.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_sym.so")

CASES = {
    "a": ((1, 4, 3, 2), (8, 8, 4), None),
    "b": ((2, 3, 2, 3), (5, 6, 3), None),
    "c": ((1, 32, 16, 4), (128, 128, 64), 4096),
}


def load():
    L = ctypes.CDLL(LIB)
    vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    L.refsym_create.restype = vp
    L.refsym_create.argtypes = [u32] * 7
    L.refsym_destroy.argtypes = [vp]
    L.refsym_generate.restype = ctypes.c_int
    L.refsym_generate.argtypes = [vp, u32, vp]
    for f in ("refsym_transform_lors", "refsym_transform_voxels", "refsym_transform_detectors"):
        getattr(L, f).argtypes = [vp, u32, u64, vp, vp]
    return L


def _apply(L, h, fn, mask, ids):
    ids = np.ascontiguousarray(ids, np.uint32)
    out = np.zeros_like(ids)
    getattr(L, fn)(h, mask, ids.size, ids.ctypes.data, out.ctypes.data)
    return out


def tables(L, scanner, grid, sample):
    nl, nb, bs, nr = scanner
    nx, ny, nz = grid
    nc = nl * nb * bs * nr
    h = L.refsym_create(nl, nb, bs, nr, nx, ny, nz)
    try:
        gen = np.zeros((8, 7), np.uint32)
        buf = np.zeros(8, np.uint32)
        for sym in range(8):
            n = L.refsym_generate(h, sym, buf.ctypes.data)
            gen[sym, :n] = buf[:n]
        if sample is None:
            lors = np.arange(nc * nc, dtype=np.uint32)
            voxels = np.arange(nx * ny * nz, dtype=np.uint32)
        else:
            rng = np.random.default_rng(2048)
            lors = np.unique(rng.integers(0, nc * nc, sample, dtype=np.uint64)).astype(np.uint32)
            voxels = rng.integers(0, nx * ny * nz, sample, dtype=np.uint64).astype(np.uint32)
        dets = np.arange(nc, dtype=np.uint32)
        lor_t = np.stack([_apply(L, h, "refsym_transform_lors", m, lors) for m in range(8)])
        vox_t = np.stack([_apply(L, h, "refsym_transform_voxels", m, voxels) for m in range(8)])
        det_t = np.stack([_apply(L, h, "refsym_transform_detectors", m, dets) for m in range(8)])
    finally:
        L.refsym_destroy(h)
    return gen, lors, lor_t, voxels, vox_t, det_t


def main():
    L = load()
    out = {}
    for name, (scanner, grid, sample) in CASES.items():
        gen, lors, lor_t, voxels, vox_t, det_t = tables(L, scanner, grid, sample)
        out[f"{name}_scanner"] = np.array(scanner, np.uint32)
        out[f"{name}_grid"] = np.array(grid, np.uint32)
        out[f"{name}_gen"] = gen
        out[f"{name}_lors"] = lors
        out[f"{name}_lor_t"] = lor_t
        out[f"{name}_voxels"] = voxels
        out[f"{name}_vox_t"] = vox_t
        out[f"{name}_det_t"] = det_t
    np.savez_compressed(os.path.join(HERE, "sym_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "sym_ref.npz"))


if __name__ == "__main__":
    main()
