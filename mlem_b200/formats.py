"""File formats of the reference MLEM tools, in numpy.

These are byte-compatible with the reference's loaders and writers:

* CSR4 system matrix -- helper_files_common/csr4matrix.cpp:32-157
  (28-byte header: b"PCSR", version byte 4 at offset 4, symmetry flags at 5,
  nRows u32 at 8, nColumns u32 at 12, nnz u64 at 16, scanConfigBytes u32 at
  24; then the scanner-geometry block; then nRows uint64 row END offsets with
  no leading zero; then nnz 8-byte elements {uint32 column, float32 value},
  helper_files_common/matrixelement.hpp:37-46).
* Sinogram / image / checkpoint vectors -- raw headerless arrays
  (helper_files_common/vector.hpp:33-53, 77-87, 102-140): int32 counts,
  float32 images, and the img.chkpt / iter.chkpt pair of
  mlem_mpi/mpicsr4mlem.cpp:95-154.

The C++ loader used by the command-line driver lives in
mlem_b200/csrc/host/csr4.cpp; this module is the Python mirror used to write
synthetic inputs and to read results.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

CSR4_MAGIC = b"PCSR"
CSR4_VERSION = 4
CSR4_HEADER_BYTES = 28
CSR4_MIN_SCANCONFIG_BYTES = 60
ELEM_DTYPE = np.dtype([("index", "<u4"), ("value", "<f4")])

IMG_CHECKPOINT_NAME = "img.chkpt"
ITER_CHECKPOINT_NAME = "iter.chkpt"


@dataclass
class Csr4:
    """A CSR4 matrix held in host memory (or memory-mapped)."""

    n_rows: int
    n_cols: int
    row_end: np.ndarray  # uint64[R], END offsets
    elems: np.ndarray  # ELEM_DTYPE[Z]
    flags: int = 0
    grid: tuple = (0, 0, 0)
    voxel_size: tuple = (1.0, 1.0, 1.0)
    # detector of the scanner block: (n_layers, n_blocks, block_size, n_rings)
    scanner: tuple = (1, 1, 1, 1)

    @property
    def nnz(self) -> int:
        return int(self.row_end[-1]) if self.n_rows else 0

    def row_ptr(self) -> np.ndarray:
        """R+1 offsets with a leading zero (the device layout)."""
        out = np.zeros(self.n_rows + 1, np.uint64)
        out[1:] = self.row_end
        return out

    @property
    def cols(self) -> np.ndarray:
        return self.elems["index"]

    @property
    def vals(self) -> np.ndarray:
        return self.elems["value"]


def scanner_config_block(grid=(0, 0, 0), voxel_size=(1.0, 1.0, 1.0),
                         scanner=(1, 1, 1, 1)) -> bytes:
    """The scanner-geometry block csr4matrix.cpp:100-138 parses: n_layers
    layers (5 floats each), n_blocks, block_size with block_size - 1 gaps,
    n_rings with n_rings - 1 gaps, the voxel size and the voxel grid.  The
    default is the minimal 60-byte block (one layer, one block of size 1, one
    ring).  Crystal dimensions and gaps are written as 1.0 / 0.0: only the
    counts matter to the MLEM path."""
    n_layers, n_blocks, block_size, n_rings = scanner
    b = struct.pack("<I", n_layers) + struct.pack("<5f", 1.0, 1.0, 1.0, 1.0, 0.0) * n_layers
    b += struct.pack("<II", n_blocks, block_size) + struct.pack("<f", 0.0) * (block_size - 1)
    b += struct.pack("<I", n_rings) + struct.pack("<f", 0.0) * (n_rings - 1)
    b += struct.pack("<3f", *voxel_size)
    b += struct.pack("<3I", *grid)
    if scanner == (1, 1, 1, 1):
        assert len(b) == CSR4_MIN_SCANCONFIG_BYTES
    return b


def csr4_header(n_rows: int, n_cols: int, nnz: int, scan: bytes, flags: int = 0) -> bytes:
    return (CSR4_MAGIC + struct.pack("<BBxx", CSR4_VERSION, flags)
            + struct.pack("<IIQI", n_rows, n_cols, nnz, len(scan)))


def write_csr4(path, n_rows, n_cols, row_end, elems, grid=(0, 0, 0),
               voxel_size=(1.0, 1.0, 1.0), flags=0, scanner=(1, 1, 1, 1)) -> None:
    row_end = np.ascontiguousarray(row_end, dtype=np.uint64)
    elems = np.ascontiguousarray(elems)
    if elems.dtype != ELEM_DTYPE:
        elems = elems.view(ELEM_DTYPE)
    if row_end.shape != (n_rows,):
        raise ValueError("row_end must hold one END offset per row")
    nnz = int(row_end[-1]) if n_rows else 0
    if elems.shape[0] != nnz:
        raise ValueError("element count does not match the last row END offset")
    scan = scanner_config_block(grid, voxel_size, scanner)
    with open(path, "wb") as f:
        f.write(csr4_header(n_rows, n_cols, nnz, scan, flags))
        f.write(scan)
        row_end.tofile(f)
        elems.tofile(f)


def read_csr4(path, mmap: bool = True) -> Csr4:
    """Parse and validate a CSR4 file the way csr4matrix.cpp:32-157 does, but
    with 64-bit size arithmetic (the reference's uint32 size check at :85-92
    wraps for files above 4 GiB)."""
    size = os.path.getsize(path)
    if size < CSR4_HEADER_BYTES:
        raise ValueError(f"File too short {path}")
    with open(path, "rb") as f:
        head = f.read(min(1000, size))
    if head[:4] != CSR4_MAGIC:
        raise ValueError(f"Input file '{path}' is not a CSR matrix")
    if head[4] != CSR4_VERSION:
        raise ValueError(f"Input file '{path}' has wrong CSR version (need v4)")
    flags = head[5]
    n_rows, n_cols, nnz, scan_bytes = struct.unpack_from("<IIQI", head, 8)
    need = CSR4_HEADER_BYTES + scan_bytes + 8 * n_rows + 8 * nnz
    if size < need:
        raise ValueError(f"Input file '{path}' is too short: {size} B instead of at least {need} B")
    if scan_bytes < CSR4_MIN_SCANCONFIG_BYTES:
        raise ValueError("Cannot find scanner geometry configuration")
    p = CSR4_HEADER_BYTES
    (n_layers,) = struct.unpack_from("<I", head, p); p += 4 + 20 * n_layers
    (n_blocks,) = struct.unpack_from("<I", head, p); p += 4
    (blocksize,) = struct.unpack_from("<I", head, p); p += 4 + 4 * max(blocksize - 1, 0)
    (n_rings,) = struct.unpack_from("<I", head, p); p += 4 + 4 * max(n_rings - 1, 0)
    voxel_size = struct.unpack_from("<3f", head, p); p += 12
    grid = struct.unpack_from("<3I", head, p); p += 12
    if p - CSR4_HEADER_BYTES != scan_bytes:
        raise ValueError("Error reading scanner geometry configuration")
    off = CSR4_HEADER_BYTES + scan_bytes
    if mmap:
        row_end = np.memmap(path, dtype=np.uint64, mode="r", offset=off, shape=(n_rows,))
        elems = (np.memmap(path, dtype=ELEM_DTYPE, mode="r", offset=off + 8 * n_rows, shape=(nnz,))
                 if nnz else np.zeros(0, ELEM_DTYPE))
    else:
        with open(path, "rb") as f:
            f.seek(off)
            row_end = np.fromfile(f, dtype=np.uint64, count=n_rows)
            elems = np.fromfile(f, dtype=ELEM_DTYPE, count=nnz)
    return Csr4(n_rows, n_cols, row_end, elems, flags, tuple(grid), tuple(voxel_size),
                (n_layers, n_blocks, blocksize, n_rings))


def read_vector(path, dtype) -> np.ndarray:
    """vector.hpp:33-53: the length is the file size / element size; a size
    that is not a multiple of the element size is an error."""
    dtype = np.dtype(dtype)
    size = os.path.getsize(path)
    if size % dtype.itemsize:
        raise ValueError(f"Cannot open file {path}")
    return np.fromfile(path, dtype=dtype)


def write_vector(path, arr, dtype=None, sync: bool = False) -> None:
    """vector.hpp:77-87 (writeToFile) or :102-114 (writeToFileSync when sync)."""
    a = np.ascontiguousarray(arr if dtype is None else np.asarray(arr, dtype=dtype))
    with open(path, "wb") as f:
        a.tofile(f)
        if sync:
            f.flush()
            os.fsync(f.fileno())


def read_checkpoint(directory, n_cols):
    """Return (image, next_iteration) when BOTH checkpoint files exist
    (mpicsr4mlem.cpp:536-553), else None.  The image size must match
    (vector.hpp:116-140)."""
    img = os.path.join(directory, IMG_CHECKPOINT_NAME)
    itr = os.path.join(directory, ITER_CHECKPOINT_NAME)
    if not (os.path.exists(img) and os.path.exists(itr)):
        return None
    image = read_vector(img, np.float32)
    if image.size != n_cols:
        raise ValueError(f"Mismatch element number {img}")
    with open(itr, "rb") as f:
        raw = f.read(4)
    if len(raw) != 4:
        raise ValueError(f"Cannot read file {itr}")
    return image, struct.unpack("<i", raw)[0]
