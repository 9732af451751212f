"""ctypes binding of oracle/liboracle.so -- the parity checker (tests only).

The oracle is the project's C restatement of mlem_seq/seqcsr4mlem.cpp; the
golden fixtures under tests/golden/ pin it to the reference binary itself.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

_vp = ctypes.c_void_p
_lib = None


def _ptr(a):
    return a.ctypes.data_as(_vp)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", ORACLE_DIR, os.path.join(ORACLE_DIR, "liboracle.so")],
                           check=True, capture_output=True)
        L = ctypes.CDLL(ORACLE_SO)
        u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        L.oracle_column_sums.argtypes = [u32, u32, _vp, _vp, _vp]
        L.oracle_init_value.restype = ctypes.c_float
        L.oracle_init_value.argtypes = [u32, _vp, u64, _vp, _vp, _vp]
        L.oracle_fwproj.argtypes = [u32, _vp, _vp, _vp, _vp]
        L.oracle_correl.argtypes = [u64, _vp, _vp, _vp]
        L.oracle_bkproj.argtypes = [u32, u32, _vp, _vp, _vp, _vp]
        L.oracle_update.argtypes = [u32, _vp, _vp, _vp]
        L.oracle_mlem.restype = i32
        L.oracle_mlem.argtypes = [u32, u32, _vp, _vp, _vp, u64, i32, i32, _vp, _vp, _vp]
        L.oracle_osem.restype = i32
        L.oracle_osem.argtypes = [u32, u32, _vp, _vp, _vp, u64, i32, u32, i32, _vp, _vp, _vp]
        L.oracle_subset_column_sums.argtypes = [u32, u32, _vp, _vp, u32, u32, _vp]
        L.oracle_expand_symmetries.restype = u64
        L.oracle_expand_symmetries.argtypes = [u32, _vp, _vp] + [u32] * 8 + [_vp, _vp]
        L.oracle_mlem_f64.restype = i32
        L.oracle_mlem_f64.argtypes = [u32, u32, _vp, _vp, _vp, u64, i32, _vp]
        L.oracle_mlem_relaxed_f64.argtypes = [u32, u32, _vp, _vp, _vp, _vp, _vp, i32, _vp]
        L.oracle_project_f64.argtypes = [u32, _vp, _vp, _vp, _vp]
        L.oracle_poisson_grad_f64.argtypes = [u32, u32, _vp, _vp, _vp, _vp, _vp]
        L.oracle_transpose.argtypes = [u32, u32, _vp, _vp, _vp, _vp]
        L.oracle_partition.argtypes = [u32, _vp, i32, _vp, _vp]
        _lib = L
    return _lib


def _mat(m):
    re = np.ascontiguousarray(m.row_end, dtype=np.uint64)
    el = np.ascontiguousarray(m.elems)
    return re, el


def column_sums(m):
    re, el = _mat(m)
    out = np.zeros(m.n_cols, np.float32)
    lib().oracle_column_sums(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(out))
    return out


def init_value(norm, sino):
    norm = np.ascontiguousarray(norm, np.float32)
    sino = np.ascontiguousarray(sino, np.int32)
    return float(lib().oracle_init_value(norm.size, _ptr(norm), sino.size, _ptr(sino), None, None))


def fwproj(m, x):
    re, el = _mat(m)
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros(m.n_rows, np.float32)
    lib().oracle_fwproj(m.n_rows, _ptr(re), _ptr(el), _ptr(x), _ptr(out))
    return out


def correl(f, s):
    f = np.ascontiguousarray(f, np.float32)
    s = np.ascontiguousarray(s, np.int32)
    out = np.zeros(f.size, np.float32)
    lib().oracle_correl(f.size, _ptr(f), _ptr(s), _ptr(out))
    return out


def bkproj(m, c):
    re, el = _mat(m)
    c = np.ascontiguousarray(c, np.float32)
    out = np.zeros(m.n_cols, np.float32)
    lib().oracle_bkproj(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(c), _ptr(out))
    return out


def update(u, norm, x):
    u = np.ascontiguousarray(u, np.float32)
    norm = np.ascontiguousarray(norm, np.float32)
    x = np.array(x, np.float32, copy=True)
    lib().oracle_update(x.size, _ptr(u), _ptr(norm), _ptr(x))
    return x


def mlem(m, sino, n_iter, ftz=True, start_image=None):
    """Returns (image float32[C], per-iteration float image sums)."""
    re, el = _mat(m)
    sino = np.ascontiguousarray(sino, np.int32)
    img = np.zeros(m.n_cols, np.float32)
    sums = np.zeros(max(n_iter, 1), np.float32)
    st = None if start_image is None else np.ascontiguousarray(start_image, np.float32)
    rc = lib().oracle_mlem(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(sino), sino.size,
                           n_iter, 1 if ftz else 0, None if st is None else _ptr(st),
                           _ptr(img), _ptr(sums))
    if rc != 0:
        raise ValueError(f"oracle_mlem failed ({rc})")
    return img, sums[:n_iter]


def osem(m, sino, n_iter, n_subsets, ftz=True, start_image=None):
    """Ordered subsets of interleaved rows: (image float32[C], per-iteration sums)."""
    re, el = _mat(m)
    sino = np.ascontiguousarray(sino, np.int32)
    img = np.zeros(m.n_cols, np.float32)
    sums = np.zeros(max(n_iter, 1), np.float32)
    st = None if start_image is None else np.ascontiguousarray(start_image, np.float32)
    rc = lib().oracle_osem(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(sino), sino.size,
                           n_iter, n_subsets, 1 if ftz else 0, None if st is None else _ptr(st),
                           _ptr(img), _ptr(sums))
    if rc != 0:
        raise ValueError(f"oracle_osem failed ({rc})")
    return img, sums[:n_iter]


def expand_symmetries(m):
    """The full matrix of a symmetry-compressed formats.Csr4 (flags, scanner, grid)."""
    from mlem_b200 import formats
    re, el = _mat(m)
    nl, nb, bs, nr = m.scanner
    nx, ny, nz = m.grid
    args = (m.n_rows, _ptr(re), _ptr(el), int(m.flags) & 7, nl, nb, bs, nr, nx, ny, nz)
    z = lib().oracle_expand_symmetries(*args, None, None)
    out_re = np.zeros(m.n_rows, np.uint64)
    out_el = np.zeros(z, formats.ELEM_DTYPE)
    lib().oracle_expand_symmetries(*args, _ptr(out_re), _ptr(out_el))
    return formats.Csr4(m.n_rows, m.n_cols, out_re, out_el, 0, tuple(m.grid))


def subset_column_sums(m, n_subsets, s):
    re, el = _mat(m)
    out = np.zeros(m.n_cols, np.float32)
    lib().oracle_subset_column_sums(m.n_rows, m.n_cols, _ptr(re), _ptr(el), n_subsets, s,
                                    _ptr(out))
    return out


def mlem_f64(m, sino, n_iter):
    re, el = _mat(m)
    sino = np.ascontiguousarray(sino, np.int32)
    img = np.zeros(m.n_cols, np.float64)
    rc = lib().oracle_mlem_f64(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(sino), sino.size,
                               n_iter, _ptr(img))
    if rc != 0:
        raise ValueError(f"oracle_mlem_f64 failed ({rc})")
    return img


def mlem_relaxed_f64(m, sino, x0, omega):
    re, el = _mat(m)
    sino = np.ascontiguousarray(sino, np.int32)
    x0 = np.ascontiguousarray(x0, np.float64)
    omega = np.ascontiguousarray(omega, np.float64)
    out = np.zeros(m.n_cols, np.float64)
    lib().oracle_mlem_relaxed_f64(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(sino), _ptr(x0),
                                  _ptr(omega), omega.size, _ptr(out))
    return out


def project_f64(m, x):
    re, el = _mat(m)
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros(m.n_rows, np.float64)
    lib().oracle_project_f64(m.n_rows, _ptr(re), _ptr(el), _ptr(x), _ptr(out))
    return out


def poisson_grad_f64(m, s, x):
    re, el = _mat(m)
    s = np.ascontiguousarray(s, np.int32)
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros(m.n_cols, np.float64)
    lib().oracle_poisson_grad_f64(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(s), _ptr(x),
                                  _ptr(out))
    return out


def transpose(m):
    re, el = _mat(m)
    col_ptr = np.zeros(m.n_cols + 1, np.uint64)
    ce = np.zeros_like(el)
    lib().oracle_transpose(m.n_rows, m.n_cols, _ptr(re), _ptr(el), _ptr(col_ptr), _ptr(ce))
    return col_ptr, ce


def partition(m, n_ranks):
    re, _ = _mat(m)
    starts = np.zeros(n_ranks, np.uint32)
    ends = np.zeros(n_ranks, np.uint32)
    lib().oracle_partition(m.n_rows, _ptr(re), n_ranks, _ptr(starts), _ptr(ends))
    return starts, ends


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))


REF_CUDA_SO = os.path.join(REF_DIR, "libref_cuda.so")


def ref_cuda_mlem(m, sino, n_iter, variant):
    """The reference's own CUDA kernels (oracle/ref_cuda/harness.cu over
    mlem_cuda/helper_files/cudaKernels.cu): (image float32[C], ms[6] per
    iteration: clear, forward, correlation, back projection, update, all)."""
    L = ctypes.CDLL(REF_CUDA_SO)
    L.ref_cuda_mlem.restype = ctypes.c_int
    L.ref_cuda_mlem.argtypes = [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, _vp, ctypes.c_int,
                                ctypes.c_int, _vp, _vp]
    re, el = _mat(m)
    sino = np.ascontiguousarray(sino, np.int32)
    img = np.zeros(m.n_cols, np.float32)
    ms = np.zeros(6, np.float64)
    rc = L.ref_cuda_mlem(_ptr(re), _ptr(el), m.n_rows, m.n_cols, _ptr(sino), n_iter, variant,
                         _ptr(img), _ptr(ms))
    if rc != 0:
        raise RuntimeError(f"ref_cuda_mlem failed ({rc})")
    return img, ms
