"""Loaders for the in-tree native libraries.

* lib/libmlem_b200.so -- the CUDA library behind include/mlem_b200.h (kernels,
  device contexts, host-side CSR4/vector IO).
* lib/libmlem_gen.so  -- the host build of the synthetic Siddon generator.

Both are built in-tree by mlem_b200/build.py.  There is no fallback: if a
library is missing, loading raises with the command that builds it.
"""
from __future__ import annotations

import ctypes
import os
import threading

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
CORE_PATH = os.path.join(LIB_DIR, "libmlem_b200.so")
GEN_PATH = os.path.join(LIB_DIR, "libmlem_gen.so")
CLI_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bin", "mlem_b200")

_lock = threading.Lock()
_gen = None
_core = None

c_u32, c_u64, c_i32, c_i64 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int64
c_dbl, c_vp, c_char_p = ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p


class NativeLibraryMissing(RuntimeError):
    pass


def _load(path: str) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            f"{path} is not built; run `python -m mlem_b200.build` (or __graft_entry__.build())")
    return ctypes.CDLL(path)


def gen_lib() -> ctypes.CDLL:
    global _gen
    with _lock:
        if _gen is None:
            lib = _load(GEN_PATH)
            lib.mlem_gen_siddon_counts.restype = c_u64
            lib.mlem_gen_siddon_counts.argtypes = [c_u32] * 6 + [c_dbl, c_dbl, c_u64, c_vp]
            lib.mlem_gen_siddon_fill.restype = ctypes.c_int
            lib.mlem_gen_siddon_fill.argtypes = [c_u32] * 6 + [c_dbl, c_dbl, c_u64, c_vp, c_vp]
            lib.mlem_gen_project_f64.restype = None
            lib.mlem_gen_project_f64.argtypes = [c_u32, c_vp, c_vp, c_vp, c_vp]
            _gen = lib
        return _gen


def core_lib() -> ctypes.CDLL:
    """The CUDA library with every include/mlem_b200.h entry point typed."""
    global _core
    with _lock:
        if _core is None:
            lib = _load(CORE_PATH)
            from ._capi_sig import declare
            declare(lib)
            _core = lib
        return _core
