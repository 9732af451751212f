"""ctypes signatures of include/mlem_b200.h, parsed from the header itself so
the binding cannot drift from the C ABI."""
from __future__ import annotations

import ctypes
import os
import re

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "mlem_b200.h")


class MlemInfo(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_uint32), ("n_cols", ctypes.c_uint32),
                ("nnz", ctypes.c_uint64), ("n_frames", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("device", ctypes.c_int), ("has_csc", ctypes.c_int),
                ("max_col_len", ctypes.c_uint32), ("max_row_len", ctypes.c_uint32),
                ("device_bytes", ctypes.c_uint64), ("nnz_with_counts", ctypes.c_uint64),
                ("rows_with_counts", ctypes.c_uint32)]


class MlemTuning(ctypes.Structure):
    _fields_ = [("bk_mode", ctypes.c_int), ("group", ctypes.c_int),
                ("frame_tile", ctypes.c_int), ("blocks_per_sm", ctypes.c_int),
                ("visit", ctypes.c_int), ("ms_per_iter", ctypes.c_double)]


class MlemCsr4Header(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_uint32), ("n_cols", ctypes.c_uint32),
                ("nnz", ctypes.c_uint64), ("version", ctypes.c_uint8), ("flags", ctypes.c_uint8),
                ("scan_config_bytes", ctypes.c_uint32), ("grid", ctypes.c_uint32 * 3),
                ("voxel_size", ctypes.c_float * 3), ("file_size", ctypes.c_uint64),
                ("data_offset", ctypes.c_uint64), ("n_layers", ctypes.c_uint32),
                ("n_blocks", ctypes.c_uint32), ("block_size", ctypes.c_uint32),
                ("n_rings", ctypes.c_uint32)]


class MlemSymmetry(ctypes.Structure):
    _fields_ = [("sym", ctypes.c_uint32), ("n_layers", ctypes.c_uint32),
                ("n_blocks", ctypes.c_uint32), ("block_size", ctypes.c_uint32),
                ("n_rings", ctypes.c_uint32), ("grid", ctypes.c_uint32 * 3)]


_SCALARS = {
    "int": ctypes.c_int, "uint32_t": ctypes.c_uint32, "uint64_t": ctypes.c_uint64,
    "int32_t": ctypes.c_int32, "double": ctypes.c_double, "float": ctypes.c_float,
}
_STRUCT_PTRS = {
    "mlem_info*": ctypes.POINTER(MlemInfo), "mlem_tuning*": ctypes.POINTER(MlemTuning),
    "mlem_csr4_header*": ctypes.POINTER(MlemCsr4Header),
    "mlem_symmetry*": ctypes.POINTER(MlemSymmetry),
}


def _ctype(decl: str):
    """ctypes type of one declaration "type name" (or "type name[N]")."""
    m = re.match(r"^(.*?)\b([A-Za-z_]\w*)\s*(\[\d*\])?$", decl.strip())
    t = m.group(1).replace("const", "").replace(" ", "") + ("*" if m.group(3) else "")
    if t == "char*":
        return ctypes.c_char_p
    if t in _STRUCT_PTRS:
        return _STRUCT_PTRS[t]
    if t.endswith("*"):
        return ctypes.c_void_p
    if t == "void":
        return None
    return _SCALARS[t]


def prototypes():
    """[(name, restype, [argtypes])] of every function the header declares."""
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"^[ \t]*#.*$", "", text, flags=re.M)  # preprocessor lines
    out = []
    for m in re.finditer(r"([A-Za-z_][\w \t\*]*?)\b(mlem_\w+)\s*\(([^;{]*?)\)\s*;", text):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        restype = _ctype(ret + " result") if ret != "void" else None
        argtypes = []
        if args and args != "void":
            for a in args.split(","):
                argtypes.append(_ctype(a))
        out.append((name, restype, argtypes))
    return out


def declare(lib) -> None:
    for name, restype, argtypes in prototypes():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
