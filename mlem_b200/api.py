"""Python host API over the C ABI (include/mlem_b200.h).

Two layers:

* `Context` -- one system matrix resident on one GPU, with the
  device-resident reconstruction (B frames), tuning, the device-pointer
  entry points and the host IO of the reference formats.
* Module functions with the reference's names and argument meaning
  (mlem_seq/seqcsr4mlem.cpp:37-189): calcColumnSums, initImage, calcFwProj,
  calcCorrel, calcBkProj, calcUpdate and mlem.  Output vectors are passed in
  and filled like the reference's `Vector<float>&` parameters; a size
  mismatch raises where the reference asserts.

Every call goes to the CUDA library; there is no CPU fallback.  Errors raise
`MlemError` with the library's message.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _capi_sig as sig
from ._native import core_lib

MLEM_OK = 0
MLEM_ERR_INVALID = 1
MLEM_ERR_CUDA = 2
MLEM_ERR_IO = 3
MLEM_ERR_FORMAT = 4
MLEM_ERR_NOMEM = 5
MLEM_ERR_STATE = 6
MLEM_ERR_MATRIX = 7
MLEM_NO_CHECKPOINT = 8

FLAG_EXACT = 0x1
FLAG_NO_CSC = 0x2
FLAG_CHECKED = 0x4
FLAG_NATURAL_LAYOUT = 0x8
FLAG_NO_ROW_ORDER = 0x10
FLAG_EXPAND_SYMMETRY = 0x20
FLAG_MIRROR_KERNELS = 0x40

BK_AUTO, BK_CSC, BK_ATOMIC, BK_FUSED, BK_REGION, BK_MIRRORED = 0, 1, 2, 3, 4, 5
BATCH_INTERLEAVED, BATCH_ITEMS = 0, 1
VISIT_FILE, VISIT_SORTED, VISIT_SORTED_CHUNKED, VISIT_SORTED_STAGED = 0, 1, 2, 3
VISIT_NAMES = {VISIT_FILE: "file", VISIT_SORTED: "sorted", VISIT_SORTED_CHUNKED: "sorted-chunked",
               VISIT_SORTED_STAGED: "sorted-staged"}
BATCH_NAMES = {BATCH_INTERLEAVED: "interleaved", BATCH_ITEMS: "items"}
BK_NAMES = {BK_CSC: "csc", BK_ATOMIC: "atomic", BK_FUSED: "fused", BK_REGION: "region",
            BK_MIRRORED: "mirrored"}

ELEM_DTYPE = np.dtype([("index", "<u4"), ("value", "<f4")])


class MlemError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_status_name(status)}: {message}")
        self.status = status
        self.message = message


def _status_name(s: int) -> str:
    return core_lib().mlem_status_string(s).decode()


def _raise(status: int, ctx=None):
    if status == MLEM_OK:
        return
    lib = core_lib()
    msg = (lib.mlem_last_error(ctx) if ctx else lib.mlem_global_error()).decode(errors="replace")
    raise MlemError(status, msg)


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a, n=None, name="array"):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if n is not None and a.size != n:
        raise MlemError(MLEM_ERR_INVALID, f"{name} has {a.size} entries, expected {n}")
    return a


def _i32(a, n=None, name="array"):
    a = np.ascontiguousarray(a, dtype=np.int32)
    if n is not None and a.size != n:
        raise MlemError(MLEM_ERR_INVALID, f"{name} has {a.size} entries, expected {n}")
    return a


class Context:
    """A CSR4 matrix on one GPU (mlem_create)."""

    def __init__(self, row_end, elems, n_rows: int, n_cols: int, flags: int = 0, device: int = 0,
                 grid=None):
        """grid = (nx, ny, nz) with nx*ny*nz == n_cols enables the device brick
        layout of the image (results are unchanged); None keeps natural order."""
        lib = core_lib()
        row_end = np.ascontiguousarray(row_end, dtype=np.uint64)
        elems = np.ascontiguousarray(elems)
        nnz = int(row_end[-1]) if n_rows else 0
        h = ctypes.c_void_p()
        g = None
        if grid is not None and int(np.prod(grid)) == n_cols:
            g = (ctypes.c_uint32 * 3)(*[int(v) for v in grid])
        st = lib.mlem_create_grid(ctypes.byref(h), _p(row_end), _p(elems), n_rows, n_cols, nnz, g,
                                  flags, device)
        _raise(st)
        self._h = h
        self._refresh()

    @classmethod
    def _wrap(cls, h):
        self = cls.__new__(cls)
        self._h = h
        self._refresh()
        return self

    @classmethod
    def from_matrix(cls, m, flags: int = 0, device: int = 0) -> "Context":
        """From a formats.Csr4 (host arrays or a memory-mapped file); its grid
        selects the device brick layout when it matches the column count."""
        grid = getattr(m, "grid", None)
        return cls(m.row_end, m.elems, m.n_rows, m.n_cols, flags, device,
                   grid if grid and int(np.prod(grid)) == m.n_cols else None)

    @classmethod
    def from_file(cls, path: str, flags: int = 0, device: int = 0) -> "Context":
        h = ctypes.c_void_p()
        _raise(core_lib().mlem_create_from_file(ctypes.byref(h), str(path).encode(), flags, device))
        return cls._wrap(h)

    @classmethod
    def symmetric(cls, m, flags: int = 0, device: int = 0) -> "Context":
        """The full matrix of a symmetry-compressed formats.Csr4 (its header
        flags select the mirrors, its scanner block and grid the geometry):
        mlem_create_symmetric."""
        n_layers, n_blocks, block_size, n_rings = m.scanner
        sym = sig.MlemSymmetry(int(m.flags) & 7, n_layers, n_blocks, block_size, n_rings,
                               (ctypes.c_uint32 * 3)(*m.grid))
        re_ = np.ascontiguousarray(m.row_end, dtype=np.uint64)
        el = np.ascontiguousarray(m.elems)
        h = ctypes.c_void_p()
        _raise(core_lib().mlem_create_symmetric(ctypes.byref(h), _p(re_), _p(el), m.n_rows,
                                                m.n_cols, int(re_[-1]) if m.n_rows else 0,
                                                ctypes.byref(sym), flags, device))
        return cls._wrap(h)

    @classmethod
    def siddon(cls, g, flags: int = 0, device: int = 0) -> "Context":
        """Generate the synthetic matrix of synth.Geometry `g` on the device."""
        h = ctypes.c_void_p()
        _raise(core_lib().mlem_create_siddon(ctypes.byref(h), g.nx, g.ny, g.nz, g.n_rows,
                                             g.min_count, g.max_count, g.radius_scale, g.min_len,
                                             g.seed, flags, device))
        return cls._wrap(h)

    def _refresh(self):
        info = sig.MlemInfo()
        _raise(core_lib().mlem_get_info(self._h, ctypes.byref(info)), self._h)
        self.n_rows, self.n_cols, self.nnz = info.n_rows, info.n_cols, info.nnz
        self.n_frames = info.n_frames
        self.info = info

    def close(self):
        if getattr(self, "_h", None):
            core_lib().mlem_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st):
        _raise(st, self._h)

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream: int = 0) -> None:
        """Enqueue on cudaStream_t `stream` (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._chk(core_lib().mlem_set_stream(self._h, stream or None))

    def kernels_per_iteration(self) -> int:
        n = ctypes.c_int()
        self._chk(core_lib().mlem_kernels_per_iteration(self._h, ctypes.byref(n)))
        return n.value

    # -- matrix copies -------------------------------------------------------
    def csr(self):
        row_end = np.zeros(self.n_rows, np.uint64)
        elems = np.zeros(self.nnz, ELEM_DTYPE)
        self._chk(core_lib().mlem_get_csr(self._h, _p(row_end), _p(elems)))
        return row_end, elems

    def csc(self):
        col_ptr = np.zeros(self.n_cols + 1, np.uint64)
        elems = np.zeros(self.nnz, ELEM_DTYPE)
        self._chk(core_lib().mlem_get_csc(self._h, _p(col_ptr), _p(elems)))
        return col_ptr, elems

    # -- the reference's functions on host arrays ------------------------------
    def column_sums(self) -> np.ndarray:
        out = np.zeros(self.n_cols, np.float32)
        self._chk(core_lib().mlem_calc_column_sums(self._h, _p(out)))
        return out

    def init_value(self, sino) -> float:
        s = _i32(sino)
        v = ctypes.c_float()
        self._chk(core_lib().mlem_init_value(self._h, _p(s), s.size, ctypes.byref(v)))
        return v.value

    def fwproj(self, image) -> np.ndarray:
        x = _f32(image, self.n_cols, "image")
        out = np.zeros(self.n_rows, np.float32)
        self._chk(core_lib().mlem_calc_fwproj(self._h, _p(x), _p(out)))
        return out

    def correl(self, fwproj, sino) -> np.ndarray:
        f = _f32(fwproj, self.n_rows, "fwproj")
        s = _i32(sino)
        out = np.zeros(self.n_rows, np.float32)
        self._chk(core_lib().mlem_calc_correl(self._h, _p(f), _p(s), s.size, _p(out)))
        return out

    def bkproj(self, correl) -> np.ndarray:
        c = _f32(correl, self.n_rows, "correlation")
        out = np.zeros(self.n_cols, np.float32)
        self._chk(core_lib().mlem_calc_bkproj(self._h, _p(c), _p(out)))
        return out

    def update(self, update, norm, image) -> np.ndarray:
        u = _f32(update, self.n_cols, "update")
        n = _f32(norm, self.n_cols, "norm")
        x = np.array(_f32(image, self.n_cols, "image"), copy=True)
        self._chk(core_lib().mlem_calc_update(self._h, _p(u), _p(n), _p(x)))
        return x

    def project_f64(self, x) -> np.ndarray:
        xv = _f32(x, self.n_cols, "image")
        out = np.zeros(self.n_rows, np.float64)
        self._chk(core_lib().mlem_project_f64(self._h, _p(xv), _p(out)))
        return out

    # -- device-resident reconstruction ----------------------------------------
    def set_sinograms(self, sino) -> None:
        s = _i32(sino)
        if s.ndim == 1:
            s = s.reshape(1, -1)
        if s.shape[1] != self.n_rows:
            raise MlemError(MLEM_ERR_INVALID,
                            f"sinogram has {s.shape[1]} entries, the matrix {self.n_rows} rows")
        self._chk(core_lib().mlem_set_sinograms(self._h, _p(s), s.shape[0]))
        self.n_frames = s.shape[0]

    def init_images(self) -> np.ndarray:
        out = np.zeros(self.n_frames, np.float32)
        self._chk(core_lib().mlem_init_images(self._h, _p(out)))
        return out

    def set_images(self, images) -> None:
        x = _f32(images, self.n_frames * self.n_cols, "images")
        self._chk(core_lib().mlem_set_images(self._h, _p(x)))

    def iterate(self, n: int, stats: bool = True):
        """Run n iterations; returns (sums [n,B] f64, zeros [n,B], subnormals [n,B])."""
        B = self.n_frames
        sums = np.zeros((n, B), np.float64) if stats else None
        zeros = np.zeros((n, B), np.uint64) if stats else None
        subn = np.zeros((n, B), np.uint64) if stats else None
        self._chk(core_lib().mlem_iterate(self._h, n, _p(sums), _p(zeros), _p(subn)))
        return sums, zeros, subn

    def get_images(self) -> np.ndarray:
        out = np.zeros((self.n_frames, self.n_cols), np.float32)
        self._chk(core_lib().mlem_get_images(self._h, _p(out)))
        return out

    def step_host(self, sino, images) -> np.ndarray:
        """One iteration end to end on host buffers (images updated in place)."""
        s = _i32(sino)
        B = s.size // self.n_rows
        x = images
        if not (isinstance(x, np.ndarray) and x.dtype == np.float32 and x.flags.c_contiguous):
            raise MlemError(MLEM_ERR_INVALID, "images must be a C-contiguous float32 array")
        self._chk(core_lib().mlem_step_host(self._h, _p(s), _p(x), B))
        self.n_frames = B
        return x

    def profile_phases(self, n: int):
        """(ms[4], bytes[4], launches[4]) per iteration for the phases project,
        backproject, update, stats."""
        ms = np.zeros(4, np.float64)
        by = np.zeros(4, np.float64)
        ln = np.zeros(4, np.int32)
        self._chk(core_lib().mlem_profile_phases(self._h, n, _p(ms), _p(by), _p(ln)))
        return ms, by, ln

    def step_host_ptr(self, sino_ptr: int, images_ptr: int, n_frames: int) -> None:
        """mlem_step_host on raw host pointers (e.g. pinned torch tensors)."""
        self._chk(core_lib().mlem_step_host(self._h, sino_ptr, images_ptr, n_frames))
        self.n_frames = n_frames

    def stream_host(self, sinos, images=None) -> None:
        """mlem_stream_host: len(sinos) iterations, iteration k with sinograms
        sinos[k] ([B][R] int32 arrays, B = the context's frames) and, when
        images is given, its images written into images[k] ([B][C] float32,
        C-contiguous; None entries skip the download)."""
        ss = [_i32(x) for x in sinos]
        for x in ss:
            if x.size != self.n_frames * self.n_rows:
                raise MlemError(MLEM_ERR_INVALID, f"sinograms of {x.size} entries, expected "
                                f"{self.n_frames} x {self.n_rows}")
        ims = None
        if images is not None:
            if len(images) != len(ss):
                raise MlemError(MLEM_ERR_INVALID, "one image buffer (or None) per iteration")
            for x in images:
                if x is not None and not (isinstance(x, np.ndarray) and x.dtype == np.float32 and
                                          x.flags.c_contiguous and x.flags.writeable and
                                          x.size == self.n_frames * self.n_cols):
                    raise MlemError(MLEM_ERR_INVALID,
                                    "images must be writable C-contiguous float32 arrays of B x C")
            ims = [None if x is None else x.ctypes.data for x in images]
        self.stream_host_ptr([x.ctypes.data for x in ss], ims)

    def stream_host_ptr(self, sino_ptrs, image_ptrs=None) -> None:
        """mlem_stream_host on raw host pointers (e.g. pinned torch tensors):
        one sinogram pointer per iteration, and one image pointer (or None)
        per iteration or no image list."""
        n = len(sino_ptrs)
        sp = (ctypes.c_void_p * max(n, 1))(*sino_ptrs)
        ip = None
        if image_ptrs is not None:
            if len(image_ptrs) != n:
                raise MlemError(MLEM_ERR_INVALID, "one image pointer (or None) per iteration")
            ip = ctypes.cast((ctypes.c_void_p * max(n, 1))(*image_ptrs), ctypes.c_void_p)
        self._chk(core_lib().mlem_stream_host(self._h, ctypes.cast(sp, ctypes.c_void_p), ip, n))

    # -- tuning -------------------------------------------------------------------
    @staticmethod
    def _tuning_dict(t) -> dict:
        return dict(bk_mode=t.bk_mode, group=t.group, frame_tile=t.frame_tile,
                    blocks_per_sm=t.blocks_per_sm, visit=t.visit, ms_per_iter=t.ms_per_iter)

    def tuning(self) -> dict:
        t = sig.MlemTuning()
        self._chk(core_lib().mlem_get_tuning(self._h, ctypes.byref(t)))
        return self._tuning_dict(t)

    def set_tuning(self, bk_mode=BK_CSC, group=32, frame_tile=1, blocks_per_sm=8,
                   visit=0) -> None:
        """visit: VISIT_FILE, VISIT_SORTED, or VISIT_SORTED_CHUNKED / VISIT_SORTED_STAGED
        (one-pass method, group 32)."""
        t = sig.MlemTuning(bk_mode, group, frame_tile, blocks_per_sm, visit, 0.0)
        self._chk(core_lib().mlem_set_tuning(self._h, ctypes.byref(t)))

    def set_subsets(self, n: int) -> None:
        """Ordered subsets (OSEM): rows r % n form subset r's sub-iteration;
        1 turns them off.  Runs on the one-pass method (BK_FUSED)."""
        self._chk(core_lib().mlem_set_subsets(self._h, int(n)))

    def subsets(self) -> int:
        n = ctypes.c_uint32()
        self._chk(core_lib().mlem_get_subsets(self._h, ctypes.byref(n)))
        return n.value

    def subset_column_sums(self, s: int) -> np.ndarray:
        out = np.zeros(self.n_cols, np.float32)
        self._chk(core_lib().mlem_subset_column_sums(self._h, int(s), _p(out)))
        return out

    def autotune(self, deterministic_only: bool = False) -> dict:
        t = sig.MlemTuning()
        self._chk(core_lib().mlem_autotune(self._h, 1 if deterministic_only else 0, ctypes.byref(t)))
        return self._tuning_dict(t)

    # -- device pointers (ints) ----------------------------------------------------
    def fwproj_d(self, x_ptr: int, y_ptr: int, n_frames: int = 1, stream: int = 0) -> None:
        self._chk(core_lib().mlem_fwproj_d(self._h, x_ptr, y_ptr, n_frames, stream))

    def bkproj_d(self, y_ptr: int, x_ptr: int, n_frames: int = 1, stream: int = 0) -> None:
        self._chk(core_lib().mlem_bkproj_d(self._h, y_ptr, x_ptr, n_frames, stream))

    def fwproj_correl_d(self, x_ptr, sino_ptr, correl_ptr, n_frames=1, stream=0) -> None:
        self._chk(core_lib().mlem_fwproj_correl_d(self._h, x_ptr, sino_ptr, correl_ptr, n_frames,
                                                  stream))

    def fused_update_d(self, x_ptr, sino_ptr, update_ptr, n_frames=1, stream=0) -> None:
        """update = A^T calcCorrel(sino, A x) in one pass over the matrix."""
        self._chk(core_lib().mlem_fused_update_d(self._h, x_ptr, sino_ptr, update_ptr, n_frames,
                                                 stream))

    def ratio_rows_d(self, x_ptr, sino_ptr, rows_ptr, update_ptr, stream=0) -> None:
        """update = A^T calcCorrel(sino, A x) and rows = A x (0 for rows
        without a count) in one pass (one frame)."""
        self._chk(core_lib().mlem_ratio_rows_d(self._h, x_ptr, sino_ptr, rows_ptr, update_ptr,
                                               stream))

    def adjoint_update_d(self, du_ptr, sino_ptr, rows_ptr, update_ptr, stream=0) -> None:
        """update = A^T df, df = -(A du) (sino / rows) / rows where both are
        nonzero, in one pass (one frame)."""
        self._chk(core_lib().mlem_adjoint_update_d(self._h, du_ptr, sino_ptr, rows_ptr, update_ptr,
                                                   stream))

    def bkproj_update_d(self, correl_ptr, x_ptr, n_frames=1, stream=0) -> None:
        self._chk(core_lib().mlem_bkproj_update_d(self._h, correl_ptr, x_ptr, n_frames, stream))

    def apply_update_d(self, update_ptr, x_ptr, n_frames=1, stream=0) -> None:
        self._chk(core_lib().mlem_apply_update_d(self._h, update_ptr, x_ptr, n_frames, stream))

    def norm_d(self) -> int:
        p = ctypes.c_void_p()
        self._chk(core_lib().mlem_norm_d(self._h, ctypes.byref(p)))
        return p.value

    def set_norm_d(self, norm_ptr: int, stream: int = 0) -> None:
        self._chk(core_lib().mlem_set_norm_d(self._h, norm_ptr, stream))


# ---------------------------------------------------------------------------
# Uneven multi-matrix batches.
class Batch:
    """Several contexts (uneven matrices and frame counts) iterated together:
    one persistent kernel per iteration takes row work items of all matrices
    from a shared counter (mlem_batch_*; no counterpart in the reference,
    which runs one matrix per process, mlem_seq/seqcsr4mlem.cpp:137-189).

    The contexts keep their own images: read them with ctx.get_images().
    They must outlive the batch."""

    def __init__(self, contexts: Sequence[Context]):
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[c.handle for c in self.contexts])
        h = ctypes.c_void_p()
        _raise(core_lib().mlem_batch_create(ctypes.byref(h), arr, len(self.contexts)))
        self._h = h.value

    def close(self):
        if getattr(self, "_h", None):
            core_lib().mlem_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st):
        if st != MLEM_OK:
            raise MlemError(st, core_lib().mlem_batch_last_error(self._h).decode(errors="replace"))

    def set_schedule(self, policy: int = BATCH_INTERLEAVED, items_per_block: int = 4,
                     blocks_per_sm: int = 4, frame_tile: int = 0, visit: int = VISIT_FILE) -> None:
        self._chk(core_lib().mlem_batch_set_schedule(self._h, policy, items_per_block,
                                                     blocks_per_sm, frame_tile, visit))

    def set_tiles(self, tiles) -> None:
        """A frame tile per context (0: the batch's tile); contexts sharing a
        tile share one kernel per iteration."""
        tiles = [int(t) for t in tiles]
        if len(tiles) != len(self.contexts):
            raise MlemError(MLEM_ERR_INVALID, "one frame tile per context")
        arr = (ctypes.c_int * len(tiles))(*tiles)
        self._chk(core_lib().mlem_batch_set_tiles(self._h, arr))

    def tiles(self) -> list:
        """The frame tile each context runs with."""
        arr = (ctypes.c_int * len(self.contexts))()
        self._chk(core_lib().mlem_batch_get_tiles(self._h, arr))
        return list(arr)

    def set_visits(self, visits) -> None:
        """A row visit per context (-1: the batch's visit); contexts sharing a
        frame tile and a visit share one kernel per iteration."""
        visits = [int(v) for v in visits]
        if len(visits) != len(self.contexts):
            raise MlemError(MLEM_ERR_INVALID, "one row visit per context")
        arr = (ctypes.c_int * len(visits))(*visits)
        self._chk(core_lib().mlem_batch_set_visits(self._h, arr))

    def visits(self) -> list:
        """The row visit each context runs with."""
        arr = (ctypes.c_int * len(self.contexts))()
        self._chk(core_lib().mlem_batch_get_visits(self._h, arr))
        return list(arr)

    def schedule(self) -> dict:
        pol, ipb, bps = ctypes.c_int(), ctypes.c_uint32(), ctypes.c_int()
        tile, visit, n, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint32(), ctypes.c_double()
        self._chk(core_lib().mlem_batch_get_schedule(self._h, ctypes.byref(pol), ctypes.byref(ipb),
                                                     ctypes.byref(bps), ctypes.byref(tile),
                                                     ctypes.byref(visit), ctypes.byref(n),
                                                     ctypes.byref(ms)))
        return dict(policy=pol.value, items_per_block=ipb.value, blocks_per_sm=bps.value,
                    frame_tile=tile.value, visit=visit.value, n_items=n.value,
                    ms_per_iter=ms.value, tiles=self.tiles(), visits=self.visits())

    def autotune(self) -> dict:
        ms = ctypes.c_double()
        self._chk(core_lib().mlem_batch_autotune(self._h, ctypes.byref(ms)))
        return self.schedule()

    def iterate(self, n: int, stats: bool = True):
        """n iterations of every context; returns one [n, B_i] array of image
        sums per context (None without stats)."""
        if not stats:
            self._chk(core_lib().mlem_batch_iterate(self._h, n, None))
            return None
        sums = [np.zeros((n, c.n_frames), np.float64) for c in self.contexts]
        ptrs = (ctypes.c_void_p * len(sums))(*[a.ctypes.data for a in sums])
        self._chk(core_lib().mlem_batch_iterate(self._h, n, ptrs))
        return sums

    def profile(self, n: int):
        """(ms[4], bytes[4], launches[4]) per iteration: the multi-matrix
        kernel, -, the calcUpdate launches, the statistics."""
        ms = np.zeros(4, np.float64)
        by = np.zeros(4, np.float64)
        ln = np.zeros(4, np.int32)
        self._chk(core_lib().mlem_batch_profile(self._h, n, _p(ms), _p(by), _p(ln)))
        return ms, by, ln


# ---------------------------------------------------------------------------
# The reference's functions (mlem_seq/seqcsr4mlem.cpp), same names and
# argument meaning; `matrix` is a Context.
def _fill(dst, src, what):
    if dst.shape != src.shape:  # the reference asserts the sizes
        raise MlemError(MLEM_ERR_INVALID, f"{what}: size {dst.size} != {src.size}")
    dst[...] = src


def calcColumnSums(matrix: Context, norm: np.ndarray) -> np.ndarray:
    """seqcsr4mlem.cpp:37-49."""
    _fill(norm, matrix.column_sums(), "calcColumnSums")
    return norm


def initImage(norm: np.ndarray, image: np.ndarray, lmsino: np.ndarray, matrix: Context) -> float:
    """seqcsr4mlem.cpp:52-66: image[:] = float(sum(sino) / sum(norm)) (double sums)."""
    del norm  # the context holds the column sums it computed
    v = matrix.init_value(lmsino)
    image[...] = np.float32(v)
    return v


def calcFwProj(matrix: Context, input: np.ndarray, result: np.ndarray) -> np.ndarray:
    """seqcsr4mlem.cpp:69-91."""
    _fill(result, matrix.fwproj(input), "calcFwProj")
    return result


def calcCorrel(fwproj: np.ndarray, input: np.ndarray, correlation: np.ndarray,
               matrix: Context) -> np.ndarray:
    """seqcsr4mlem.cpp:94-105."""
    if not (fwproj.size == input.size == correlation.size):
        raise MlemError(MLEM_ERR_INVALID, "calcCorrel: size mismatch")
    _fill(correlation, matrix.correl(fwproj, input), "calcCorrel")
    return correlation


def calcBkProj(matrix: Context, correlation: np.ndarray, update: np.ndarray) -> np.ndarray:
    """seqcsr4mlem.cpp:108-120."""
    _fill(update, matrix.bkproj(correlation), "calcBkProj")
    return update


def calcUpdate(update: np.ndarray, norm: np.ndarray, image: np.ndarray,
               matrix: Context) -> np.ndarray:
    """seqcsr4mlem.cpp:123-134 (image updated in place)."""
    if not (image.size == update.size == norm.size):
        raise MlemError(MLEM_ERR_INVALID, "calcUpdate: size mismatch")
    image[...] = matrix.update(update, norm, image)
    return image


def mlem(matrix: Context, lmsino, image: Optional[np.ndarray] = None, nIterations: int = 1,
         start_image: Optional[np.ndarray] = None):
    """seqcsr4mlem.cpp:137-189 on the device: column sums (done at create),
    initImage (or a restart image), nIterations iterations.  lmsino may hold
    B sinograms [B, R]; returns (images [B, C], per-iteration sums [n, B])."""
    s = np.asarray(lmsino, dtype=np.int32)
    matrix.set_sinograms(s)
    if start_image is not None:
        matrix.set_images(start_image)
    else:
        matrix.init_images()
    sums, _, _ = matrix.iterate(nIterations)
    out = matrix.get_images()
    if image is not None:
        image[...] = out.reshape(image.shape)
    return out, sums


class MatrixFree:
    """Matrix-free MLEM on the synthetic Siddon geometry (mlem_mf_*): the rays
    are traced again in every pass instead of streaming a stored matrix.
    One frame; natural voxel order."""

    def __init__(self, g, device: int = 0):
        h = ctypes.c_void_p()
        _raise(core_lib().mlem_mf_create_siddon(ctypes.byref(h), g.nx, g.ny, g.nz, g.n_rows,
                                                g.min_count, g.max_count, g.radius_scale,
                                                g.min_len, g.seed, device))
        self._h = h
        self.n_rows, self.n_cols = g.n_rows, g.n_cols

    def close(self):
        if self._h:
            core_lib().mlem_mf_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: int = 0) -> None:
        _raise(core_lib().mlem_mf_set_stream(self._h, stream or None))

    def column_sums(self) -> np.ndarray:
        out = np.zeros(self.n_cols, np.float32)
        _raise(core_lib().mlem_mf_column_sums(self._h, _p(out)))
        return out

    def set_sinogram(self, sino) -> None:
        s = _i32(sino, self.n_rows, "sinogram")
        _raise(core_lib().mlem_mf_set_sinogram(self._h, _p(s)))

    def init_image(self) -> float:
        v = ctypes.c_float()
        _raise(core_lib().mlem_mf_init_image(self._h, ctypes.byref(v)))
        return float(v.value)

    def iterate(self, n: int) -> None:
        _raise(core_lib().mlem_mf_iterate(self._h, n))

    def get_image(self) -> np.ndarray:
        out = np.zeros(self.n_cols, np.float32)
        _raise(core_lib().mlem_mf_get_image(self._h, _p(out)))
        return out

    def info(self) -> dict:
        b, cap = ctypes.c_uint64(), ctypes.c_uint32()
        _raise(core_lib().mlem_mf_info(self._h, ctypes.byref(b), ctypes.byref(cap)))
        return {"device_bytes": int(b.value), "lane_capacity": int(cap.value)}


def measure_l2_rates(device: int = 0) -> dict:
    """mlem_measure_l2_rates: what the L2 serves to random addresses, per
    second -- float gathers of 4 bytes and of 64-byte rows, float reductions
    of 4 bytes and of 64-byte rows (the rates that bound the one-pass walk)."""
    r = np.zeros(4, np.float64)
    _raise(core_lib().mlem_measure_l2_rates(device, _p(r)))
    return {"gather_4B_per_s": float(r[0]), "gather_64B_rows_per_s": float(r[1]),
            "red_4B_per_s": float(r[2]), "red_64B_rows_per_s": float(r[3])}


NOALLOC_MAX_VOXELS = 1048576


def iterate_noalloc_d(row_ptr: int, elems: int, n_elems: int, n_rows: int, n_cols: int,
                      sino: int, norm: int, image: int, stream: int = 0) -> None:
    """mlem_iterate_noalloc_d: one MLEM iteration on caller-owned device
    buffers (integer device addresses) for callers that cannot let the
    library allocate device memory; its update vector lives in a fixed
    4 MiB static device array (at most NOALLOC_MAX_VOXELS voxels), shared by
    all calls on a device, so overlapping calls race.  Rows whose offsets
    decrease or pass n_elems, and columns >= n_cols, are skipped and raise
    MlemError(MLEM_ERR_MATRIX) after the iteration."""
    _raise(core_lib().mlem_iterate_noalloc_d(row_ptr, elems, n_elems, n_rows, n_cols, sino, norm,
                                             image, stream or None))


# ---------------------------------------------------------------------------
# Host IO through the C ABI (the command-line driver's code path).
# ---------------------------------------------------------------------------
def csr4_header(path: str) -> dict:
    h = sig.MlemCsr4Header()
    _raise(core_lib().mlem_csr4_read_header(str(path).encode(), ctypes.byref(h)))
    return dict(n_rows=h.n_rows, n_cols=h.n_cols, nnz=h.nnz, version=h.version, flags=h.flags,
                scan_config_bytes=h.scan_config_bytes, grid=tuple(h.grid),
                voxel_size=tuple(h.voxel_size), file_size=h.file_size, data_offset=h.data_offset)


def csr4_read(path: str):
    h = csr4_header(path)
    row_end = np.zeros(h["n_rows"], np.uint64)
    elems = np.zeros(h["nnz"], ELEM_DTYPE)
    _raise(core_lib().mlem_csr4_read(str(path).encode(), _p(row_end), _p(elems)))
    return h, row_end, elems


def csr4_write(path: str, row_end, elems, n_rows: int, n_cols: int, grid=(0, 0, 0)) -> None:
    row_end = np.ascontiguousarray(row_end, dtype=np.uint64)
    elems = np.ascontiguousarray(elems)
    g = (ctypes.c_uint32 * 3)(*grid)
    _raise(core_lib().mlem_csr4_write(str(path).encode(), _p(row_end), _p(elems), n_rows, n_cols, g))


def vector_read(path: str, dtype) -> np.ndarray:
    dt = np.dtype(dtype)
    n = ctypes.c_uint64()
    _raise(core_lib().mlem_vector_read(str(path).encode(), dt.itemsize, None, 0, ctypes.byref(n)))
    out = np.zeros(n.value, dt)
    _raise(core_lib().mlem_vector_read(str(path).encode(), dt.itemsize, _p(out), out.size,
                                       ctypes.byref(n)))
    return out


def vector_write(path: str, arr, sync: bool = False) -> None:
    a = np.ascontiguousarray(arr)
    _raise(core_lib().mlem_vector_write(str(path).encode(), _p(a), a.itemsize, a.size,
                                        1 if sync else 0))


def checkpoint_write(directory: str, image, next_iter: int) -> None:
    x = _f32(image)
    _raise(core_lib().mlem_checkpoint_write(str(directory).encode(), _p(x), x.size, next_iter))


def checkpoint_read(directory: str, n_cols: int):
    """(image, next_iteration) or None when no complete checkpoint exists."""
    x = np.zeros(n_cols, np.float32)
    it = ctypes.c_int32()
    st = core_lib().mlem_checkpoint_read(str(directory).encode(), _p(x), n_cols, ctypes.byref(it))
    if st == MLEM_NO_CHECKPOINT:
        return None
    _raise(st)
    return x, it.value


def checkpoint_remove(directory: str) -> None:
    _raise(core_lib().mlem_checkpoint_remove(str(directory).encode()))


def partition_rows(row_end, n_ranks: int):
    re_ = np.ascontiguousarray(row_end, dtype=np.uint64)
    starts = np.zeros(n_ranks, np.uint32)
    ends = np.zeros(n_ranks, np.uint32)
    _raise(core_lib().mlem_partition_rows(_p(re_), re_.size, n_ranks, _p(starts), _p(ends)))
    return starts, ends
