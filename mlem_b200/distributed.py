"""Row-sharded MLEM over several GPUs (one process per GPU, torch.distributed).

The reference's distributed MLEM (mlem_mpi/fusedmpimlem.cpp:195-236 with the
partition of mlem_mpi/mpicsr4mlem.cpp:202-234) splits the system matrix
into contiguous, nnz-balanced row blocks.  Every rank holds its block and a
full copy of the image; per iteration it forward-projects its rows,
correlates them with its part of the sinogram, back-projects them into a
full-size partial update, and ONE all-reduce (sum) of the C-float update
vector gives every rank the same update, applied identically everywhere.
The column sums are all-reduced once (mpicsr4mlem.cpp:266), the initial
value uses the global sums (initImage, seqcsr4mlem.cpp:52-66).

The orchestration here is independent of where the shard's arithmetic runs:
`CudaShard` is the product backend (the CUDA library through the C ABI's
device-pointer entry points, on torch's current stream, so NCCL orders after
the kernels); the CPU tests drive the same `reconstruct` with a checker
backend over gloo.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Protocol

import numpy as np

from . import api


@dataclass
class RowBlock:
    start: int
    end: int
    row_end: np.ndarray  # END offsets rebased to the block's first element
    elems: np.ndarray


def partition(row_end: np.ndarray, world: int):
    """(starts, ends) per rank: the reference's nnz-balanced partition."""
    return api.partition_rows(row_end, world)


def row_block(row_end: np.ndarray, elems: np.ndarray, start: int, end: int) -> RowBlock:
    """Rows [start, end) of a CSR4 matrix as a stand-alone CSR4 block."""
    base = int(row_end[start - 1]) if start > 0 else 0
    stop = int(row_end[end - 1]) if end > start else base
    re_ = np.ascontiguousarray(row_end[start:end], dtype=np.uint64) - np.uint64(base)
    return RowBlock(start, end, re_, np.ascontiguousarray(elems[base:stop]))


class Shard(Protocol):
    """Arithmetic of one rank's row block.  Vectors are backend tensors."""

    n_cols: int

    def local_norm(self): ...                  # column sums of the block, float32[C]
    def set_norm(self, norm) -> None: ...      # install the global column sums
    def local_count_sum(self) -> float: ...    # double sum of the block's sinogram
    def project_correl(self, x): ...           # correlation of the block's rows
    def backproject(self, correl): ...         # partial update, float32[C]
    # optional: partial_update(x) = backproject(project_correl(x)) in one step
    def apply(self, update, x) -> None: ...    # x *= calcUpdate factor(update, norm)
    def fill(self, value: float): ...          # new image filled with value
    def to_host(self, x) -> np.ndarray: ...


def sequential_sum(v: np.ndarray) -> float:
    """Double sum of v in array order (the loop of initImage,
    seqcsr4mlem.cpp:55-56): np.cumsum accumulates left to right, unlike
    np.sum's pairwise summation."""
    v = np.asarray(v).ravel()
    return float(np.cumsum(v, dtype=np.float64)[-1]) if v.size else 0.0


def init_image(shard: Shard, dist, group=None, start_image=None):
    """Install the global column sums on the shard (one all-reduce,
    mpicsr4mlem.cpp:266) and return the starting image: initImage's value
    from the global sums (seqcsr4mlem.cpp:52-66), or `start_image` (restart).
    Every rank takes the same collective steps."""
    import torch

    norm = shard.local_norm()
    dist.all_reduce(norm, op=dist.ReduceOp.SUM, group=group)       # mpicsr4mlem.cpp:266
    shard.set_norm(norm)
    if start_image is None:
        sumin = torch.tensor([shard.local_count_sum()], dtype=torch.float64,
                             device=norm.device)
        dist.all_reduce(sumin, op=dist.ReduceOp.SUM, group=group)
        sumnorm = sequential_sum(shard.to_host(norm))
        return shard.fill(float(np.float32(float(sumin.item()) / sumnorm)))
    x = shard.fill(0.0)
    x.copy_(torch.as_tensor(np.asarray(start_image, np.float32)).to(x.device))
    return x


def iterate(shard: Shard, x, n_iter: int, dist, group=None):
    """n_iter iterations on the replicated image x (updated in place): the
    shard's partial update, ONE sum all-reduce of the C floats
    (fusedmpimlem.cpp:227), the identical update on every rank."""
    one_step = getattr(shard, "partial_update", None)
    for _ in range(n_iter):
        if one_step is not None:
            update = one_step(x)  # fusedmpimlem.cpp:205-225 in one pass over the block
        else:
            update = shard.backproject(shard.project_correl(x))
        dist.all_reduce(update, op=dist.ReduceOp.SUM, group=group)  # fusedmpimlem.cpp:227
        shard.apply(update, x)
    return x


def reconstruct(shard: Shard, n_iter: int, dist, group=None, start_image=None):
    """Run initImage + n_iter iterations; returns the (replicated) image on
    the host.  `dist` is torch.distributed (or any module with all_reduce
    and ReduceOp); every rank takes the same collective steps."""
    x = init_image(shard, dist, group, start_image)
    iterate(shard, x, n_iter, dist, group)
    return shard.to_host(x)


class CudaShard:
    """A row block on this rank's GPU, driven through the C ABI.

    With one_pass (the default) every iteration computes the block's partial
    update in one pass over its rows (partial_update), which reads no CSC, so
    the context is built without one (MLEM_FLAG_NO_CSC: half the device
    memory, and the block's column sums by atomics).  With one_pass=False
    the shard offers only the two passes (project_correl, then backproject
    over the CSC).  The one-pass update takes the caller's sinogram block, so
    it walks every row of the block, those without counts included."""

    def __init__(self, block: RowBlock, n_cols: int, sino_block: np.ndarray, device: int,
                 flags: int = 0, one_pass: bool = True, grid=None):
        import torch

        self.torch = torch
        self.device = torch.device("cuda", device)
        self.n_cols = n_cols
        self.n_rows = block.end - block.start
        if one_pass:
            flags |= api.FLAG_NO_CSC
        else:
            self.partial_update = None  # iterate() then takes the two passes
        # grid (nx, ny, nz): the device keeps the image in Morton order, as a
        # whole-matrix context of that geometry does
        self.ctx = api.Context(block.row_end, block.elems, self.n_rows, n_cols, flags, device, grid)
        self.stream = torch.cuda.current_stream(self.device)
        self.ctx.set_stream(self.stream.cuda_stream)
        s = np.ascontiguousarray(sino_block, np.int32)
        if s.size != self.n_rows:
            raise api.MlemError(api.MLEM_ERR_INVALID, "sinogram block size differs from the rows")
        self.sino = torch.from_numpy(s).to(self.device)
        self._sumin = float(np.sum(s, dtype=np.float64))
        if one_pass and self.n_rows:
            # the block's counts also in the context, whose one-pass update then
            # leaves out the rows without counts
            self.ctx.set_sinograms(s)
        self.correl = torch.zeros(max(self.n_rows, 1), dtype=torch.float32, device=self.device)
        self.update = torch.zeros(n_cols, dtype=torch.float32, device=self.device)

    def local_norm(self):
        return self.torch.from_numpy(self.ctx.column_sums()).to(self.device)

    def set_norm(self, norm):
        self.ctx.set_norm_d(norm.data_ptr(), self.stream.cuda_stream)

    def local_count_sum(self) -> float:
        return self._sumin

    def project_correl(self, x):
        if self.n_rows:
            self.ctx.fwproj_correl_d(x.data_ptr(), self.sino.data_ptr(), self.correl.data_ptr(), 1,
                                     self.stream.cuda_stream)
        return self.correl

    def backproject(self, correl):
        if self.n_rows:
            self.ctx.bkproj_d(correl.data_ptr(), self.update.data_ptr(), 1, self.stream.cuda_stream)
        else:
            self.update.zero_()
        return self.update

    def set_sinogram(self, sino_block) -> None:
        """New counts for the block (host array, pinned or not)."""
        s = np.ascontiguousarray(sino_block, np.int32)
        if s.size != self.n_rows:
            raise api.MlemError(api.MLEM_ERR_INVALID, "sinogram block size differs from the rows")
        self.sino.copy_(self.torch.from_numpy(s), non_blocking=True)
        self._sumin = float(np.sum(s, dtype=np.float64))
        if getattr(self, "partial_update", None) is not None and self.n_rows:
            self.ctx.set_sinograms(s)

    def partial_update(self, x):
        """The block's partial update A_b^T calcCorrel(s_b, A_b x) in one pass
        over its rows (the one-pass kernels), from the block's counts held by
        the context (its rows without counts are left out)."""
        if self.n_rows:
            self.ctx.fused_update_d(x.data_ptr(), 0, self.update.data_ptr(), 1,
                                    self.stream.cuda_stream)
        else:
            self.update.zero_()
        return self.update

    def apply(self, update, x):
        self.ctx.apply_update_d(update.data_ptr(), x.data_ptr(), 1, self.stream.cuda_stream)

    def fill(self, value: float):
        return self.torch.full((self.n_cols,), value, dtype=self.torch.float32, device=self.device)

    def to_host(self, x) -> np.ndarray:
        return x.detach().cpu().numpy()

    def close(self):
        self.ctx.close()
