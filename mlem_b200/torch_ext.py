"""Differentiable MLEM for PyTorch over the same C ABI.

* `forward_project(x, ctx)`: y = A x as a torch.autograd.Function whose
  backward is the hand-written back-projection kernel (A^T g), and
  `back_project(y, ctx)` the converse.  x is float32 [C] or [B, C] on the
  context's GPU; work runs on torch's current stream.
* `unrolled_mlem(x0, omega, sino, ctx)`: K relaxed MLEM iterations
      x_{k+1} = x_k * r_k ** omega_k,  r_k = calcUpdate factor(A^T (s / A x_k), norm)
  (omega_k = 1 is the reference iteration, mlem_seq/seqcsr4mlem.cpp:163-167)
  with gradients with respect to x0 and omega.  The forward pass keeps, per
  iteration, the row sums A x_k and the update factor r_k (K x (R + C)
  floats) when they fit `keep_bytes`; the backward pass then propagates the
  adjoint through calcCorrel and both projections in one pass over the
  matrix per iteration.  Otherwise it keeps only the K images x_k
  (per-iteration checkpoints) and first recomputes A x_k and A^T(s / A x_k)
  from them in one more pass.  A context with MLEM_FLAG_MIRROR_KERNELS runs
  the same arithmetic as separate projections.

Zero rules follow the reference: the correlation is 0 where the projection
is 0 (calcCorrel), the update factor is the raw back projection where the
column sum is 0 (calcUpdate); where r_k == 0 the image entry is 0 and its
gradient with respect to omega_k is taken as 0.
"""
from __future__ import annotations

import torch

from . import api


def _check(x: torch.Tensor, n: int, what: str) -> torch.Tensor:
    if not x.is_cuda or x.dtype != torch.float32:
        raise api.MlemError(api.MLEM_ERR_INVALID, f"{what} must be a float32 CUDA tensor")
    if x.shape[-1] != n:
        raise api.MlemError(api.MLEM_ERR_INVALID, f"{what} has {x.shape[-1]} entries, expected {n}")
    return x


def _frames(x: torch.Tensor):
    """[C] -> ([C, 1], 1); [B, C] -> ([C, B] interleaved, B)."""
    if x.dim() == 1:
        return x.contiguous().view(-1, 1), 1
    return x.t().contiguous(), x.shape[0]


def _unframes(y: torch.Tensor, B: int, batched: bool):
    return y.view(-1) if not batched else y.t().contiguous()


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _fw(ctx: "api.Context", x: torch.Tensor) -> torch.Tensor:
    xi, B = _frames(_check(x, ctx.n_cols, "image"))
    y = torch.empty((ctx.n_rows, B), dtype=torch.float32, device=x.device)
    ctx.fwproj_d(xi.data_ptr(), y.data_ptr(), B, _stream())
    return _unframes(y, B, x.dim() > 1)


def _bk(ctx: "api.Context", y: torch.Tensor) -> torch.Tensor:
    yi, B = _frames(_check(y, ctx.n_rows, "projection"))
    x = torch.empty((ctx.n_cols, B), dtype=torch.float32, device=y.device)
    ctx.bkproj_d(yi.data_ptr(), x.data_ptr(), B, _stream())
    return _unframes(x, B, y.dim() > 1)


class _ForwardProject(torch.autograd.Function):
    @staticmethod
    def forward(fctx, x, ctx):
        fctx.mctx = ctx
        return _fw(ctx, x)

    @staticmethod
    def backward(fctx, g):
        return _bk(fctx.mctx, g.contiguous()), None


class _BackProject(torch.autograd.Function):
    @staticmethod
    def forward(fctx, y, ctx):
        fctx.mctx = ctx
        return _bk(ctx, y)

    @staticmethod
    def backward(fctx, g):
        return _fw(fctx.mctx, g.contiguous()), None


def forward_project(x: torch.Tensor, ctx: "api.Context") -> torch.Tensor:
    return _ForwardProject.apply(x, ctx)


def back_project(y: torch.Tensor, ctx: "api.Context") -> torch.Tensor:
    return _BackProject.apply(y, ctx)


def norm_tensor(ctx: "api.Context", device) -> torch.Tensor:
    return torch.from_numpy(ctx.column_sums()).to(device)


def _mirrored(ctx) -> bool:
    """A context with MLEM_FLAG_MIRROR_KERNELS applies the mirrors inside its
    projection kernels; the one-pass backward kernels walk full rows only."""
    return bool(ctx.info.flags & api.FLAG_MIRROR_KERNELS)


def _ratio_rows(ctx, x, sino_i, norm):
    """calcUpdate factor of A^T (s / A x) and the row sums f = A x (0 for the
    rows without a count), in one pass over the matrix (mlem_ratio_rows_d).
    A mirrored context takes the fused update and a separate forward
    projection instead (f is then A x on every row)."""
    u = torch.empty_like(x)
    if _mirrored(ctx):
        ctx.fused_update_d(x.data_ptr(), sino_i.data_ptr(), u.data_ptr(), 1, _stream())
        f = _fw(ctx, x)
    else:
        f = torch.empty(ctx.n_rows, dtype=torch.float32, device=x.device)
        ctx.ratio_rows_d(x.data_ptr(), sino_i.data_ptr(), f.data_ptr(), u.data_ptr(), _stream())
    r = torch.where(norm != 0, u / torch.where(norm != 0, norm, torch.ones_like(norm)), u)
    return r, f


def _adjoint(ctx, du, sino_i, f):
    """A^T df with df = -(A du) s / f^2 where the row has a count and f != 0:
    the adjoint of calcCorrel and both projections, in one pass
    (mlem_adjoint_update_d; a mirrored context: a forward and a back
    projection with df formed between them)."""
    du = du.contiguous()
    if _mirrored(ctx):
        dc = _fw(ctx, du)
        live = (sino_i != 0) & (f != 0)
        fs = torch.where(live, f, torch.ones_like(f))
        df = torch.where(live, -(dc * (sino_i.to(torch.float32) / fs)) / fs, torch.zeros_like(f))
        return _bk(ctx, df)
    out = torch.empty_like(du)
    ctx.adjoint_update_d(du.data_ptr(), sino_i.data_ptr(), f.data_ptr(), out.data_ptr(), _stream())
    return out


class _UnrolledMLEM(torch.autograd.Function):
    @staticmethod
    def forward(fctx, x0, omega, sino_f, norm, ctx, sino_i, keep):
        K = omega.shape[0]
        xs = [x0.detach()]
        rs, fs = [], []
        x = x0.detach().contiguous()
        for k in range(K):
            r, f = _ratio_rows(ctx, x, sino_i, norm)
            if keep:
                rs.append(r)
                fs.append(f)
            x = x * torch.where(r > 0, r.clamp_min(1e-38) ** omega[k], torch.zeros_like(r))
            xs.append(x)
        fctx.mctx = ctx
        fctx.sino_i = sino_i
        fctx.keep = keep
        saved = [torch.stack(xs[:-1]), omega, sino_f, norm, x]
        if keep:
            saved += [torch.stack(rs), torch.stack(fs)]
        fctx.save_for_backward(*saved)
        return x

    @staticmethod
    def backward(fctx, g):
        ctx = fctx.mctx
        saved = fctx.saved_tensors
        xs, omega, sino_f, norm = saved[:4]
        K = omega.shape[0]
        g = g.contiguous()
        d_omega = torch.zeros_like(omega)
        for k in range(K - 1, -1, -1):
            xk = xs[k].contiguous()
            if fctx.keep:  # kept by the forward pass
                r, f = saved[5][k], saved[6][k]
            else:  # recomputed from the checkpoint
                r, f = _ratio_rows(ctx, xk, fctx.sino_i, norm)
            pos = r > 0
            rs = torch.where(pos, r, torch.ones_like(r))
            p = torch.where(pos, rs ** omega[k], torch.zeros_like(r))  # r^w
            x_next = xk * p
            d_omega[k] = torch.sum(g * x_next * torch.where(pos, torch.log(rs), torch.zeros_like(r)))
            gx = g * p                                          # direct path
            dr = torch.where(pos, g * xk * omega[k] * rs ** (omega[k] - 1), torch.zeros_like(r))
            du = torch.where(norm != 0, dr / torch.where(norm != 0, norm, torch.ones_like(norm)), dr)
            # adjoint of A^T, of calcCorrel (c = s / f where f != 0: dc/df = -s / f^2,
            # formed as -(dc (s / f)) / f so that a tiny f never squares to 0; a row
            # with zero counts has c = 0 whatever f is: no gradient) and of A
            gx = gx + _adjoint(ctx, du, fctx.sino_i, f)
            g = gx
        return g, d_omega, None, None, None, None, None


def unrolled_mlem(x0: torch.Tensor, omega: torch.Tensor, sino: torch.Tensor,
                  ctx: "api.Context", norm: torch.Tensor | None = None,
                  keep_bytes: int = 2 << 30) -> torch.Tensor:
    """K = len(omega) relaxed MLEM iterations from x0 (float32 [C] CUDA).
    The forward pass keeps each iteration's row sums and update factor for
    the backward pass when they take at most keep_bytes (0: always
    recompute them)."""
    _check(x0, ctx.n_cols, "x0")
    if norm is None:
        norm = norm_tensor(ctx, x0.device)
    sino_i = sino.to(device=x0.device, dtype=torch.int32).contiguous()
    sino_f = sino_i.to(torch.float32)
    K = int(omega.shape[0])
    keep = K * (ctx.n_rows + ctx.n_cols) * 4 <= keep_bytes
    return _UnrolledMLEM.apply(x0, omega.to(device=x0.device, dtype=torch.float32), sino_f, norm,
                               ctx, sino_i, keep)
