"""Symmetry-compressed matrices with the mirrors applied in the kernels
(MLEM_FLAG_MIRROR_KERNELS, MLEM_BK_MIRRORED): only the stored elements live
on the device, and every result equals the full matrix's -- the matrix the
oracle regenerates as the reference's viewer does -- within the float
tolerance (the mirrored rows are summed with atomics)."""
import os
import subprocess

import numpy as np
import pytest
import torch

from mlem_b200 import api, formats

import oracle_bind as ob
from test_symmetry_oracle import GRID, SCANNER, sym_matrix

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "mlem_b200", "bin", "mlem_b200")
TOL = 1e-4
MK = api.FLAG_MIRROR_KERNELS


def _frames(m, B, seed):
    rng = np.random.default_rng(seed)
    return rng.poisson(20, (B, m.n_rows)).astype(np.int32)


def _full_dense(full):
    A = np.zeros((full.n_rows, full.n_cols), np.float64)
    rows = np.repeat(np.arange(full.n_rows), np.diff(np.concatenate([[0], full.row_end])).astype(np.int64))
    np.add.at(A, (rows, full.elems["index"].astype(np.int64)), full.elems["value"].astype(np.float64))
    return A


# grid (8, 8, 4): Morton codes, mirrors as XOR masks; (6, 8, 4): ranked Morton
# order, mirror tables; NATURAL_LAYOUT: natural order, mirror tables
LAYOUTS = [((8, 8, 4), 0), ((6, 8, 4), 0), ((8, 8, 4), api.FLAG_NATURAL_LAYOUT)]


@pytest.mark.parametrize("sym", [1, 2, 4, 5, 7])
@pytest.mark.parametrize("grid,flags", LAYOUTS)
def test_column_sums_and_mlem(sym, grid, flags):
    m = sym_matrix(sym, seed=60 + sym, grid=grid)
    full = ob.expand_symmetries(m)
    sino = _frames(m, 1, sym)[0]
    want, _ = ob.mlem(full, sino, 8)
    with api.Context.symmetric(m, flags=MK | flags) as ctx:
        assert ctx.nnz == m.nnz  # the stored elements only
        assert ob.rel_l2(ctx.column_sums(), ob.column_sums(full)) <= 1e-6
        ctx.set_sinograms(sino)
        ctx.init_images()
        ctx.iterate(8)
        assert ob.rel_l2(ctx.get_images()[0], want) <= TOL


def test_host_step_and_streamed_iterations():
    """mlem_step_host and mlem_stream_host on a mirrored context (the
    sinogram per iteration indexes the full matrix's rows): each iteration
    against the oracle's on the expanded matrix."""
    m = sym_matrix(7, seed=91, grid=(8, 8, 4))
    full = ob.expand_symmetries(m)
    B = 2
    sinos = [_frames(m, B, 100 + k) for k in range(4)]
    with api.Context.symmetric(m, flags=MK) as ctx:
        ctx.set_sinograms(sinos[0])
        init = ctx.init_images()
        cur = np.repeat(np.asarray(init, np.float32)[:, None], m.n_cols, axis=1)
        got = [np.zeros((B, m.n_cols), np.float32) for _ in sinos]
        ctx.stream_host(sinos, got)
        for k, s in enumerate(sinos):
            for b in range(B):
                want, _ = ob.mlem(full, s[b], 1, start_image=cur[b])
                assert ob.rel_l2(got[k][b], want) <= TOL, (k, b)
            cur = got[k]
        x = cur.copy()
        ctx.step_host(sinos[0], x)
        for b in range(B):
            want, _ = ob.mlem(full, sinos[0][b], 1, start_image=cur[b])
            assert ob.rel_l2(x[b], want) <= TOL, b


@pytest.mark.parametrize("B,tile", [(3, 1), (3, 4), (8, 2), (16, 16), (12, 8)])
@pytest.mark.parametrize("visit", [api.VISIT_FILE, api.VISIT_SORTED])
def test_frames_tiles_visits(B, tile, visit):
    m = sym_matrix(7, seed=70 + B, grid=(6, 8, 4))
    full = ob.expand_symmetries(m)
    sinos = _frames(m, B, B)
    with api.Context.symmetric(m, flags=MK) as ctx:
        ctx.set_sinograms(sinos)
        ctx.set_tuning(bk_mode=api.BK_MIRRORED, group=32, frame_tile=tile, blocks_per_sm=4,
                       visit=visit)
        ctx.init_images()
        ctx.iterate(6)
        got = ctx.get_images()
        for b in range(B):
            want, _ = ob.mlem(full, sinos[b], 6)
            assert ob.rel_l2(got[b], want) <= TOL, b


def test_projections_and_fused_update():
    m = sym_matrix(5, seed=81, grid=(6, 8, 4))
    full = ob.expand_symmetries(m)
    A = _full_dense(full)
    rng = np.random.default_rng(3)
    B = 4
    x = rng.uniform(0.5, 2.0, (B, m.n_cols)).astype(np.float32)
    y = rng.uniform(0.0, 1.0, (B, m.n_rows)).astype(np.float32)
    sino = _frames(m, B, 5)
    with api.Context.symmetric(m, flags=MK) as ctx:
        # host-buffer reference functions (one frame)
        f1 = api.calcFwProj(ctx, x[0], np.zeros(m.n_rows, np.float32))
        assert ob.rel_l2(f1, A @ x[0]) <= 1e-6
        u1 = api.calcBkProj(ctx, y[0], np.zeros(m.n_cols, np.float32))
        assert ob.rel_l2(u1, A.T @ y[0]) <= 1e-6
        # device-pointer entry points, B frames frame-interleaved
        xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
        yd = torch.from_numpy(np.ascontiguousarray(y.T)).cuda()
        out_r = torch.empty((m.n_rows, B), device="cuda")
        out_c = torch.empty((m.n_cols, B), device="cuda")
        ctx.fwproj_d(xd.data_ptr(), out_r.data_ptr(), B)
        torch.cuda.synchronize()
        assert ob.rel_l2(out_r.cpu().numpy().T, (A @ x.T.astype(np.float64)).T) <= 1e-6
        ctx.bkproj_d(yd.data_ptr(), out_c.data_ptr(), B)
        torch.cuda.synchronize()
        assert ob.rel_l2(out_c.cpu().numpy().T, (A.T @ y.T.astype(np.float64)).T) <= 1e-6
        sd = torch.from_numpy(np.ascontiguousarray(sino.T)).cuda()
        ctx.fwproj_correl_d(xd.data_ptr(), sd.data_ptr(), out_r.data_ptr(), B)
        f = A @ x.T.astype(np.float64)
        c = np.where(f != 0, sino.T / np.where(f != 0, f, 1), 0)
        torch.cuda.synchronize()
        assert ob.rel_l2(out_r.cpu().numpy(), c) <= 1e-5
        ctx.fused_update_d(xd.data_ptr(), sd.data_ptr(), out_c.data_ptr(), B)
        torch.cuda.synchronize()
        assert ob.rel_l2(out_c.cpu().numpy(), A.T @ c) <= 1e-5


def test_memory_and_refusals():
    m = sym_matrix(7, seed=91)
    sino = _frames(m, 1, 9)[0]
    with api.Context.symmetric(m, flags=api.FLAG_NO_CSC) as full_ctx, \
            api.Context.symmetric(m, flags=MK | api.FLAG_NO_CSC) as ctx:
        assert ctx.nnz * 4 < full_ctx.nnz  # sym 7: eight mirrors of every stored element
        ctx.set_sinograms(sino)
        ctx.init_images()
        assert ctx.tuning()["bk_mode"] == api.BK_MIRRORED
        with pytest.raises(api.MlemError):
            ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4)
        with pytest.raises(api.MlemError):  # the chunked walks are one-pass only
            ctx.set_tuning(bk_mode=api.BK_MIRRORED, group=32, frame_tile=1, blocks_per_sm=4,
                           visit=api.VISIT_SORTED_CHUNKED)
        with pytest.raises(api.MlemError):
            ctx.set_tuning(bk_mode=api.BK_MIRRORED, group=16, frame_tile=1, blocks_per_sm=4)
        with pytest.raises(api.MlemError):
            ctx.set_subsets(2)
        with pytest.raises(api.MlemError):
            ctx.project_f64(np.ones(m.n_cols, np.float32))
        with pytest.raises(api.MlemError):
            api.Batch([ctx])
        with pytest.raises(api.MlemError):
            ctx.autotune(deterministic_only=True)
        t = ctx.autotune()
        assert t["bk_mode"] == api.BK_MIRRORED and t["ms_per_iter"] > 0
        ctx.init_images()
        ctx.iterate(5)
        want, _ = ob.mlem(ob.expand_symmetries(m), sino, 5)
        assert ob.rel_l2(ctx.get_images()[0], want) <= TOL
    with pytest.raises(api.MlemError):  # bit-exact kernels need the full matrix
        api.Context.symmetric(m, flags=MK | api.FLAG_EXACT)
    with api.Context.from_matrix(m) as plain:
        with pytest.raises(api.MlemError):  # a context without mirrors
            plain.set_tuning(bk_mode=api.BK_MIRRORED, group=32, frame_tile=1, blocks_per_sm=4)


def test_file_flag_and_cli(tmp_path):
    m = sym_matrix(7, seed=101)
    path = str(tmp_path / "sym.csr4")
    formats.write_csr4(path, m.n_rows, m.n_cols, m.row_end, m.elems, grid=GRID, flags=7,
                       scanner=SCANNER)
    full = ob.expand_symmetries(m)
    with api.Context.from_file(path, flags=MK) as ctx:
        assert ctx.nnz == m.nnz
        assert ctx.tuning()["bk_mode"] == api.BK_MIRRORED
    with pytest.raises(api.MlemError):
        api.Context.from_file(path, flags=MK | api.FLAG_EXPAND_SYMMETRY)
    sino = _frames(m, 1, 11)[0]
    sp, out = str(tmp_path / "s.sino"), str(tmp_path / "img.out")
    formats.write_vector(sp, sino, np.int32)
    want, _ = ob.mlem(full, sino, 5)
    for tune in ("0", "1"):
        env = dict(os.environ, MLEM_B200_EXPAND_SYMMETRY="kernels", MLEM_B200_AUTOTUNE=tune)
        subprocess.run([CLI, path, sp, out, "5"], check=True, env=env, capture_output=True)
        assert ob.rel_l2(formats.read_vector(out, np.float32), want) <= TOL


def test_torch_projector_and_unrolled_mlem():
    """The torch extension over a mirrored context: forward and back projection
    equal the full matrix's, and the unrolled MLEM's forward pass equals the
    oracle's MLEM on the full matrix."""
    from mlem_b200 import torch_ext

    m = sym_matrix(7, seed=111, grid=(6, 8, 4))
    full = ob.expand_symmetries(m)
    A = _full_dense(full)
    sino = _frames(m, 1, 13)[0]
    with api.Context.symmetric(m, flags=MK) as ctx:
        x = torch.rand(m.n_cols, device="cuda", dtype=torch.float32, requires_grad=True)
        y = torch_ext.forward_project(x, ctx)
        assert ob.rel_l2(y.detach().cpu().numpy(), A @ x.detach().cpu().numpy().astype(np.float64)) <= 1e-6
        g = torch.rand(m.n_rows, device="cuda", dtype=torch.float32)
        (y * g).sum().backward()
        assert ob.rel_l2(x.grad.cpu().numpy(), A.T @ g.cpu().numpy().astype(np.float64)) <= 1e-6
        norm = ob.column_sums(full)
        x0 = torch.full((m.n_cols,), float(ob.init_value(norm, sino)), device="cuda")
        xk = torch_ext.unrolled_mlem(x0, torch.ones(4), torch.from_numpy(sino), ctx)
        want, _ = ob.mlem(full, sino, 4)
        assert ob.rel_l2(xk.detach().cpu().numpy(), want) <= TOL
