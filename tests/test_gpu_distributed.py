"""Row-sharded MLEM (mlem_b200.distributed) on the GPU.

The multi-GPU scheme of mlem_mpi/fusedmpimlem.cpp:195-236: nnz-balanced row
blocks, a replicated image, one sum-reduction of the partial update per
iteration.  With one GPU per test run, the shards' arithmetic (CudaShard over
the device-pointer entry points) is checked two ways:
* two row blocks on the same GPU, their partial updates summed in-process --
  the numbers a two-GPU run all-reduces;
* the real torch.distributed driver over NCCL with a single rank.
Both must match the oracle's run of the whole matrix within relative L2 1e-4.
"""
import socket

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

TOL_MLEM = 1e-4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_row_blocks_sum_to_the_whole_matrix(golden):
    torch = pytest.importorskip("torch")
    from mlem_b200 import distributed

    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    starts, ends = distributed.partition(m.row_end, 2)
    shards = []
    try:
        for a, b in zip(starts, ends):
            blk = distributed.row_block(m.row_end, m.elems, int(a), int(b))
            shards.append(distributed.CudaShard(blk, m.n_cols, sino[int(a):int(b)], 0))
        norm = shards[0].local_norm() + shards[1].local_norm()
        for s in shards:
            s.set_norm(norm)
        sumin = sum(s.local_count_sum() for s in shards)
        sumnorm = 0.0
        for v in norm.cpu().numpy().tolist():
            sumnorm += v
        init = float(np.float32(sumin / sumnorm))
        xs = [s.fill(init) for s in shards]
        for it in range(iters):
            # both ways a shard computes its partial update: two passes, or one
            updates = [(s.backproject(s.project_correl(x)) if it % 2 else s.partial_update(x)).clone()
                       for s, x in zip(shards, xs)]
            total = updates[0] + updates[1]  # what the all-reduce delivers to every rank
            for s, x in zip(shards, xs):
                s.apply(total, x)
        torch.cuda.synchronize()
        a, b = (s.to_host(x) for s, x in zip(shards, xs))
        assert a.tobytes() == b.tobytes()  # every rank applies the identical update
        want, _ = ob.mlem(m, sino, iters)
        assert ob.rel_l2(a, want) <= TOL_MLEM
        assert ob.rel_l2(a, gold) <= TOL_MLEM
    finally:
        for s in shards:
            s.close()


def test_nccl_driver_single_rank(golden):
    torch = pytest.importorskip("torch")
    import torch.distributed as dist

    from mlem_b200 import distributed

    m, sino, iters, gold, _ = golden.case("tiny_it10")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1)
    shard = None
    try:
        torch.cuda.set_device(0)
        starts, ends = distributed.partition(m.row_end, 1)
        blk = distributed.row_block(m.row_end, m.elems, int(starts[0]), int(ends[0]))
        shard = distributed.CudaShard(blk, m.n_cols, sino, 0)
        img = distributed.reconstruct(shard, iters, dist)
        want, _ = ob.mlem(m, sino, iters)
        assert ob.rel_l2(img, want) <= TOL_MLEM
    finally:
        if shard is not None:
            shard.close()
        dist.destroy_process_group()


def test_fused_update_from_the_context_sinogram(golden):
    """mlem_fused_update_d with sino NULL takes the context's own counts and
    leaves out the rows without counts: equal to the update from the same
    counts passed explicitly (every row walked) up to the order of the
    float atomics."""
    torch = pytest.importorskip("torch")
    from mlem_b200 import api

    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    rng = np.random.default_rng(4)
    s = np.ascontiguousarray(sino, np.int32).copy()
    s[rng.random(m.n_rows) < 0.4] = 0
    dev = torch.device("cuda", 0)
    with api.Context.from_matrix(m, flags=api.FLAG_NO_CSC) as ctx:
        ctx.set_sinograms(s)
        x = torch.from_numpy(rng.uniform(0.5, 2.0, m.n_cols).astype(np.float32)).to(dev)
        sd = torch.from_numpy(s).to(dev)
        u_own = torch.zeros(m.n_cols, dtype=torch.float32, device=dev)
        u_arg = torch.zeros_like(u_own)
        st = torch.cuda.current_stream().cuda_stream
        ctx.fused_update_d(x.data_ptr(), 0, u_own.data_ptr(), 1, st)
        ctx.fused_update_d(x.data_ptr(), sd.data_ptr(), u_arg.data_ptr(), 1, st)
        torch.cuda.synchronize()
        assert ob.rel_l2(u_own.cpu().numpy(), u_arg.cpu().numpy()) <= 1e-6
        want = ob.bkproj(m, ob.correl(ob.fwproj(m, x.cpu().numpy()), s))
        assert ob.rel_l2(u_own.cpu().numpy(), want) <= 1e-5
        with pytest.raises(api.MlemError):  # the context holds one frame
            ctx.fused_update_d(x.data_ptr(), 0, u_own.data_ptr(), 2, st)
