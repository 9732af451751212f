"""Row-sharded MLEM orchestration on CPU: world_size-2 gloo process groups.

The product shard runs the CUDA library; here the same `reconstruct` loop
(partition, column-sum all-reduce, one update all-reduce per iteration) is
driven by a checker shard whose arithmetic is the oracle, so the
distributed plumbing is verified without a GPU.
"""
import datetime
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class OracleShard:
    def __init__(self, block, n_cols, sino_block):
        import torch

        import oracle_bind as ob
        from mlem_b200 import formats
        self.ob, self.torch = ob, torch
        self.n_cols = n_cols
        self.m = formats.Csr4(block.end - block.start, n_cols, block.row_end, block.elems)
        self.sino = np.ascontiguousarray(sino_block, np.int32)

    def local_norm(self):
        return self.torch.from_numpy(self.ob.column_sums(self.m))

    def set_norm(self, norm):
        self.norm = norm.numpy().copy()

    def local_count_sum(self):
        return float(np.sum(self.sino, dtype=np.float64))

    def project_correl(self, x):
        f = self.ob.fwproj(self.m, x.numpy())
        return self.torch.from_numpy(self.ob.correl(f, self.sino))

    def backproject(self, c):
        return self.torch.from_numpy(self.ob.bkproj(self.m, c.numpy()))

    def apply(self, u, x):
        x.copy_(self.torch.from_numpy(self.ob.update(u.numpy(), self.norm, x.numpy())))

    def fill(self, v):
        return self.torch.full((self.n_cols,), v, dtype=self.torch.float32)

    def to_host(self, x):
        return x.numpy().copy()


def _worker(rank, world, port, out_dir, mode):
    sys.path[:0] = [ROOT, HERE]
    import torch.distributed as dist

    import golden_cases
    from mlem_b200 import distributed

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    m, sino, iters, gold, _ = golden_cases.case("tiny_it10")
    starts, ends = distributed.partition(m.row_end, world)
    blk = distributed.row_block(m.row_end, m.elems, int(starts[rank]), int(ends[rank]))
    shard = OracleShard(blk, m.n_cols, sino[blk.start:blk.end])
    try:
        if mode == "die" and rank == 1:
            os._exit(3)  # a rank that never joins the first collective
        if mode == "pieces":
            # the benchmark's order: start image, warm-up, timed iterations,
            # then single steps
            x = distributed.init_image(shard, dist)
            distributed.iterate(shard, x, 2, dist)
            distributed.iterate(shard, x, iters - 5, dist)
            for _ in range(3):
                distributed.iterate(shard, x, 1, dist)
            img = shard.to_host(x)
        else:
            img = distributed.reconstruct(shard, iters, dist)
        np.save(os.path.join(out_dir, f"img{rank}.npy"), img)
        dist.barrier()
    except Exception as e:  # the surviving rank must see an error, not hang
        with open(os.path.join(out_dir, f"err{rank}.txt"), "w") as f:
            f.write(type(e).__name__ + ": " + str(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _launch(world, mode, tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), mode)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            raise AssertionError("worker did not finish")
    return ps


def test_row_sharded_mlem_matches_single_process(tmp_path, golden):
    import oracle_bind as ob
    _launch(2, "ok", tmp_path)
    m, sino, iters, gold, _ = golden.case("tiny_it10")
    a = np.load(tmp_path / "img0.npy")
    b = np.load(tmp_path / "img1.npy")
    assert a.tobytes() == b.tobytes()  # the replicated image is identical on every rank
    want, _ = ob.mlem(m, sino, iters, ftz=False)
    assert ob.rel_l2(a, want) <= 1e-5
    assert ob.rel_l2(a, gold) <= 1e-4


def test_partition_blocks_cover_the_matrix(golden):
    from mlem_b200 import distributed
    m, *_ = golden.case("plain_small_it10")
    for world in (2, 3, 8):
        s, e = distributed.partition(m.row_end, world)
        blocks = [distributed.row_block(m.row_end, m.elems, int(a), int(b)) for a, b in zip(s, e)]
        assert sum(len(bk.elems) for bk in blocks) == m.nnz
        rebuilt = np.concatenate([bk.elems for bk in blocks])
        assert rebuilt.tobytes() == np.ascontiguousarray(m.elems).tobytes()
        nnz = [len(bk.elems) for bk in blocks]
        assert max(nnz) - min(nnz) <= 2 * int(np.diff(m.row_ptr()).max()) + 1


def test_dead_rank_is_detected_not_hung(tmp_path):
    _launch(2, "die", tmp_path)
    err = tmp_path / "err0.txt"
    assert err.exists(), "rank 0 should have failed its collective"
    assert not (tmp_path / "img0.npy").exists()


def test_iterations_in_pieces_equal_one_reconstruction(tmp_path, golden):
    import oracle_bind as ob
    _launch(2, "pieces", tmp_path)
    m, sino, iters, gold, _ = golden.case("tiny_it10")
    a = np.load(tmp_path / "img0.npy")
    b = np.load(tmp_path / "img1.npy")
    assert a.tobytes() == b.tobytes()
    want, _ = ob.mlem(m, sino, iters, ftz=False)
    assert ob.rel_l2(a, want) <= 1e-5


def test_sequential_sum_is_the_reference_order():
    from mlem_b200 import distributed
    rng = np.random.default_rng(2)
    v = rng.uniform(0, 1e4, 100_001).astype(np.float32)
    acc = 0.0
    for t in v.tolist():
        acc += t
    assert distributed.sequential_sum(v) == acc
