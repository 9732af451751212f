"""GPU checks at full size: the plain-full workload (4,194,304 LORs x 1,048,576 voxels,
7.8e8 elements) and the 16-frame batch on the same matrix, too large for the oracle to
finish in seconds.  They rest on a property that holds at any size: MLEM keeps the counts.

calcUpdate (seqcsr4mlem.cpp:123-134) sets x_j <- x_j u_j / norm_j with the back projection
u_j = sum_i a_ij s_i / f_i and f_i = sum_j a_ij x_j, so after every iteration
sum_j norm_j x_j = sum_i s_i over the rows with f_i != 0.  A row with counts adds a positive
term to every voxel it crosses, so those voxels stay positive and its f_i never becomes 0:
the identity covers every count.  Float rounding moves it by about 2e-8 on the oracle's
small cases (relative); the tolerance here is 1e-6.  The methods' images are also compared
with each other at the parity tolerance (1e-4 relative L2).
"""
import numpy as np
import pytest

from mlem_b200 import api, synth

import oracle_bind as ob

pytestmark = pytest.mark.gpu

TOL_COUNTS = 1e-6
TOL_MLEM = 1e-4

METHODS = {
    "fused/chunked": dict(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                          visit=api.VISIT_SORTED_CHUNKED),
    "fused/staged": dict(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                         visit=api.VISIT_SORTED_STAGED),
    "atomic/sorted": dict(bk_mode=api.BK_ATOMIC, group=32, frame_tile=1, blocks_per_sm=8,
                          visit=api.VISIT_SORTED),
    "csc/file": dict(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8,
                     visit=api.VISIT_FILE),
    "csc/sorted": dict(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8,
                       visit=api.VISIT_SORTED),
    "region": dict(bk_mode=api.BK_REGION, group=32, frame_tile=1, blocks_per_sm=8,
                   visit=api.VISIT_FILE),
}


@pytest.fixture(scope="module")
def full():
    w = synth.WORKLOADS["plain-full"]
    ctx = api.Context.siddon(w.geometry)
    frames = synth.make_frames(w, ctx.project_f64)
    norm = ctx.column_sums().astype(np.float64)
    yield ctx, frames.sinograms.astype(np.int32), norm
    ctx.close()


def counts_error(norm, x, sino):
    """Relative difference of sum_j norm_j x_j and sum_i s_i, per frame."""
    kept = x.astype(np.float64) @ norm
    total = sino.astype(np.float64).sum(axis=1)
    return np.abs(kept - total) / total


def test_full_size_methods_keep_the_counts_and_agree(full):
    ctx, sino, norm = full
    ctx.set_sinograms(sino)
    images = {}
    for name, t in METHODS.items():
        ctx.set_tuning(**t)
        ctx.init_images()
        for k in range(3):
            ctx.iterate(1)
            err = counts_error(norm, ctx.get_images(), sino)
            assert err.max() <= TOL_COUNTS, (name, k, err)
        images[name] = ctx.get_images()[0]
    ref = images["csc/file"]
    for name, img in images.items():
        assert ob.rel_l2(img, ref) <= TOL_MLEM, name


def test_full_size_projections_are_adjoint(full):
    """<A x, y> = <x, A^T y> for the device projections at full size (float32 kernels,
    the inner products in float64), and A^T 1 equals the column sums."""
    ctx, _, norm = full
    rng = np.random.default_rng(5)
    x = rng.random(ctx.n_cols, dtype=np.float32)
    y = rng.random(ctx.n_rows, dtype=np.float32)
    lhs = ctx.fwproj(x).astype(np.float64) @ y.astype(np.float64)
    rhs = x.astype(np.float64) @ ctx.bkproj(y).astype(np.float64)
    assert abs(lhs - rhs) <= 1e-6 * abs(rhs)
    ones = ctx.bkproj(np.ones(ctx.n_rows, np.float32))
    assert ob.rel_l2(ones, norm) <= 1e-6


def test_full_size_deterministic_method_repeats_to_the_bit(full):
    """The CSC method over the cut copy of the CSC in visiting order, twice from the same
    start: the same image to the bit (the copy holds 7.8e8 x 0.75 entries here)."""
    ctx, sino, norm = full
    ctx.set_sinograms(sino)
    ctx.set_tuning(**METHODS["csc/sorted"])
    runs = []
    for _ in range(2):
        ctx.init_images()
        ctx.iterate(4)
        runs.append(ctx.get_images())
    assert runs[0].tobytes() == runs[1].tobytes()
    assert counts_error(norm, runs[0], sino).max() <= TOL_COUNTS


def test_full_size_batch_of_16_keeps_every_frames_counts(full):
    """The 16-frame workload in one pass over the matrix per iteration (frame tile 16),
    and each frame against its own single-frame run of the same method."""
    ctx, _, norm = full
    wb = synth.WORKLOADS["batched-b16"]
    sinos = synth.make_frames(wb, ctx.project_f64).sinograms.astype(np.int32)
    ctx.set_sinograms(sinos)
    ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=16, blocks_per_sm=4,
                   visit=api.VISIT_SORTED_STAGED)
    ctx.init_images()
    ctx.iterate(2)
    x = ctx.get_images()
    assert counts_error(norm, x, sinos).max() <= TOL_COUNTS
    for b in (0, 7, 15):
        ctx.set_sinograms(sinos[b:b + 1])
        ctx.set_tuning(**METHODS["fused/staged"])
        ctx.init_images()
        ctx.iterate(2)
        assert ob.rel_l2(x[b], ctx.get_images()[0]) <= TOL_MLEM, b


def test_full_size_streamed_steps_keep_each_steps_counts(full):
    """mlem_stream_host at full size, a different sinogram each step (four steps, so the
    last one runs on the second buffer set): each step's image keeps that step's counts."""
    ctx, sino, norm = full
    rng = np.random.default_rng(11)
    steps = [sino[0]] + [rng.poisson(sino[0]).astype(np.int32) for _ in range(3)]
    ctx.set_sinograms(sino)
    ctx.set_tuning(**METHODS["fused/chunked"])
    ctx.init_images()
    got = [np.zeros((1, ctx.n_cols), np.float32) for _ in steps]
    ctx.stream_host([s[None] for s in steps], got)
    for k, (s, x) in enumerate(zip(steps, got)):
        assert counts_error(norm, x, s[None]).max() <= TOL_COUNTS, k
    ctx.iterate(1)  # the context continues on the last step's sinogram
    assert counts_error(norm, ctx.get_images(), steps[-1][None]).max() <= TOL_COUNTS
