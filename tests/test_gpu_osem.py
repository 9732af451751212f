"""Ordered subsets (mlem_set_subsets) on the GPU against the oracle's OSEM.

Rows r % S form subset r's sub-iteration; the image after every full
iteration must match oracle_osem (tests/test_osem_oracle.py pins it to the
reference binary for one subset) within relative L2 1e-4, for every row
visit of the one-pass method, several subset counts and frame tiles.
"""
import numpy as np
import pytest

from mlem_b200 import api

import oracle_bind as ob

pytestmark = pytest.mark.gpu

TOL = 1e-4
VISITS = [api.VISIT_FILE, api.VISIT_SORTED, api.VISIT_SORTED_CHUNKED, api.VISIT_SORTED_STAGED]


@pytest.fixture(scope="module")
def ctxs(golden):
    out = {}
    for name in ("tiny_it10", "edge_it7", "plain_small_it10"):
        m, sino, iters, gold, _ = golden.case(name)
        out[name] = (api.Context.from_matrix(m), m, sino, iters)
    yield out
    for c, *_ in out.values():
        c.close()


@pytest.mark.parametrize("name", ["tiny_it10", "edge_it7", "plain_small_it10"])
@pytest.mark.parametrize("S", [2, 4, 7])
@pytest.mark.parametrize("visit", VISITS)
def test_osem_matches_oracle(ctxs, name, S, visit):
    ctx, m, sino, iters = ctxs[name]
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4, visit=visit)
    ctx.set_subsets(S)
    try:
        assert ctx.subsets() == S
        ctx.init_images()
        sums, _, _ = ctx.iterate(iters)
        img = ctx.get_images()[0]
        want, want_sums = ob.osem(m, sino, iters, S)
        assert ob.rel_l2(img, want) <= TOL, ob.rel_l2(img, want)
        np.testing.assert_allclose(sums[:, 0], want_sums, rtol=1e-4)
    finally:
        ctx.set_subsets(1)


def test_subset_column_sums_bit_exact(ctxs):
    ctx, m, sino, iters = ctxs["plain_small_it10"]
    for S in (2, 5):
        ctx.set_subsets(S)
        for s in range(S):
            assert ctx.subset_column_sums(s).tobytes() == ob.subset_column_sums(m, S, s).tobytes()
    ctx.set_subsets(1)


@pytest.mark.parametrize("tile,visit", [(1, api.VISIT_SORTED), (2, api.VISIT_SORTED_STAGED),
                                        (4, api.VISIT_SORTED_CHUNKED), (4, api.VISIT_FILE)])
def test_osem_frames(ctxs, tile, visit):
    ctx, m, sino, iters = ctxs["plain_small_it10"]
    rng = np.random.default_rng(5)
    sinos = np.stack([sino if b == 0 else rng.permutation(sino) for b in range(4)]).astype(np.int32)
    ctx.set_sinograms(sinos)
    ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=tile, blocks_per_sm=4, visit=visit)
    ctx.set_subsets(3)
    try:
        ctx.init_images()
        ctx.iterate(5)
        got = ctx.get_images()
        for b in range(4):
            want, _ = ob.osem(m, sinos[b], 5, 3)
            assert ob.rel_l2(got[b], want) <= TOL
    finally:
        ctx.set_subsets(1)


def test_one_subset_and_back(ctxs):
    """set_subsets(1) is plain MLEM again; graph and step-by-step agree."""
    ctx, m, sino, iters = ctxs["tiny_it10"]
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                   visit=api.VISIT_SORTED_CHUNKED)
    ctx.set_subsets(4)
    ctx.set_subsets(1)
    ctx.init_images()
    ctx.iterate(iters)
    want, _ = ob.mlem(m, sino, iters)
    assert ob.rel_l2(ctx.get_images()[0], want) <= TOL
    ctx.set_subsets(4)
    ctx.init_images()
    ctx.iterate(iters)  # one captured graph
    a = ctx.get_images()[0]
    ctx.init_images()
    for _ in range(iters):
        ctx.iterate(1)
    b = ctx.get_images()[0]
    assert ob.rel_l2(a, b) <= 1e-5
    ctx.set_subsets(1)


def test_osem_without_csc_and_without_row_order(golden):
    m, sino, iters, _, _ = golden.case("plain_small_it10")
    want, _ = ob.osem(m, sino, iters, 4)
    for flags, visit in ((api.FLAG_NO_CSC, api.VISIT_SORTED_STAGED),
                         (api.FLAG_NO_ROW_ORDER, api.VISIT_FILE)):
        with api.Context.from_matrix(m, flags=flags) as ctx:
            ctx.set_sinograms(sino)
            ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                           visit=visit)
            ctx.set_subsets(4)
            ctx.init_images()
            ctx.iterate(iters)
            assert ob.rel_l2(ctx.get_images()[0], want) <= TOL


def test_osem_autotune_and_rejections(ctxs, golden):
    ctx, m, sino, iters = ctxs["plain_small_it10"]
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4)
    ctx.set_subsets(4)
    try:
        ctx.init_images()
        before = ctx.get_images()
        best = ctx.autotune()
        assert best["bk_mode"] == api.BK_FUSED
        assert ctx.get_images().tobytes() == before.tobytes()
        with pytest.raises(api.MlemError):
            ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1)
        with pytest.raises(api.MlemError):
            ctx.autotune(deterministic_only=True)
        with pytest.raises(api.MlemError):
            ctx.set_subsets(0)
        with pytest.raises(api.MlemError):
            ctx.subset_column_sums(4)
        with pytest.raises(api.MlemError):  # a batch runs plain MLEM only
            api.Batch([ctx])
        ctx.iterate(2)  # still usable
    finally:
        ctx.set_subsets(1)
    with pytest.raises(api.MlemError):
        ctx.set_subsets(m.n_rows + 1)
    with api.Context.from_matrix(m, flags=api.FLAG_EXACT) as ex:
        with pytest.raises(api.MlemError):
            ex.set_subsets(2)
    # switching to another method with one subset is allowed again
    ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1)


@pytest.mark.parametrize("visit", [api.VISIT_SORTED, api.VISIT_SORTED_CHUNKED, api.VISIT_SORTED_STAGED])
def test_osem_skips_rows_without_counts(golden, visit):
    """The sorted walks of every subset leave out its rows whose counts are
    zero; the lists follow new sinograms in place (graph kept), are built
    when subsets are set after the sinograms, and through mlem_step_host."""
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    rng = np.random.default_rng(21)
    s = np.ascontiguousarray(sino, np.int32).copy()
    dead = rng.random(m.n_rows) < 0.5
    s[dead] = 0
    S = 4
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(s)
        ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4, visit=visit)
        ctx.set_subsets(S)  # after the sinograms
        for it in range(2):
            ctx.init_images()
            ctx.iterate(3)
            want, _ = ob.osem(m, s, 3, S)
            assert ob.rel_l2(ctx.get_images()[0], want) <= TOL, it
            s = s.copy()  # other rows with counts: the lists are rebuilt in place
            s[~dead] = 0
            s[dead] = rng.poisson(30, int(dead.sum()))
            ctx.set_sinograms(s)
        x0 = np.full((1, m.n_cols), 0.5, np.float32)
        x = x0.copy()
        ctx.step_host(s, x)
        want, _ = ob.osem(m, s, 1, S, start_image=x0[0])
        assert ob.rel_l2(x[0], want) <= TOL
        ctx.set_subsets(1)
