"""Uneven multi-matrix batches (mlem_batch_*): several matrices of different
size and frame count iterated by one persistent kernel per iteration.

Every frame of every context must match the oracle's own run of that
(matrix, sinogram) within relative L2 1e-4, whatever the schedule (work-item
granularity, resident blocks, frame tile).
"""
import numpy as np
import pytest

from mlem_b200 import api

import oracle_bind as ob

pytestmark = pytest.mark.gpu

TOL_MLEM = 1e-4
ITERS = 10
# (golden case, frames): padded frame counts 16, 8 and 4 -- three matrices of
# different size, like a batch over three scanner geometries
MEMBERS = (("plain_small_it10", 4), ("tiny_it10", 12), ("edge_it7", 8))


def _frames(sino, B, seed):
    rng = np.random.default_rng(seed)
    return np.stack([sino if b == 0 else rng.permutation(sino) for b in range(B)]).astype(np.int32)


@pytest.fixture(scope="module")
def members(golden):
    out = []
    for i, (name, B) in enumerate(MEMBERS):
        m, sino, _, _, _ = golden.case(name)
        sinos = _frames(sino, B, 17 + i)
        want = np.stack([ob.mlem(m, sinos[b], ITERS)[0] for b in range(B)])
        out.append((m, sinos, want))
    return out


def _contexts(members, flags=0):
    ctxs = []
    for m, sinos, _ in members:
        c = api.Context.from_matrix(m, flags=flags)
        c.set_sinograms(sinos)
        c.init_images()
        ctxs.append(c)
    return ctxs


def _check(ctxs, members):
    for c, (m, sinos, want) in zip(ctxs, members):
        got = c.get_images()
        for b in range(sinos.shape[0]):
            assert ob.rel_l2(got[b], want[b]) <= TOL_MLEM, (m.n_rows, b)


IL, IT = api.BATCH_INTERLEAVED, api.BATCH_ITEMS
FILE, SORTED, STAGED = api.VISIT_FILE, api.VISIT_SORTED, api.VISIT_SORTED_STAGED


@pytest.mark.parametrize("policy,items_per_block,blocks_per_sm,tile,visit", [
    (IL, 4, 4, 0, FILE), (IL, 1, 3, 1, SORTED), (IL, 1, 8, 4, FILE), (IL, 1, 4, 2, SORTED),
    (IT, 4, 4, 0, FILE), (IT, 1, 3, 4, SORTED), (IT, 32, 4, 2, SORTED), (IT, 2, 1, 1, FILE),
    (IT, 1024, 8, 4, SORTED), (IT, 16, 4, 4, SORTED),
    (IT, 4, 4, 0, STAGED), (IT, 1, 3, 1, STAGED), (IT, 64, 8, 4, STAGED), (IT, 1024, 4, 2, STAGED)])
def test_batch_matches_oracle(members, policy, items_per_block, blocks_per_sm, tile, visit):
    ctxs = _contexts(members)
    try:
        with api.Batch(ctxs) as b:
            b.set_schedule(policy, items_per_block, blocks_per_sm, tile, visit)
            sched = b.schedule()
            assert sched["policy"] == policy and sched["visit"] == visit
            if policy == api.BATCH_ITEMS:
                assert sched["n_items"] >= len(ctxs)
            if tile:
                assert sched["frame_tile"] == tile
            b.iterate(ITERS)
        _check(ctxs, members)
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("policy,visit", [(IT, SORTED), (IT, STAGED), (IL, FILE)])
@pytest.mark.parametrize("tiles", [[4, 16, 8], [1, 4, 2], [2, 0, 1], [0, 2, 0]])
def test_batch_tiles_per_context(members, policy, visit, tiles):
    """Contexts with frame tiles of their own (padded frame counts 4, 16, 8):
    one kernel per tile group, every image equal to the oracle's."""
    ctxs = _contexts(members)
    try:
        with api.Batch(ctxs) as b:
            b.set_schedule(policy, 4, 4, 4, visit)
            b.set_tiles(tiles)
            assert b.tiles() == [t if t else 4 for t in tiles]
            b.iterate(ITERS)
            assert b.schedule()["tiles"] == [t if t else 4 for t in tiles]
            _, _, launches = b.profile(1)
            assert launches[0] == len(set(t if t else 4 for t in tiles))
            ctxs_again = _contexts(members)  # fresh images: the profile ran one iteration
            for c, c2 in zip(ctxs, ctxs_again):
                c.set_images(c2.get_images())
                c2.close()
            b.iterate(ITERS)
            b.set_schedule(policy, 4, 4, 2, visit)  # a batch tile again: every context follows it
            assert b.tiles() == [2, 2, 2]
        _check(ctxs, members)
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("policy,batch_visit,visits,tiles", [
    (IT, SORTED, [STAGED, SORTED, FILE], [0, 0, 0]),
    (IT, SORTED, [-1, STAGED, -1], [4, 4, 2]),
    (IT, STAGED, [FILE, -1, SORTED], [4, 0, 4]),
    (IL, SORTED, [FILE, SORTED, -1], [0, 0, 0]),
    (IL, FILE, [SORTED, -1, SORTED], [1, 4, 2]),
])
def test_batch_visits_per_context(members, policy, batch_visit, visits, tiles):
    """Contexts with row visits of their own: one kernel per (frame tile,
    visit) group, every image equal to the oracle's."""
    ctxs = _contexts(members)
    try:
        with api.Batch(ctxs) as b:
            b.set_schedule(policy, 4, 4, 4, batch_visit)
            b.set_tiles(tiles)
            b.set_visits(visits)
            eff_v = [v if v >= 0 else batch_visit for v in visits]
            eff_t = [t if t else 4 for t in tiles]
            assert b.visits() == eff_v and b.tiles() == eff_t
            assert b.schedule()["visits"] == eff_v
            b.iterate(ITERS)
            _, _, launches = b.profile(1)
            assert launches[0] == len(set(zip(eff_t, eff_v)))
            b.set_schedule(policy, 4, 4, 0, FILE)  # a batch visit again: every context follows it
            assert b.visits() == [FILE] * 3
        for c, (m, sinos, want) in zip(ctxs, members):  # the profiled iteration is one more
            want1 = np.stack([ob.mlem(m, sinos[f], ITERS + 1)[0] for f in range(sinos.shape[0])])
            got = c.get_images()
            for f in range(sinos.shape[0]):
                assert ob.rel_l2(got[f], want1[f]) <= TOL_MLEM, (m.n_rows, f)
    finally:
        for c in ctxs:
            c.close()


def test_batch_sums_and_chunking(members):
    """70 iterations (one 64-iteration graph plus 6 single launches) give
    the same images as 70 iterations of each context on its own, and the
    returned sums are the image sums."""
    ctxs = _contexts(members)
    solo = _contexts(members)
    try:
        with api.Batch(ctxs) as b:
            sums = b.iterate(70)
        for c, s, own in zip(ctxs, sums, solo):
            own.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=4, blocks_per_sm=8)
            own_sums, _, _ = own.iterate(70)
            a, w = c.get_images(), own.get_images()
            assert s.shape == (70, c.n_frames)
            for f in range(c.n_frames):
                assert ob.rel_l2(a[f], w[f]) <= TOL_MLEM
                np.testing.assert_allclose(s[:, f], own_sums[:, f], rtol=1e-4)
                assert abs(s[-1, f] - a[f].astype(np.float64).sum()) <= 1e-6 * abs(s[-1, f])
    finally:
        for c in ctxs + solo:
            c.close()


def test_batch_autotune_restores_images(members):
    ctxs = _contexts(members)
    try:
        before = [c.get_images() for c in ctxs]
        with api.Batch(ctxs) as b:
            sched = b.autotune()
            assert sched["ms_per_iter"] > 0
            assert sched["frame_tile"] in (1, 2, 4)  # must divide 4, 8 and 16
            for t, padded in zip(sched["tiles"], (4, 16, 8)):
                assert t in (1, 2, 4, 8, 16) and padded % t == 0
            for v in sched["visits"]:
                assert v in (FILE, SORTED) or (v == STAGED and sched["policy"] == IT)
            for c, x in zip(ctxs, before):
                assert c.get_images().tobytes() == x.tobytes()
            b.iterate(ITERS)
        _check(ctxs, members)
    finally:
        for c in ctxs:
            c.close()


def test_batch_follows_new_sinograms(members):
    """A context given other frames after the batch was made is picked up
    (new buffers, new frame count, new schedule) at the next iterate."""
    ctxs = _contexts(members)
    try:
        with api.Batch(ctxs) as b:
            b.iterate(2)
            m, sinos, want = members[0]
            ctxs[0].set_sinograms(sinos[:2])
            ctxs[0].init_images()
            b.iterate(ITERS)
            got = ctxs[0].get_images()
            for f in range(2):
                assert ob.rel_l2(got[f], want[f]) <= TOL_MLEM
    finally:
        for c in ctxs:
            c.close()


def test_batch_rejects_bad_input(members):
    ctxs = _contexts(members)
    unsorted = _contexts(members[:1], flags=api.FLAG_NO_ROW_ORDER)[0]
    m = members[0][0]
    exact = api.Context.from_matrix(m, flags=api.FLAG_EXACT)
    exact.set_sinograms(members[0][1])
    exact.init_images()
    bare = api.Context.from_matrix(m)
    try:
        with pytest.raises(api.MlemError):
            api.Batch([ctxs[0], exact])
        with pytest.raises(api.MlemError):
            api.Batch([ctxs[0], bare])  # no sinograms
        with pytest.raises(api.MlemError):
            api.Batch([ctxs[0], ctxs[0]])
        with pytest.raises(api.MlemError):
            api.Batch([])
        with api.Batch(ctxs) as b:
            with pytest.raises(api.MlemError):
                b.set_schedule(api.BATCH_ITEMS, 4, 4, 8)  # does not divide the padded count 4
            with pytest.raises(api.MlemError):
                b.set_schedule(api.BATCH_ITEMS, 0, 4, 0)
            with pytest.raises(api.MlemError):
                b.set_schedule(api.BATCH_INTERLEAVED, 4, 0, 0)
            with pytest.raises(api.MlemError):
                b.set_schedule(api.BATCH_INTERLEAVED, 4, 4, 3)
            with pytest.raises(api.MlemError):
                b.set_schedule(7, 4, 4, 0)
            with pytest.raises(api.MlemError):
                b.set_schedule(IL, 4, 4, 0, 9)
            with pytest.raises(api.MlemError):  # a single-matrix order only
                b.set_schedule(IT, 4, 4, 0, api.VISIT_SORTED_CHUNKED)
            with pytest.raises(api.MlemError):  # staged: the items schedule only
                b.set_schedule(IL, 4, 4, 0, STAGED)
            with pytest.raises(api.MlemError):  # 8 does not divide the padded count 4
                b.set_tiles([8, 0, 0])
            with pytest.raises(api.MlemError):
                b.set_tiles([4, 3, 0])
            with pytest.raises(api.MlemError):
                b.set_tiles([4, 4])
            b.set_schedule(IL, 4, 4, 0, FILE)
            with pytest.raises(api.MlemError):  # staged: the items schedule only
                b.set_visits([STAGED, -1, -1])
            with pytest.raises(api.MlemError):
                b.set_visits([-1, 9, -1])
            with pytest.raises(api.MlemError):
                b.set_visits([-2, -1, -1])
            with pytest.raises(api.MlemError):  # a single-matrix order only
                b.set_visits([-1, -1, api.VISIT_SORTED_CHUNKED])
            with pytest.raises(api.MlemError):
                b.set_visits([-1, -1])
            assert b.visits() == [FILE] * 3
            b.iterate(ITERS)  # still usable after the rejected calls
        _check(ctxs, members)
        with api.Batch([unsorted] + ctxs[1:]) as b:
            with pytest.raises(api.MlemError):  # a context without a row order
                b.set_schedule(IL, 4, 4, 0, SORTED)
            with pytest.raises(api.MlemError):
                b.set_schedule(IT, 4, 4, 0, STAGED)
            with pytest.raises(api.MlemError):
                b.set_visits([SORTED, -1, -1])
            b.set_visits([FILE, SORTED, -1])  # the contexts with a row order may sort
            assert b.visits() == [FILE, SORTED, FILE]
    finally:
        for c in ctxs + [exact, bare, unsorted]:
            c.close()


@pytest.mark.parametrize("policy,visit", [(IT, SORTED), (IT, STAGED), (IL, SORTED)])
def test_batch_skips_rows_without_counts(members, policy, visit):
    """Sorted visits walk each context's rows with counts only; new sinograms
    with the same frame counts (the list rebuilt in place) are picked up."""
    ctxs = _contexts(members)
    rng = np.random.default_rng(21)
    try:
        with api.Batch(ctxs) as b:
            b.set_schedule(policy, 4, 4, 0, visit)
            for it in range(2):
                sinos = []
                for c, (m, s, _) in zip(ctxs, members):
                    s = s.copy()
                    s[:, rng.random(m.n_rows) < 0.5] = 0
                    c.set_sinograms(s)
                    c.init_images()
                    sinos.append(s)
                b.iterate(ITERS)
                for c, (m, _, _), s in zip(ctxs, members, sinos):
                    got = c.get_images()
                    for f in range(s.shape[0]):
                        want, _ = ob.mlem(m, s[f], ITERS)
                        assert ob.rel_l2(got[f], want) <= TOL_MLEM, (it, m.n_rows, f)
    finally:
        for c in ctxs:
            c.close()
