"""GPU parity: the CUDA path through the C ABI against the oracle and the
golden images of the reference binary.

Tolerances: bit-exact for index work (CSC transpose, generator, column sums,
MLEM_FLAG_EXACT runs); relative L2 <= 1e-4 for the fast float kernels after
the full iteration count (the tolerance the hot path is held to); 1e-5 for
a single projection.
"""
import numpy as np
import pytest

from mlem_b200 import api, formats, synth

import oracle_bind as ob
from golden_cases import CASES

pytestmark = pytest.mark.gpu

TOL_MLEM = 1e-4
TOL_PROJ = 1e-5


@pytest.fixture(scope="module")
def ctxs(golden):
    out = {}
    for name in CASES:
        m, sino, iters, gold, entry = golden.case(name)
        out[name] = (api.Context.from_matrix(m), m, sino, iters, gold)
    yield out
    for v in out.values():
        v[0].close()


@pytest.mark.parametrize("name", CASES)
def test_csc_transpose_bit_exact(ctxs, name):
    ctx, m, *_ = ctxs[name]
    col_ptr, ce = ctx.csc()
    cp_o, ce_o = ob.transpose(m)
    assert np.array_equal(col_ptr, cp_o)
    assert ce.tobytes() == ce_o.tobytes()


@pytest.mark.parametrize("name", CASES)
def test_csr_roundtrip(ctxs, name):
    ctx, m, *_ = ctxs[name]
    row_end, el = ctx.csr()
    assert np.array_equal(row_end, m.row_end)
    assert el.tobytes() == np.ascontiguousarray(m.elems).tobytes()


@pytest.mark.parametrize("name", CASES)
def test_column_sums_bit_exact(ctxs, name):
    ctx, m, *_ = ctxs[name]
    assert ctx.column_sums().tobytes() == ob.column_sums(m).tobytes()


@pytest.mark.parametrize("name", CASES)
def test_pieces_against_oracle(ctxs, name):
    ctx, m, sino, *_ = ctxs[name]
    rng = np.random.default_rng(3)
    x = rng.uniform(0.5, 2.0, m.n_cols).astype(np.float32)
    f, f_o = ctx.fwproj(x), ob.fwproj(m, x)
    assert ob.rel_l2(f, f_o) < TOL_PROJ
    c, c_o = ctx.correl(f_o, sino), ob.correl(f_o, sino)
    assert c.tobytes() == c_o.tobytes()  # elementwise IEEE divide: bit-exact
    u, u_o = ctx.bkproj(c_o), ob.bkproj(m, c_o)
    assert ob.rel_l2(u, u_o) < TOL_PROJ
    norm = ob.column_sums(m)
    xu, xu_o = ctx.update(u_o, norm, x), ob.update(u_o, norm, x)
    assert xu.tobytes() == xu_o.tobytes()
    assert ctx.init_value(sino) == ob.init_value(norm, sino)


MODES = [api.BK_CSC, api.BK_ATOMIC, api.BK_FUSED, api.BK_REGION]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("mode,visit", [(m, api.VISIT_FILE) for m in MODES] + [
    (api.BK_CSC, api.VISIT_SORTED), (api.BK_ATOMIC, api.VISIT_SORTED),
    (api.BK_FUSED, api.VISIT_SORTED), (api.BK_FUSED, api.VISIT_SORTED_CHUNKED),
    (api.BK_FUSED, api.VISIT_SORTED_STAGED)])
def test_mlem_matches_reference_image(ctxs, name, mode, visit):
    ctx, m, sino, iters, gold = ctxs[name]
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=mode, group=32, frame_tile=1, blocks_per_sm=8, visit=visit)
    ctx.init_images()
    sums, zeros, _ = ctx.iterate(iters)
    img = ctx.get_images()[0]
    err_ref = ob.rel_l2(img, gold)
    assert err_ref <= TOL_MLEM, err_ref
    ref64 = ob.mlem_f64(m, sino, iters)
    assert ob.rel_l2(img, ref64) <= TOL_MLEM
    assert abs(sums[-1, 0] - float(np.sum(img, dtype=np.float64))) <= 1e-9 * abs(sums[-1, 0]) + 1e-30
    assert zeros[-1, 0] == int((img == 0).sum())


@pytest.mark.parametrize("name", CASES)
def test_exact_mode_is_bit_exact_with_reference_binary(golden, name):
    m, sino, iters, gold, _ = golden.case(name)
    with api.Context.from_matrix(m, flags=api.FLAG_EXACT) as ctx:
        img, _ = api.mlem(ctx, sino, nIterations=iters)
        assert img[0].tobytes() == gold.tobytes()
        # the piecewise functions are bit-exact too
        x = np.full(m.n_cols, 1.5, np.float32)
        assert ctx.fwproj(x).tobytes() == ob.fwproj(m, x).tobytes()
        c = ob.correl(ob.fwproj(m, x), sino)
        assert ctx.bkproj(c).tobytes() == ob.bkproj(m, c).tobytes()


def test_csc_mode_is_deterministic(ctxs):
    ctx, m, sino, iters, gold = ctxs["plain_small_it10"]
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=api.BK_CSC, group=16, frame_tile=1, blocks_per_sm=4)
    ctx.init_images()
    ctx.iterate(iters)
    a = ctx.get_images()
    ctx.init_images()
    for _ in range(iters):
        ctx.iterate(1)
    b = ctx.get_images()
    assert a.tobytes() == b.tobytes()


def test_csc_in_visiting_order_is_deterministic(golden):
    """The CSC method with the sorted visit gathers the correlations by
    visiting position from a CSC in that order: reproducible to the bit, in
    one context or another, whole or step by step."""
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    imgs = []
    for _ in range(2):
        with api.Context.from_matrix(m) as ctx:
            ctx.set_sinograms(sino)
            ctx.set_tuning(bk_mode=api.BK_CSC, group=16, frame_tile=1, blocks_per_sm=4,
                           visit=api.VISIT_SORTED)
            ctx.init_images()
            ctx.iterate(iters)
            imgs.append(ctx.get_images())
            ctx.init_images()
            for _ in range(iters):
                ctx.iterate(1)
            imgs.append(ctx.get_images())
    assert all(x.tobytes() == imgs[0].tobytes() for x in imgs)
    assert ob.rel_l2(imgs[0][0], gold) <= TOL_MLEM


@pytest.mark.parametrize("tile", [1, 2])
def test_csc_in_visiting_order_skips_rows_without_counts(golden, tile):
    """The CSC method's forward pass over the CSC in visiting order walks only
    the rows with counts (the list rebuilt with every sinogram) and leaves the
    others' correlations 0: against the oracle with half the rows at zero
    counts, reproducible to the bit, and after a new sinogram of other zero
    rows through mlem_step_host."""
    m, sino, _, _, _ = golden.case("plain_small_it10")
    rng = np.random.default_rng(41)
    B = 2
    sinos = np.stack([rng.permutation(sino) for _ in range(B)]).astype(np.int32)
    dead = rng.random(m.n_rows) < 0.5
    sinos[:, dead] = 0
    imgs = []
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sinos)
        ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=tile, blocks_per_sm=4,
                       visit=api.VISIT_SORTED)
        for _ in range(2):
            ctx.init_images()
            ctx.iterate(6)
            imgs.append(ctx.get_images())
        assert imgs[0].tobytes() == imgs[1].tobytes()
        for b in range(B):
            want, _ = ob.mlem(m, sinos[b], 6)
            assert ob.rel_l2(imgs[0][b], want) <= TOL_MLEM, b
        other = sinos.copy()
        other[:, ~dead] = 0
        other[:, dead] = rng.poisson(20, (B, int(dead.sum())))
        x0 = np.full((B, m.n_cols), 0.5, np.float32)
        x = x0.copy()
        ctx.step_host(other, x)
        for b in range(B):
            want, _ = ob.mlem(m, other[b], 1, start_image=x0[b])
            assert ob.rel_l2(x[b], want) <= TOL_MLEM, b


@pytest.mark.parametrize("group,tile", [(32, 1), (16, 1), (32, 2)])
def test_csc_cut_copy_is_refilled_with_each_sinogram(golden, group, tile):
    """With sinograms set, the CSC method's back projection walks a copy of
    the CSC in visiting order cut to the rays with counts, refilled from the
    full CSC with every set of sinograms: after sinograms with other rows at
    zero counts, the images equal those of a fresh context, to the bit."""
    m, sino, _, _, _ = golden.case("plain_small_it10")
    rng = np.random.default_rng(5 + group + tile)
    B = tile
    first = np.stack([rng.permutation(sino) for _ in range(B)]).astype(np.int32)
    first[:, rng.random(m.n_rows) < 0.4] = 0
    second = np.stack([rng.permutation(sino) for _ in range(B)]).astype(np.int32)
    second[:, rng.random(m.n_rows) < 0.3] = 0
    second[0, ::7] = 0  # and some rows empty in one frame only
    tuning = dict(bk_mode=api.BK_CSC, group=group, frame_tile=tile, blocks_per_sm=4,
                  visit=api.VISIT_SORTED)

    def run(ctx, s):
        ctx.set_sinograms(s)
        ctx.init_images()
        ctx.iterate(5)
        return ctx.get_images()

    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(first)
        ctx._refresh()
        before = ctx.info.device_bytes
        ctx.set_tuning(**tuning)
        ctx._refresh()
        # the CSC in visiting order and its cut copy (entries, lengths, flags)
        Z, R, C = m.nnz, m.n_rows, m.n_cols
        assert ctx.info.device_bytes - before == 2 * (Z + 2) * 8 + 4 * R + 4 * C + \
            4 * ((R + 31) // 32 + 1)
        run(ctx, first)
        again = run(ctx, second)
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(second)
        ctx.set_tuning(**tuning)
        fresh = run(ctx, second)
    assert again.tobytes() == fresh.tobytes()
    for b in range(B):
        want, _ = ob.mlem(m, second[b], 5)
        assert ob.rel_l2(fresh[b], want) <= TOL_MLEM, b


@pytest.mark.parametrize("group,tile", [(32, 1), (16, 4), (8, 16), (32, 2)])
def test_csc_in_visiting_order_with_frames(golden, group, tile):
    m, sino, iters, gold, _ = golden.case("tiny_it10")
    rng = np.random.default_rng(7 * tile)
    B = 16
    sinos = np.stack([rng.permutation(sino) if b else sino for b in range(B)]).astype(np.int32)
    sinos[3, ::3] = 0  # rows without counts in some frames
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sinos)
        ctx.set_tuning(bk_mode=api.BK_CSC, group=group, frame_tile=tile, blocks_per_sm=8,
                       visit=api.VISIT_SORTED)
        ctx.init_images()
        ctx.iterate(iters)
        imgs = ctx.get_images()
        # the device-pointer and host-buffer projections stay in row order
        x = np.full(m.n_cols, 1.25, np.float32)
        assert ob.rel_l2(ctx.fwproj(x), ob.fwproj(m, x)) <= TOL_PROJ
        c = ob.correl(ob.fwproj(m, x), sino)
        assert ob.rel_l2(ctx.bkproj(c), ob.bkproj(m, c)) <= TOL_PROJ
    for b in range(B):
        want, _ = ob.mlem(m, sinos[b], iters)
        assert ob.rel_l2(imgs[b], want) <= TOL_MLEM, b


@pytest.mark.parametrize("group,tile", [(8, 1), (16, 4), (32, 8), (32, 16), (16, 16), (4, 16)])
@pytest.mark.parametrize("mode", MODES)
def test_batched_frames_match_separate_runs(golden, group, tile, mode):
    m, sino, iters, gold, _ = golden.case("tiny_it10")
    rng = np.random.default_rng(group * 100 + tile)
    B = 16
    sinos = np.stack([rng.permutation(sino) if b else sino for b in range(B)]).astype(np.int32)
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sinos)
        ctx.set_tuning(bk_mode=mode, group=group, frame_tile=tile, blocks_per_sm=8)
        ctx.init_images()
        ctx.iterate(iters)
        imgs = ctx.get_images()
    for b in range(B):
        want, _ = ob.mlem(m, sinos[b], iters)
        assert ob.rel_l2(imgs[b], want) <= TOL_MLEM, b


@pytest.mark.parametrize("B", [3, 5, 12])
def test_odd_frame_counts(golden, B):
    m, sino, iters, gold, _ = golden.case("edge_it7")
    sinos = np.stack([np.roll(sino, b) for b in range(B)]).astype(np.int32)
    with api.Context.from_matrix(m) as ctx:
        imgs, sums = api.mlem(ctx, sinos, nIterations=iters)
        assert sums.shape == (iters, B)
    for b in range(B):
        want, _ = ob.mlem(m, sinos[b], iters)
        assert ob.rel_l2(imgs[b], want) <= TOL_MLEM


def test_step_host_matches_iterate(ctxs):
    ctx, m, sino, iters, gold = ctxs["tiny_it10"]
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8)
    init = ctx.init_images()
    x = np.full((1, m.n_cols), init[0], np.float32)
    for _ in range(iters):
        ctx.step_host(sino, x)
    ctx.init_images()
    ctx.iterate(iters)
    assert x.tobytes() == ctx.get_images().tobytes()


@pytest.mark.parametrize("visit", [api.VISIT_FILE, api.VISIT_SORTED])
def test_stream_host_matches_step_host(ctxs, visit):
    """mlem_stream_host with one sinogram per iteration equals the same
    iterations through mlem_step_host, bit for bit with the deterministic CSC
    method (the image stays on the device between the streamed iterations).
    With the sorted visit both walk the whole CSC in visiting order: its copy
    cut to the rays with counts is made by mlem_set_sinograms only."""
    ctx, m, sino, iters, gold = ctxs["tiny_it10"]
    rng = np.random.default_rng(31)
    sinos = [rng.permutation(sino).astype(np.int32) for _ in range(6)]
    for s in sinos[::2]:
        s[rng.random(m.n_rows) < 0.3] = 0
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8, visit=visit)
    init = ctx.init_images()
    x = np.full((1, m.n_cols), init[0], np.float32)
    want = []
    for s in sinos:
        ctx.step_host(s, x)
        want.append(x.copy())
    ctx.set_sinograms(sino)
    ctx.init_images()
    got = [np.zeros((1, m.n_cols), np.float32) for _ in sinos]
    got[2] = None  # no download for iteration 2
    ctx.stream_host(sinos, got)
    for k, g in enumerate(got):
        if g is not None:
            assert g.tobytes() == want[k].tobytes(), k
    assert ctx.get_images().tobytes() == want[-1].tobytes()
    ctx._refresh()
    assert ctx.info.rows_with_counts == int((sinos[-1] != 0).sum())
    if visit == api.VISIT_SORTED:
        # the same iterations after mlem_set_sinograms (the cut copy): other
        # rounding, the same images within the tolerance
        x = want[0]
        for k, s in enumerate(sinos[1:], 1):
            ctx.set_sinograms(s)
            ctx.set_images(x)
            ctx.iterate(1)
            x = ctx.get_images()
            assert ob.rel_l2(x[0], want[k][0]) <= TOL_PROJ, k


@pytest.mark.parametrize("n", [3, 4])
@pytest.mark.parametrize("mode,visit", [(api.BK_CSC, api.VISIT_SORTED),
                                        (api.BK_FUSED, api.VISIT_SORTED_CHUNKED)])
def test_stream_host_leaves_the_last_sinograms(ctxs, n, mode, visit):
    """mlem_stream_host uploads each step's sinograms and rebuilds their list
    of rows with counts into one of two buffer sets while the step before
    iterates; afterwards the context iterates on the last step's sinograms,
    whichever set holds them (odd and even step counts)."""
    ctx, m, sino, iters, gold = ctxs["tiny_it10"]
    rng = np.random.default_rng(17 + n)
    sinos = [rng.permutation(sino).astype(np.int32) for _ in range(n)]
    for s in sinos:
        s[rng.random(m.n_rows) < 0.3] = 0
    ctx.set_sinograms(sino)
    ctx.set_tuning(bk_mode=mode, group=32, frame_tile=1, blocks_per_sm=4, visit=visit)
    init = ctx.init_images()
    ctx.stream_host(sinos)
    ctx.iterate(2)
    got = ctx.get_images()
    ctx._refresh()
    assert ctx.info.rows_with_counts == int((sinos[-1] != 0).sum())
    x = np.full((1, m.n_cols), init[0], np.float32)
    for s in sinos + [sinos[-1]] * 2:
        ctx.step_host(s, x)
    if mode == api.BK_CSC:  # deterministic: the same sums in the same order
        assert got.tobytes() == x.tobytes()
    else:
        assert ob.rel_l2(got[0], x[0]) <= TOL_PROJ


@pytest.mark.parametrize("flags", [0, api.FLAG_NATURAL_LAYOUT])
@pytest.mark.parametrize("frames", [1, 3])
def test_stream_host_against_oracle(golden, flags, frames):
    """Streamed iterations on the one-pass method, each with other sinograms,
    against the oracle's MLEM step by step, in both voxel layouts and with one
    and three frames (padded to four); images=None downloads nothing."""
    m, sino, _, _, _ = golden.case("plain_small_it10")
    rng = np.random.default_rng(32 + frames)
    n = 5
    sinos = [np.stack([rng.permutation(sino) for _ in range(frames)]).astype(np.int32)
             for _ in range(n)]
    with api.Context.from_matrix(m, flags=flags) as ctx:
        ctx.set_sinograms(sinos[0])
        ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                       visit=api.VISIT_SORTED_CHUNKED)
        x = ctx.init_images()
        cur = np.repeat(np.asarray(x, np.float32)[:, None], m.n_cols, axis=1)
        got = [np.zeros((frames, m.n_cols), np.float32) for _ in range(n)]
        ctx.stream_host(sinos, got)
        for k in range(n):
            for b in range(frames):
                want, _ = ob.mlem(m, sinos[k][b], 1, start_image=cur[b])
                assert ob.rel_l2(got[k][b], want) <= TOL_MLEM, (k, b)
            cur = got[k]
        ctx.stream_host(sinos[:2])  # no images: the context's own advance
        assert ctx.get_images().shape == (frames, m.n_cols)
        with pytest.raises(api.MlemError):
            ctx.stream_host([sinos[0][:, :-1]])  # wrong size
        with pytest.raises(api.MlemError):
            ctx.stream_host(sinos[:2], [got[0]])  # one buffer per iteration


@pytest.mark.parametrize("via_file", [False, True])
def test_large_element_upload_round_trip(tmp_path, via_file):
    """Element arrays of 128 MiB and more go up through host threads and a
    ring of page-locked buffers, 16 MiB per copy: the device matrix equals the
    host arrays byte for byte (a size that is not a whole number of chunks),
    from host arrays and from a mapped CSR4 file."""
    rng = np.random.default_rng(3)
    R, C = 200_003, 4096
    row_end = np.cumsum(rng.integers(80, 120, R)).astype(np.uint64)
    nnz = int(row_end[-1])
    el = np.zeros(nnz, formats.ELEM_DTYPE)
    el["index"] = rng.integers(0, C, nnz, dtype=np.uint32)
    el["value"] = rng.random(nnz, dtype=np.float32) + 0.25
    assert nnz * 8 > 128 << 20 and (nnz * 8) % (16 << 20)
    if via_file:
        path = tmp_path / "large.csr4"
        formats.write_csr4(str(path), R, C, row_end, el)
        ctx = api.Context.from_file(str(path), flags=api.FLAG_NO_CSC)
    else:
        ctx = api.Context.from_matrix(formats.Csr4(R, C, row_end, el), flags=api.FLAG_NO_CSC)
    with ctx:
        got_end, got_el = ctx.csr()
        assert np.array_equal(got_end, row_end)
        assert got_el.tobytes() == el.tobytes()


def test_device_generator_matches_host_generator():
    g = synth.Geometry(32, 32, 16, 20000, 20, 80, seed=9)
    hm = synth.host_matrix(g)
    with api.Context.siddon(g) as ctx:
        row_end, el = ctx.csr()
        assert np.array_equal(row_end, hm.row_end)
        assert el.tobytes() == hm.elems.tobytes()
        x = synth.phantom(32, 32, 16, 4, 2)
        assert np.array_equal(ctx.project_f64(x), synth.project_f64(hm, x))


def test_skewed_matrix_long_rows_and_columns(golden):
    """A 12k-element row and columns longer than the shared-memory sort."""
    rng = np.random.default_rng(7)
    R, C = 3000, 512
    rows = [rng.integers(0, C, size=int(rng.integers(0, 30))) for _ in range(R)]
    rows[5] = rng.integers(0, C, size=12000)
    rows[6] = np.full(5000, 3)            # one column of > 4096 entries, duplicates in one row
    rows[2000] = np.full(9000, 100)
    counts = np.array([len(r) for r in rows], np.uint64)
    row_end = np.cumsum(counts, dtype=np.uint64)
    el = np.zeros(int(row_end[-1]), api.ELEM_DTYPE)
    el["index"] = np.concatenate(rows).astype(np.uint32)
    el["value"] = rng.uniform(0.1, 1.7, el.size).astype(np.float32)
    m = formats.Csr4(R, C, row_end, el)
    sino = rng.poisson(50, R).astype(np.int32)
    with api.Context.from_matrix(m) as ctx:
        cp, ce = ctx.csc()
        cp_o, ce_o = ob.transpose(m)
        assert np.array_equal(cp, cp_o) and ce.tobytes() == ce_o.tobytes()
        assert ctx.column_sums().tobytes() == ob.column_sums(m).tobytes()
        want, _ = ob.mlem(m, sino, 5)
        for mode in MODES:
            ctx.set_sinograms(sino)
            ctx.set_tuning(bk_mode=mode, group=32, frame_tile=1, blocks_per_sm=8)
            ctx.init_images()
            ctx.iterate(5)
            assert ob.rel_l2(ctx.get_images()[0], want) <= TOL_MLEM
        # sorted visits: the long rows exceed the 64 KiB next-row prefetch, a chunk and a
        # shared-memory stage
        for visit, bps in ((api.VISIT_SORTED, 8), (api.VISIT_SORTED_CHUNKED, 4),
                           (api.VISIT_SORTED_CHUNKED, 1), (api.VISIT_SORTED_STAGED, 4),
                           (api.VISIT_SORTED_STAGED, 1)):
            ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=bps,
                           visit=visit)
            ctx.init_images()
            ctx.iterate(5)
            assert ob.rel_l2(ctx.get_images()[0], want) <= TOL_MLEM
        # a batch with a regular matrix: the long rows run as segments after the batch kernel
        small_m, small_sino, _, _, _ = golden.case("tiny_it10")
        with api.Context.from_matrix(small_m) as other:
            other.set_sinograms(small_sino)
            other.init_images()
            ctx.init_images()
            for policy, visit in ((api.BATCH_ITEMS, api.VISIT_SORTED),
                                  (api.BATCH_ITEMS, api.VISIT_SORTED_STAGED),
                                  (api.BATCH_INTERLEAVED, api.VISIT_FILE)):
                with api.Batch([ctx, other]) as b:
                    b.set_schedule(policy, 64, 4, 1, visit)
                    _, _, launches = b.profile(1)
                    assert launches[0] == 1 + 2  # one group, then the long rows' two kernels
                    ctx.init_images()
                    other.init_images()
                    b.iterate(5)
                assert ob.rel_l2(ctx.get_images()[0], want) <= TOL_MLEM
                want_o, _ = ob.mlem(small_m, small_sino, 5)
                assert ob.rel_l2(other.get_images()[0], want_o) <= TOL_MLEM


@pytest.mark.parametrize("visit", [api.VISIT_FILE, api.VISIT_SORTED, api.VISIT_SORTED_CHUNKED,
                                   api.VISIT_SORTED_STAGED])
def test_long_rows_split_into_segments(visit):
    """Rows longer than 4096 elements run as segments (k_long.cu) in the
    one-pass method: rows at, just above and far above the limit, several
    frames and frame tiles, against the oracle."""
    rng = np.random.default_rng(11)
    R, C = 2000, 4096
    lens = rng.integers(0, 60, size=R)
    lens[[3, 500, 501, 1999]] = [70000, 4096, 4097, 8193]
    rows = [rng.integers(0, C, size=int(n)) for n in lens]
    row_end = np.cumsum(lens).astype(np.uint64)
    el = np.zeros(int(row_end[-1]), api.ELEM_DTYPE)
    el["index"] = np.concatenate(rows).astype(np.uint32)
    el["value"] = rng.uniform(0.1, 1.7, el.size).astype(np.float32)
    m = formats.Csr4(R, C, row_end, el)
    sinos = rng.poisson(40, (3, R)).astype(np.int32)
    want = [ob.mlem(m, sinos[b], 6)[0] for b in range(3)]
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sinos)
        for tile in (1, 2, 4):
            ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=tile, blocks_per_sm=4,
                           visit=visit)
            assert ctx.kernels_per_iteration() >= 6  # one-pass, two long-row kernels, update, stats
            ctx.init_images()
            ctx.iterate(6)
            got = ctx.get_images()
            for b in range(3):
                assert ob.rel_l2(got[b], want[b]) <= TOL_MLEM, (tile, b)


def test_invalid_inputs_raise():
    re_ = np.array([2, 3], np.uint64)
    el = np.zeros(3, api.ELEM_DTYPE)
    el["index"] = [0, 5, 1]  # column 5 >= C = 2
    with pytest.raises(api.MlemError) as e:
        api.Context(re_, el, 2, 2)
    assert e.value.status == api.MLEM_ERR_MATRIX
    el["index"] = [0, 1, 1]
    with api.Context(re_, el, 2, 2) as ctx:
        with pytest.raises(api.MlemError):
            ctx.set_sinograms(np.ones(3, np.int32))  # wrong length
        with pytest.raises(api.MlemError) as e:
            ctx.iterate(1)
        assert e.value.status == api.MLEM_ERR_STATE
        with pytest.raises(api.MlemError):
            ctx.set_tuning(bk_mode=api.BK_CSC, group=6, frame_tile=1)
        with pytest.raises(api.MlemError):
            ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=3)
        with pytest.raises(api.MlemError):
            ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, visit=4)
    with api.Context(re_, el, 2, 2, flags=api.FLAG_NO_ROW_ORDER) as ctx:
        with pytest.raises(api.MlemError):  # no row order to visit in
            ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, visit=api.VISIT_SORTED)


def test_autotune_restores_images(ctxs):
    ctx, m, sino, iters, gold = ctxs["plain_small_it10"]
    ctx.set_sinograms(np.stack([sino, sino]))
    ctx.init_images()
    before = ctx.get_images()
    best = ctx.autotune()
    assert best["ms_per_iter"] > 0
    assert ctx.get_images().tobytes() == before.tobytes()
    ctx.iterate(iters)
    assert ob.rel_l2(ctx.get_images()[0], gold) <= TOL_MLEM


@pytest.mark.parametrize("name", CASES)
def test_brick_layout_changes_no_result(golden, name):
    """The device voxel layout only relabels voxels and the row order only
    changes the order rows are visited in: CSC-mode images (per-row and
    per-column sums in a fixed order), the CSR/CSC copies and the column sums
    are bit-identical to natural voxel order and file row order."""
    m, sino, iters, gold, _ = golden.case(name)
    out = []
    for flags in (0, api.FLAG_NATURAL_LAYOUT, api.FLAG_NO_ROW_ORDER,
                  api.FLAG_NATURAL_LAYOUT | api.FLAG_NO_ROW_ORDER):
        with api.Context.from_matrix(m, flags=flags) as ctx:
            ctx.set_sinograms(sino)
            ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8)
            ctx.init_images()
            ctx.iterate(iters)
            out.append((ctx.get_images().tobytes(), ctx.column_sums().tobytes(),
                        ctx.csc()[1].tobytes(), ctx.csr()[1].tobytes()))
    assert all(o == out[0] for o in out)


@pytest.mark.parametrize("frames", [1, 16])
def test_row_order_changes_only_rounding(golden, frames):
    """The sorted row visits move only the order of the scatter atomics: the
    images agree with file order within float rounding, and with the oracle
    within the MLEM tolerance."""
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    sinos = np.stack([np.roll(sino, 7 * b) for b in range(frames)]).astype(np.int32)
    want = [ob.mlem(m, sinos[b], iters)[0] for b in range(frames)]
    tile = min(frames, 8)
    runs = [(api.BK_ATOMIC, api.VISIT_FILE, tile), (api.BK_ATOMIC, api.VISIT_SORTED, tile),
            (api.BK_FUSED, api.VISIT_FILE, tile), (api.BK_FUSED, api.VISIT_SORTED, tile),
            (api.BK_FUSED, api.VISIT_SORTED_CHUNKED, tile),
            (api.BK_FUSED, api.VISIT_SORTED_STAGED, tile),
            (api.BK_FUSED, api.VISIT_SORTED_STAGED, frames)]
    imgs = []
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sinos)
        for mode, visit, ft in runs:
            ctx.set_tuning(bk_mode=mode, group=32, frame_tile=ft, blocks_per_sm=8,
                           visit=visit)
            ctx.init_images()
            ctx.iterate(iters)
            imgs.append(ctx.get_images())
    for img in imgs:
        for b in range(frames):
            assert ob.rel_l2(img[b], imgs[0][b]) <= 1e-5
            assert ob.rel_l2(img[b], want[b]) <= TOL_MLEM


def test_device_pointer_api_in_natural_order(small_ctx=None):
    torch = pytest.importorskip("torch")
    g = synth.Geometry(16, 16, 8, 3000, 5, 40, seed=3)
    hm = synth.host_matrix(g)
    x = torch.rand(hm.n_cols, device="cuda")
    res = []
    for flags in (0, api.FLAG_NATURAL_LAYOUT):
        with api.Context.from_matrix(hm, flags=flags) as ctx:
            y = torch.empty(hm.n_rows, device="cuda")
            ctx.fwproj_d(x.data_ptr(), y.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
            xb = torch.empty(hm.n_cols, device="cuda")
            ctx.bkproj_d(y.data_ptr(), xb.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            res.append((y.cpu().numpy().tobytes(), xb.cpu().numpy().tobytes()))
    assert res[0] == res[1]
    want = ob.fwproj(hm, x.cpu().numpy())
    assert ob.rel_l2(np.frombuffer(res[0][0], np.float32), want) < TOL_PROJ


@pytest.mark.parametrize("flags", [0, api.FLAG_NATURAL_LAYOUT])
@pytest.mark.parametrize("frames", [1, 3])
@pytest.mark.parametrize("long_row", [False, True])
def test_fused_update_d_matches_two_step(golden, flags, frames, long_row):
    """mlem_fused_update_d (one pass) equals mlem_fwproj_correl_d followed by
    mlem_bkproj_d (two passes) within float rounding, in both voxel layouts,
    with several frames and with a row above the long-row limit."""
    torch = pytest.importorskip("torch")
    g = synth.Geometry(16, 16, 8, 3000, 5, 40, seed=7)
    hm = synth.host_matrix(g)
    if long_row:  # append one row of 6000 elements
        rng = np.random.default_rng(2)
        extra = np.zeros(6000, api.ELEM_DTYPE)
        extra["index"] = rng.integers(0, hm.n_cols, 6000)
        extra["value"] = rng.uniform(0.1, 1.5, 6000).astype(np.float32)
        row_end = np.concatenate([hm.row_end, [hm.row_end[-1] + 6000]]).astype(np.uint64)
        hm = formats.Csr4(hm.n_rows + 1, hm.n_cols, row_end, np.concatenate([hm.elems, extra]),
                          0, hm.grid)
    rng = np.random.default_rng(3)
    x = torch.rand(hm.n_cols * frames, device="cuda") + 0.1
    s = torch.tensor(rng.poisson(5, hm.n_rows * frames).astype(np.int32), device="cuda")
    with api.Context.from_matrix(hm, flags=flags) as ctx:
        st = torch.cuda.current_stream().cuda_stream
        c = torch.empty(hm.n_rows * frames, device="cuda")
        u2 = torch.empty_like(x)
        ctx.fwproj_correl_d(x.data_ptr(), s.data_ptr(), c.data_ptr(), frames, st)
        ctx.bkproj_d(c.data_ptr(), u2.data_ptr(), frames, st)
        u1 = torch.full_like(x, 7.0)  # overwritten, not accumulated into
        ctx.fused_update_d(x.data_ptr(), s.data_ptr(), u1.data_ptr(), frames, st)
        torch.cuda.synchronize()
        assert ob.rel_l2(u1.cpu().numpy(), u2.cpu().numpy()) <= 1e-5


@pytest.mark.parametrize("visit,bps", [(api.VISIT_SORTED, 8), (api.VISIT_SORTED_CHUNKED, 4),
                                       (api.VISIT_SORTED_STAGED, 4)])
def test_rows_without_counts_are_skipped(golden, visit, bps):
    """Rows whose counts are zero in every frame add nothing to the update: the
    sorted one-pass walks leave them out, and the list follows new sinograms,
    through the captured graph and through mlem_step_host."""
    m, sino, _, _, _ = golden.case("plain_small_it10")
    rng = np.random.default_rng(5)
    B = 3
    lens = np.diff(np.concatenate([[0], np.asarray(m.row_end, np.int64)]))
    sinos = np.stack([rng.permutation(sino) for _ in range(B)]).astype(np.int32)
    dead = rng.random(m.n_rows) < 0.5
    sinos[:, dead] = 0
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sinos)
        ctx._refresh()
        live = (sinos != 0).any(axis=0)
        assert ctx.info.rows_with_counts == int(live.sum())
        assert ctx.info.nnz_with_counts == int(lens[live].sum())
        ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=4, blocks_per_sm=bps, visit=visit)
        for it in range(2):
            ctx.init_images()
            ctx.iterate(6)
            got = ctx.get_images()
            for b in range(B):
                want, _ = ob.mlem(m, sinos[b], 6)
                assert ob.rel_l2(got[b], want) <= TOL_MLEM, (it, b)
            # other rows with counts, same frame count: the list is rebuilt in place
            sinos = sinos.copy()
            sinos[:, ~dead] = 0
            sinos[:, dead] = rng.poisson(30, (B, int(dead.sum())))
            ctx.set_sinograms(sinos)
        x0 = np.full((B, m.n_cols), 0.5, np.float32)
        x = x0.copy()
        ctx.step_host(sinos, x)
        for b in range(B):
            want, _ = ob.mlem(m, sinos[b], 1, start_image=x0[b])
            assert ob.rel_l2(x[b], want) <= TOL_MLEM, b
        # a step with another sinogram reports that sinogram's rows with counts
        half = sinos.copy()
        half[:, ::2] = 0
        x = x0.copy()
        ctx.step_host(half, x)
        ctx._refresh()
        live = (half != 0).any(axis=0)
        assert ctx.info.rows_with_counts == int(live.sum())
        assert ctx.info.nnz_with_counts == int(lens[live].sum())
        zero = np.zeros_like(sinos)  # no row left: the walk visits nothing
        ctx.set_sinograms(zero)
        ctx._refresh()
        assert ctx.info.rows_with_counts == 0
        x = x0.copy()
        ctx.step_host(zero, x)
        for b in range(B):
            want, _ = ob.mlem(m, zero[b], 1, start_image=x0[b])
            assert x[b].tobytes() == want.tobytes()


def test_measure_l2_rates():
    """mlem_measure_l2_rates: four positive rates; float reductions to random
    addresses run slower than gathers of the same width (the bound of the
    one-pass walk)."""
    r = api.measure_l2_rates(0)
    assert all(v > 0 for v in r.values())
    assert r["red_4B_per_s"] < r["gather_4B_per_s"]
    assert r["red_64B_rows_per_s"] < r["gather_64B_rows_per_s"]
