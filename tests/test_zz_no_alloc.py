"""The allocation-free entry point (mlem_iterate_noalloc_d).

Callers that cannot let a library allocate device memory (a fixed device
memory budget handed out by a framework or scheduler, or a device allocator
owned by another component) run one MLEM iteration on their own device
buffers; the update vector lives in the library's fixed static device array.
Its results must match the existing entry point (a context's mlem_iterate)
after each of two calls in a row, within the 1e-5 relative L2 the
single-step parity tests use, and the oracle's iteration.  The matrix checks
it makes as it goes (row offsets against the element count, columns against
the image size) are tested with small host-made inputs whose reads all stay
inside the buffers the test allocates, so no check is needed to keep them in
bounds.  This file sorts last so that a run stopping at the first failure has
run the rest.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle_bind as ob  # noqa: E402
from mlem_b200 import api, formats  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(torch.device("cuda", 0))


class Inputs:
    """Device copies of one matrix, sinogram, column sums and start image."""

    def __init__(self, row_ptr, elems, sino, norm, x0):
        self.row_ptr = _dev(np.asarray(row_ptr, np.uint64).view(np.int64))
        self.n_elems = len(elems)
        self.elems = _dev(np.ascontiguousarray(elems).view(np.int32)) if len(elems) else None
        self.sino = _dev(np.asarray(sino, np.int32))
        self.norm = _dev(np.asarray(norm, np.float32))
        self.x = _dev(np.asarray(x0, np.float32))

    def call(self, n_rows, n_cols, n_elems=None):
        api.iterate_noalloc_d(self.row_ptr.data_ptr(),
                              self.elems.data_ptr() if self.elems is not None else 0,
                              self.n_elems if n_elems is None else n_elems, n_rows, n_cols,
                              self.sino.data_ptr(), self.norm.data_ptr(), self.x.data_ptr(),
                              torch.cuda.current_stream().cuda_stream)

    def image(self):
        torch.cuda.synchronize()
        return self.x.cpu().numpy()


def _start(m, sino):
    norm = ob.column_sums(m)
    return norm, np.full(m.n_cols, ob.init_value(norm, sino), np.float32)


def test_noalloc_matches_existing_entry_point_on_two_calls(golden):
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sino)
        ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8)
        init = ctx.init_images()
        norm = ctx.column_sums()
        d = Inputs(m.row_ptr(), m.elems, sino, norm, np.full(m.n_cols, init[0], np.float32))
        want_oracle, _ = ob.mlem(m, sino, 1)
        for call in range(2):
            d.call(m.n_rows, m.n_cols)
            ctx.iterate(1)
            want = ctx.get_images()[0]
            got = d.image()
            assert _rel_l2(got, want) <= TOL, (call, _rel_l2(got, want))
            if call == 0:
                assert _rel_l2(got, want_oracle) <= TOL


def test_noalloc_rejects_images_beyond_the_fixed_scratch():
    with pytest.raises(api.MlemError) as e:
        api.iterate_noalloc_d(0, 0, 0, 1, api.NOALLOC_MAX_VOXELS + 1, 0, 0, 0, 0)
    assert e.value.status == api.MLEM_ERR_INVALID
    assert "exceed" in e.value.message


def test_noalloc_skips_a_bad_column_and_applies_the_rest(golden):
    m, sino, *_ = golden.case("tiny_it10")
    bad = np.ascontiguousarray(m.elems).copy()
    k = len(bad) // 3
    # the caller's matrix holds one column index past the image; the oracle's
    # matrix has that element's value at 0 instead (it adds nothing anywhere)
    bad["index"][k] = m.n_cols
    fixed = np.ascontiguousarray(m.elems).copy()
    fixed["value"][k] = 0.0
    mf = formats.Csr4(m.n_rows, m.n_cols, m.row_end, fixed)
    norm, x0 = _start(mf, sino)
    d = Inputs(m.row_ptr(), bad, sino, norm, x0)
    with pytest.raises(api.MlemError) as e:
        d.call(m.n_rows, m.n_cols)
    assert e.value.status == api.MLEM_ERR_MATRIX and "column" in e.value.message
    want, _ = ob.mlem(mf, sino, 1, start_image=x0)
    assert _rel_l2(d.image(), want) <= TOL


def test_noalloc_skips_rows_with_bad_offsets(golden):
    m, sino, *_ = golden.case("tiny_it10")
    el = np.ascontiguousarray(m.elems)
    rp = m.row_ptr().copy()
    R = m.n_rows
    assert R >= 8 and int(rp[2]) >= 1 and int(rp[R] - rp[R - 1]) >= 1
    # row 2's end below its start (non-monotone), and an element count that
    # stops one element short of the last row's end.  Every offset still lies
    # inside the element buffer handed over.
    rp[3] = rp[2] - 1
    n_elems = int(rp[R]) - 1
    # the oracle's matrix: row 2 and the last row empty; row 3 starts where
    # row 2 started, as its offsets say (its range is [rp[2]-1, rp[4]))
    rows = []
    for r in range(R):
        b, e = int(rp[r]), int(rp[r + 1])
        if r == 2 or r == R - 1 or b > e:
            rows.append(el[0:0])
        else:
            rows.append(el[b:e])
    ends = np.cumsum([len(x) for x in rows]).astype(np.uint64)
    mo = formats.Csr4(R, m.n_cols, ends, np.concatenate(rows))
    norm, x0 = _start(mo, sino)
    d = Inputs(rp, el, sino, norm, x0)
    with pytest.raises(api.MlemError) as e:
        d.call(R, m.n_cols, n_elems)
    assert e.value.status == api.MLEM_ERR_MATRIX and "offsets" in e.value.message
    want, _ = ob.mlem(mo, sino, 1, start_image=x0)
    assert _rel_l2(d.image(), want) <= TOL


def test_noalloc_without_rows_applies_a_zero_update():
    C = 1000
    rng = np.random.default_rng(5)
    norm = rng.uniform(0.0, 2.0, C).astype(np.float32)
    norm[::7] = 0.0
    x0 = rng.uniform(0.5, 3.0, C).astype(np.float32)
    d = Inputs(np.zeros(1, np.uint64), np.zeros(0, formats.ELEM_DTYPE), np.zeros(1, np.int32), norm,
               x0)
    d.call(0, C)
    want = ob.update(np.zeros(C, np.float32), norm, x0)
    assert d.image().tobytes() == want.tobytes()


def test_noalloc_small_image_after_a_large_one(golden):
    """The shared array keeps the large call's update; the small call must
    clear what it uses and match the context path."""
    rng = np.random.default_rng(11)
    C_big, R_big = api.NOALLOC_MAX_VOXELS, 4096
    lens = rng.integers(50, 100, R_big)
    ends = np.cumsum(lens).astype(np.uint64)
    big_el = np.zeros(int(ends[-1]), formats.ELEM_DTYPE)
    big_el["index"] = rng.integers(0, C_big, len(big_el), dtype=np.uint32)
    big_el["value"] = rng.uniform(0.1, 1.5, len(big_el)).astype(np.float32)
    mb = formats.Csr4(R_big, C_big, ends, big_el)
    sb = rng.poisson(20, R_big).astype(np.int32)
    nb, xb = _start(mb, sb)
    Inputs(mb.row_ptr(), big_el, sb, nb, xb).call(R_big, C_big)

    m, sino, *_ = golden.case("plain_small_it10")
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sino)
        ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8)
        init = ctx.init_images()
        d = Inputs(m.row_ptr(), m.elems, sino, ctx.column_sums(),
                   np.full(m.n_cols, init[0], np.float32))
        d.call(m.n_rows, m.n_cols)
        ctx.iterate(1)
        assert _rel_l2(d.image(), ctx.get_images()[0]) <= TOL
