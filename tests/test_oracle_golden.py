"""Pin the oracle (the C restatement of seqcsr4mlem) to the reference binary.

The golden images were produced by the reference's own mlem_seq/seqcsr4mlem
compiled from its sources (tests/golden/make_golden.py); the oracle must
reproduce them bit for bit, including the FTZ mode of seqcsr4mlem.cpp:194.
"""
import numpy as np
import pytest

import oracle_bind as ob
from golden_cases import CASES


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_binary_bit_exact(golden, name):
    m, sino, iters, gold, entry = golden.case(name)
    img, sums = ob.mlem(m, sino, iters, ftz=True)
    assert img.tobytes() == gold.tobytes(), f"max abs diff {np.abs(img - gold).max()}"
    # the per-iteration image sums the reference printed (6 significant digits)
    printed = [float(s) for s in entry["image_sums_printed"]]
    assert len(printed) == iters
    for got, want in zip(sums, printed):
        assert abs(float(got) - want) <= 5e-6 * abs(want) + 1e-30
    zeros = [int((img == 0).sum())]
    assert zeros[-1] == entry["zeros"][-1]


@pytest.mark.parametrize("name", CASES)
def test_fp64_oracle_close_to_reference(golden, name):
    """Both the reference and the FP64 oracle of the same iterations: the
    float reference stays within 1e-4 relative L2 of FP64."""
    m, sino, iters, gold, _ = golden.case(name)
    ref64 = ob.mlem_f64(m, sino, iters)
    assert ob.rel_l2(gold, ref64) < 1e-4


def test_oracle_pieces_compose_to_mlem(golden):
    m, sino, iters, gold, _ = golden.case("edge_it7")
    norm = ob.column_sums(m)
    x = np.full(m.n_cols, ob.init_value(norm, sino), np.float32)
    import ctypes
    old = None
    for _ in range(iters):
        f = ob.fwproj(m, x)
        c = ob.correl(f, sino)
        u = ob.bkproj(m, c)
        x = ob.update(u, norm, x)
    # without FTZ the composition may differ only by subnormal flushing
    assert ob.rel_l2(x, gold) < 1e-6


def test_transpose_is_stable_and_complete(golden):
    m, *_ = golden.case("edge_it7")
    col_ptr, ce = ob.transpose(m)
    assert col_ptr[0] == 0 and col_ptr[-1] == m.nnz
    rows = np.repeat(np.arange(m.n_rows, dtype=np.uint32), np.diff(m.row_ptr()).astype(np.int64))
    # expected: stable sort of (column) over row-major order
    order = np.argsort(m.cols, kind="stable")
    assert np.array_equal(ce["index"], rows[order])
    assert np.array_equal(ce["value"].view(np.uint32), m.vals[order].view(np.uint32))


def test_partition_matches_reference_rule(golden):
    m, *_ = golden.case("tiny_it10")
    for n in (1, 2, 3, 8):
        s, e = ob.partition(m, n)
        assert s[0] == 0 and e[-1] == m.n_rows
        assert np.all(s[1:] == e[:-1])
        nnz = [int(m.row_ptr()[b] - m.row_ptr()[a]) for a, b in zip(s, e)]
        assert sum(nnz) == m.nnz


@pytest.mark.parametrize("name", ["plain_small_it10", "edge_it7"])
def test_rows_without_counts_change_nothing(golden, name):
    """The restated reference iteration gives the same image, bit for bit, when
    the rows whose count is zero are emptied: their calcCorrel is 0, so they
    only add +0 to the update (the fact the GPU walks rely on to leave them out)."""
    from mlem_b200 import formats

    m, sino, _, _, _ = golden.case(name)
    rng = np.random.default_rng(3)
    sino = sino.copy()
    sino[rng.random(m.n_rows) < 0.4] = 0
    keep = sino != 0
    lens = np.diff(np.concatenate([[0], np.asarray(m.row_end, np.int64)]))
    starts = np.concatenate([[0], np.asarray(m.row_end, np.int64)[:-1]])
    idx = np.concatenate([np.arange(s, s + n) for s, n in zip(starts[keep], lens[keep])]) \
        if keep.any() else np.zeros(0, np.int64)
    kept_lens = np.where(keep, lens, 0)
    m2 = formats.Csr4(m.n_rows, m.n_cols, np.cumsum(kept_lens).astype(np.uint64),
                      np.ascontiguousarray(np.asarray(m.elems)[idx]))
    # calcColumnSums stays the full matrix's (it does not depend on the counts);
    # each iteration's update must match bit for bit
    norm = ob.column_sums(m)
    x = np.full(m.n_cols, ob.init_value(norm, sino), np.float32)
    y = x.copy()
    for _ in range(5):
        ux = ob.bkproj(m, ob.correl(ob.fwproj(m, x), sino))
        uy = ob.bkproj(m2, ob.correl(ob.fwproj(m2, y), sino))
        assert ux.tobytes() == uy.tobytes()
        x = ob.update(ux, norm, x)
        y = ob.update(uy, norm, y)
    assert x.tobytes() == y.tobytes()
