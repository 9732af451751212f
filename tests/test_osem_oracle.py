"""The oracle's ordered subsets (OSEM), which the reference does not have.

OSEM is restated in oracle/mlem_oracle.c from the reference's own pieces
(calcFwProj, calcCorrel, calcBkProj and calcColumnSums of
mlem_seq/seqcsr4mlem.cpp restricted to a subset's rows) with an update that
keeps the voxels a subset does not see.  With one subset it must be the
reference iteration itself: bit for bit the golden images of the reference
binary.  That is the pin; more subsets have no reference output to match.
"""
import numpy as np
import pytest

import oracle_bind as ob
from golden_cases import CASES


@pytest.mark.parametrize("name", CASES)
def test_one_subset_is_the_reference_iteration(golden, name):
    m, sino, iters, gold, _ = golden.case(name)
    img, sums = ob.osem(m, sino, iters, 1)
    assert img.tobytes() == gold.tobytes()
    _, want_sums = ob.mlem(m, sino, iters)
    assert sums.tobytes() == want_sums.tobytes()


@pytest.mark.parametrize("name", CASES)
def test_subset_column_sums_partition_the_column_sums(golden, name):
    m = golden.case(name)[0]
    full = ob.column_sums(m)
    assert ob.subset_column_sums(m, 1, 0).tobytes() == full.tobytes()
    for S in (2, 3, 8):
        parts = np.stack([ob.subset_column_sums(m, S, s) for s in range(S)])
        np.testing.assert_allclose(parts.astype(np.float64).sum(0), full, rtol=2e-6, atol=1e-30)
        # a voxel is seen by a subset exactly when that subset has a row through it
        rows = np.repeat(np.arange(m.n_rows), np.diff(np.concatenate([[0], m.row_end.astype(np.int64)])))
        for s in range(S):
            seen = np.zeros(m.n_cols, bool)
            sel = (rows % S) == s
            seen[m.elems["index"][sel]] = True
            assert not np.any(parts[s][~seen])


def test_subsets_keep_unseen_voxels():
    """A voxel that only subset 1 sees keeps its value through subset 0."""
    from mlem_b200 import formats
    row_end = np.array([2, 4], np.uint64)
    el = np.zeros(4, formats.ELEM_DTYPE)
    el["index"] = [0, 1, 1, 2]
    el["value"] = [1.0, 1.0, 1.0, 1.0]
    m = formats.Csr4(2, 3, row_end, el)
    sino = np.array([4, 10], np.int32)
    x0 = np.array([1.0, 1.0, 1.0], np.float32)
    # after one iteration with 2 subsets: subset 0 (row 0) updates voxels 0, 1
    # and leaves voxel 2; subset 1 (row 1) updates voxels 1, 2 and leaves voxel 0
    img, _ = ob.osem(m, sino, 1, 2, start_image=x0)
    x = x0.astype(np.float64)
    c0 = 4 / (x[0] + x[1])
    x[0] *= c0 / 1.0
    x[1] *= c0 / 1.0
    c1 = 10 / (x[1] + x[2])
    x[1] *= c1 / 1.0
    x[2] *= c1 / 1.0
    np.testing.assert_allclose(img, x, rtol=1e-6)
