"""Seeded random matrices of odd shapes against the oracle on the GPU: a
single row or voxel, empty rows, zero values, zero counts, duplicate columns
and a row above the long-row limit, through every method, row visit, frame
count and ordered-subset setting.  Every image must match the oracle's run
within relative L2 1e-4."""
import numpy as np
import pytest

from mlem_b200 import api, formats

import oracle_bind as ob

pytestmark = pytest.mark.gpu

TOL = 1e-4
SHAPES = [  # rows, columns, max row length, long row
    (1, 1, 3, False), (1, 50, 40, False), (7, 5, 6, False), (300, 64, 30, False),
    (5000, 4096, 60, False), (2000, 512, 20, True),
]


def random_case(R, C, maxlen, long_row, seed):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, maxlen + 1, R)
    lens[rng.random(R) < 0.1] = 0  # empty rows
    if long_row:
        lens[R // 2] = 9000
    row_end = np.cumsum(lens).astype(np.uint64)
    Z = int(row_end[-1])
    el = np.zeros(Z, formats.ELEM_DTYPE)
    el["index"] = rng.integers(0, C, Z)  # duplicates within a row are possible
    v = rng.uniform(0.05, 1.7, Z).astype(np.float32)
    v[rng.random(Z) < 0.02] = 0.0
    el["value"] = v
    sino = rng.poisson(20, (3, R)).astype(np.int32)
    sino[:, rng.random(R) < 0.2] = 0
    return formats.Csr4(R, C, row_end, el), sino


RUNS = [(api.BK_CSC, api.VISIT_FILE, 32), (api.BK_ATOMIC, api.VISIT_SORTED, 16),
        (api.BK_FUSED, api.VISIT_FILE, 8), (api.BK_FUSED, api.VISIT_SORTED, 32),
        (api.BK_FUSED, api.VISIT_SORTED_CHUNKED, 32), (api.BK_FUSED, api.VISIT_SORTED_STAGED, 32),
        (api.BK_REGION, api.VISIT_FILE, 32)]


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{s[0]}x{s[1]}" + ("-long" if s[3] else "")
                                                for s in SHAPES])
def test_random_matrix_every_method(shape):
    R, C, maxlen, long_row = shape
    m, sino = random_case(R, C, maxlen, long_row, seed=R * 31 + C)
    if m.nnz == 0:
        pytest.skip("empty draw")
    want1 = ob.mlem(m, sino[0], 5)[0]
    want3 = [ob.mlem(m, sino[b], 5)[0] for b in range(3)]
    with api.Context.from_matrix(m) as ctx:
        for mode, visit, group in RUNS:
            if visit != api.VISIT_FILE and R < 2:
                continue  # no row order for a single row
            for frames, want in ((1, [want1]), (3, want3)):
                ctx.set_sinograms(sino[:frames])
                ctx.set_tuning(bk_mode=mode, group=group, frame_tile=1 if frames == 1 else 2,
                               blocks_per_sm=4, visit=visit)
                ctx.init_images()
                ctx.iterate(5)
                got = ctx.get_images()
                for b in range(frames):
                    assert ob.rel_l2(got[b], want[b]) <= TOL, (mode, visit, frames, b)
        if R >= 3:  # ordered subsets on the one-pass method
            ctx.set_sinograms(sino[:1])
            ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                           visit=api.VISIT_SORTED_CHUNKED)
            ctx.set_subsets(3)
            ctx.init_images()
            ctx.iterate(4)
            assert ob.rel_l2(ctx.get_images()[0], ob.osem(m, sino[0], 4, 3)[0]) <= TOL
            ctx.set_subsets(1)
