"""The allocation-free entry point (mlem_iterate_noalloc_d).

Callers that cannot let a library allocate device memory (a fixed device
memory budget, or allocations kept out of a critical section) run one MLEM
iteration on their own device buffers; the update vector lives in the
library's fixed static device array.  Its results must match the existing
entry point (a context's mlem_iterate) after each of two calls in a row,
within the 1e-5 relative L2 the single-step parity tests use.  This file
sorts last so that a run stopping at the first failure has run the rest.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mlem_b200 import api  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_existing_entry_point_on_two_calls(golden):
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    dev = torch.device("cuda", 0)
    with api.Context.from_matrix(m) as ctx:
        ctx.set_sinograms(sino)
        ctx.set_tuning(bk_mode=api.BK_CSC, group=32, frame_tile=1, blocks_per_sm=8)
        init = ctx.init_images()
        norm = ctx.column_sums()
        row_ptr = torch.from_numpy(m.row_ptr().view(np.int64)).to(dev)
        elems = torch.from_numpy(np.ascontiguousarray(m.elems).view(np.int32)).to(dev)
        sino_d = torch.from_numpy(np.ascontiguousarray(sino, np.int32)).to(dev)
        norm_d = torch.from_numpy(norm).to(dev)
        x = torch.full((m.n_cols,), float(init[0]), dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream().cuda_stream
        for call in range(2):
            api.iterate_noalloc_d(row_ptr.data_ptr(), elems.data_ptr(), m.n_rows, m.n_cols,
                                  sino_d.data_ptr(), norm_d.data_ptr(), x.data_ptr(), stream)
            ctx.iterate(1)
            want = ctx.get_images()[0]
            got = x.cpu().numpy()
            assert _rel_l2(got, want) <= TOL, (call, _rel_l2(got, want))


def test_noalloc_rejects_images_beyond_the_fixed_scratch():
    with pytest.raises(api.MlemError) as e:
        api.iterate_noalloc_d(0, 0, 1, api.NOALLOC_MAX_VOXELS + 1, 0, 0, 0, 0)
    assert e.value.status == api.MLEM_ERR_INVALID
    assert "exceed" in e.value.message
