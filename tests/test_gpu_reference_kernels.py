"""The reference's own CUDA kernels, run as the comparison baseline on the
same GPU (oracle/_ref/libref_cuda.so: mlem_cuda/helper_files/cudaKernels.cu
compiled unmodified, driven by oracle/ref_cuda/harness.cu in the iteration
order of the reference's version_4 and version_6 drivers).  The harness's
images must match the oracle within 1e-4, which pins it as a fair baseline."""
import os

import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(ob.REF_CUDA_SO), reason="reference CUDA kernels not built")
@pytest.mark.parametrize("name", ["plain_small_it10", "edge_it7", "tiny_it10"])
@pytest.mark.parametrize("variant", [4, 6])
def test_reference_kernels_match_oracle(golden, name, variant):
    m, sino, iters, gold, _ = golden.case(name)
    img, ms = ob.ref_cuda_mlem(m, sino, iters, variant)
    assert ob.rel_l2(img, gold) <= 1e-4
    assert ms[5] > 0
