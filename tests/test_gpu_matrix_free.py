"""Matrix-free MLEM (mlem_mf_*): the synthetic Siddon rays traced again in
every pass instead of a stored matrix.

The traced lengths equal the generator's up to rounding (a voxel cut at a
lane's interval boundary comes as two pieces), so the matrix-free column sums
and images are checked against the oracle run on the stored matrix of the
same geometry: column sums within 1e-5 relative L2 (the tolerance of one
projection), MLEM images within 1e-4 (the hot path's tolerance), for a
power-of-two grid (Morton parts from tables) and an odd grid (ranked Morton
order through the permutation).
"""
import numpy as np
import pytest

import oracle_bind as ob
from mlem_b200 import api, synth

pytestmark = pytest.mark.gpu

GEOMS = [synth.GEOM_SMALL, synth.Geometry(20, 24, 12, 20000, 10, 60, seed=9)]


def _sino(m, g, seed):
    x = synth.phantom(g.nx, g.ny, g.nz, 5, seed)
    return synth.poisson_sinogram(synth.project_f64(m, x), 1e6, seed + 1)


@pytest.mark.parametrize("g", GEOMS, ids=["32x32x16", "20x24x12"])
def test_matrix_free_matches_the_stored_matrix(g):
    m = synth.host_matrix(g)
    sino = _sino(m, g, 41)
    with api.MatrixFree(g) as mf:
        assert ob.rel_l2(mf.column_sums(), ob.column_sums(m)) <= 1e-5
        mf.set_sinogram(sino)
        init = mf.init_image()
        norm = ob.column_sums(m)
        assert abs(init - ob.init_value(norm, sino)) <= 1e-5 * abs(init)
        mf.iterate(10)
        img = mf.get_image()
    want, _ = ob.mlem(m, sino, 10)
    assert ob.rel_l2(img, want) <= 1e-4, ob.rel_l2(img, want)
    assert ob.rel_l2(img, ob.mlem_f64(m, sino, 10)) <= 1e-4


def test_matrix_free_skips_rays_without_counts():
    g = synth.GEOM_SMALL
    m = synth.host_matrix(g)
    sino = _sino(m, g, 43)
    sino[::3] = 0
    with api.MatrixFree(g) as mf:
        mf.set_sinogram(sino)
        mf.init_image()
        for _ in range(4):
            mf.iterate(1)
        img = mf.get_image()
    want, _ = ob.mlem(m, sino, 4)
    assert ob.rel_l2(img, want) <= 1e-4


def test_matrix_free_refuses_bad_use():
    g = synth.GEOM_SMALL
    with api.MatrixFree(g) as mf:
        with pytest.raises(api.MlemError) as e:
            mf.iterate(1)
        assert e.value.status == api.MLEM_ERR_STATE
        with pytest.raises(api.MlemError):
            mf.set_sinogram(np.zeros(g.n_rows - 1, np.int32))
