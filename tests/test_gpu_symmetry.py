"""Symmetry-compressed CSR4 matrices on the GPU (mlem_create_symmetric,
MLEM_FLAG_EXPAND_SYMMETRY): the device expansion equals the oracle's
restatement of the reference viewer's regeneration bit for bit, and MLEM on
it matches the oracle's MLEM on the expanded matrix.  Without the flag a file
keeps the reference drivers' behaviour: its symmetry flags are ignored."""
import os
import subprocess

import numpy as np
import pytest

from mlem_b200 import api, formats

import oracle_bind as ob
from test_symmetry_oracle import GRID, SCANNER, sym_matrix

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "mlem_b200", "bin", "mlem_b200")


def _sino(m, seed=1):
    return np.random.default_rng(seed).poisson(20, m.n_rows).astype(np.int32)


@pytest.mark.parametrize("sym", [1, 2, 4, 5, 7])
def test_expansion_is_bit_exact(sym):
    m = sym_matrix(sym, seed=10 + sym)
    full = ob.expand_symmetries(m)
    with api.Context.symmetric(m) as ctx:
        assert ctx.nnz == full.nnz
        re_, el = ctx.csr()
        assert np.array_equal(re_, full.row_end)
        assert el.tobytes() == np.ascontiguousarray(full.elems).tobytes()
        assert ctx.column_sums().tobytes() == ob.column_sums(full).tobytes()


@pytest.mark.parametrize("sym", [5, 7])
@pytest.mark.parametrize("mode,visit", [(api.BK_CSC, api.VISIT_FILE),
                                        (api.BK_FUSED, api.VISIT_SORTED_CHUNKED),
                                        (api.BK_FUSED, api.VISIT_SORTED_STAGED),
                                        (api.BK_ATOMIC, api.VISIT_SORTED)])
def test_mlem_on_the_full_matrix(sym, mode, visit):
    m = sym_matrix(sym, seed=20 + sym)
    full = ob.expand_symmetries(m)
    sino = _sino(m)
    want, _ = ob.mlem(full, sino, 8)
    with api.Context.symmetric(m) as ctx:
        ctx.set_sinograms(sino)
        ctx.set_tuning(bk_mode=mode, group=32, frame_tile=1, blocks_per_sm=4, visit=visit)
        ctx.init_images()
        ctx.iterate(8)
        assert ob.rel_l2(ctx.get_images()[0], want) <= 1e-4


def test_exact_mode_on_the_full_matrix():
    m = sym_matrix(7, seed=31)
    full = ob.expand_symmetries(m)
    sino = _sino(m)
    want, _ = ob.mlem(full, sino, 6)
    with api.Context.symmetric(m, flags=api.FLAG_EXACT) as ctx:
        img, _ = api.mlem(ctx, sino, nIterations=6)
        assert img[0].tobytes() == want.tobytes()


def test_file_flag_and_cli(tmp_path):
    m = sym_matrix(7, seed=41)
    path = str(tmp_path / "sym.csr4")
    formats.write_csr4(path, m.n_rows, m.n_cols, m.row_end, m.elems, grid=GRID, flags=7,
                       scanner=SCANNER)
    back = formats.read_csr4(path, mmap=False)
    assert back.scanner == SCANNER and back.flags == 7
    full = ob.expand_symmetries(m)
    with api.Context.from_file(path, flags=api.FLAG_EXPAND_SYMMETRY) as ctx:
        assert ctx.csr()[1].tobytes() == np.ascontiguousarray(full.elems).tobytes()
    with api.Context.from_file(path) as ctx:  # the reference drivers' behaviour
        assert ctx.csr()[1].tobytes() == np.ascontiguousarray(m.elems).tobytes()
    sino = _sino(m)
    sp, out = str(tmp_path / "s.sino"), str(tmp_path / "img.out")
    formats.write_vector(sp, sino, np.int32)
    env = dict(os.environ, MLEM_B200_EXPAND_SYMMETRY="1", MLEM_B200_EXACT="1")
    subprocess.run([CLI, path, sp, out, "5"], check=True, env=env, capture_output=True)
    want, _ = ob.mlem(full, sino, 5)
    assert formats.read_vector(out, np.float32).tobytes() == want.tobytes()


def test_rejects_inconsistent_geometry():
    m = sym_matrix(7, seed=51)
    bad = formats.Csr4(m.n_rows, m.n_cols, m.row_end, m.elems, 7, (8, 8, 5), (1.0, 1.0, 1.0),
                       SCANNER)
    with pytest.raises(api.MlemError):
        api.Context.symmetric(bad)  # 320 voxels in the grid, 256 columns
    bad = formats.Csr4(m.n_rows, m.n_cols, m.row_end, m.elems, 7, GRID, (1.0, 1.0, 1.0),
                       (1, 4, 3, 3))
    with pytest.raises(api.MlemError):
        api.Context.symmetric(bad)  # 36 crystals: 1296 LORs, not 576
    el = np.array(m.elems)
    el["index"][0] = m.n_cols  # out of range: rejected before mirroring
    bad = formats.Csr4(m.n_rows, m.n_cols, m.row_end, el, 7, GRID, (1.0, 1.0, 1.0), SCANNER)
    with pytest.raises(api.MlemError):
        api.Context.symmetric(bad)
