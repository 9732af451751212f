"""The oracle's expansion of symmetry-compressed CSR4 matrices.

The reference regenerates the elements a symmetric scanner's matrix omits
only in its viewer (visualizematrix/dispcsr4spy.cpp:123-140, with the mirror
tables of symhandler.cpp:33-114).  These tests check oracle_expand_symmetries
against a direct Python restatement of those loops and tables, and the
tables' own properties.
"""
import numpy as np
import pytest

import oracle_bind as ob
from mlem_b200 import formats

SCANNER = (1, 4, 3, 2)  # layers, blocks, block size, rings: 24 crystals, 576 LORs
GRID = (8, 8, 4)


def sym_matrix(sym, seed=0, scanner=SCANNER, grid=GRID, fill=0.4):
    rng = np.random.default_rng(seed)
    nl, nb, bs, nr = scanner
    nc = nl * nb * bs * nr
    R, C = nc * nc, int(np.prod(grid))
    lens = np.where(rng.random(R) < fill, rng.integers(1, 20, R), 0)
    row_end = np.cumsum(lens).astype(np.uint64)
    el = np.zeros(int(row_end[-1]), formats.ELEM_DTYPE)
    el["index"] = rng.integers(0, C, el.size)
    el["value"] = rng.uniform(0.1, 1.7, el.size).astype(np.float32)
    return formats.Csr4(R, C, row_end, el, sym, grid, (1.0, 1.0, 1.0), scanner)


def luts(scanner):
    """symhandler.cpp initLUTs, written out table by table."""
    nl, nb, bs, nr = scanner
    per_layer, n = bs * nb, bs * nb * nl * nr
    per_ring = per_layer * nl
    lut = np.zeros((8, n), np.int64)
    lut[0] = np.arange(n)
    for r in range(nr):
        for l in range(nl):
            for v in range(per_layer):
                base = l * per_layer + r * per_ring
                lut[1][v + base] = (per_layer - v + bs - 1) % per_layer + base
                lut[2][v + base] = (per_layer - v + bs * (nb // 2 + 1) - 1) % per_layer + base
    for r in range(nr):
        for v in range(per_ring):
            lut[4][v + r * per_ring] = v + (nr - 1 - r) * per_ring
    lut[3] = lut[2][lut[1]]
    lut[5] = lut[4][lut[1]]
    lut[6] = lut[4][lut[2]]
    lut[7] = lut[4][lut[2][lut[1]]]
    return lut


def expand_py(m):
    """dispcsr4spy.cpp fillTiles (version 2) as a matrix: stored rows, then
    every generated symmetry's transformed rows."""
    nl, nb, bs, nr = m.scanner
    nc = nl * nb * bs * nr
    nx, ny, nz = m.grid
    lut = luts(m.scanner)
    sx, sy, sz = m.flags & 1, (m.flags >> 1) & 1, (m.flags >> 2) & 1
    syms = [(x, y, z) for x in range(sx + 1) for y in range(sy + 1) for z in range(sz + 1)
            if (x, y, z) != (0, 0, 0)]
    rows = [[] for _ in range(m.n_rows)]
    begin = np.concatenate([[0], m.row_end[:-1]]).astype(np.int64)
    for r in range(m.n_rows):
        rows[r] += [(int(c), float(v)) for c, v in m.elems[begin[r]:int(m.row_end[r])]]
    for x, y, z in syms:
        t = lut[x + 2 * y + 4 * z]
        for r in range(m.n_rows):
            d1, d2 = t[r // nc], t[r % nc]
            rt = d1 * nc + d2 if d1 < d2 else d2 * nc + d1
            for c, v in m.elems[begin[r]:int(m.row_end[r])]:
                zz, rem = divmod(int(c), nx * ny)
                yy, xx = divmod(rem, nx)
                if x: xx = nx - 1 - xx
                if y: yy = ny - 1 - yy
                if z: zz = nz - 1 - zz
                rows[rt].append((zz * nx * ny + yy * nx + xx, float(v)))
    return rows


@pytest.mark.parametrize("sym", [1, 2, 4, 5, 7])
def test_oracle_expansion_matches_viewer_loops(sym):
    m = sym_matrix(sym, seed=sym)
    full = ob.expand_symmetries(m)
    rows = expand_py(m)
    begin = np.concatenate([[0], full.row_end[:-1]]).astype(np.int64)
    for r in range(m.n_rows):
        got = full.elems[begin[r]:int(full.row_end[r])]
        assert [int(c) for c in got["index"]] == [c for c, _ in rows[r]], r
        np.testing.assert_array_equal(got["value"], np.array([v for _, v in rows[r]], np.float32))
    assert full.nnz == m.nnz * (1 + len([1 for x in range((sym & 1) + 1) for y in range(((sym >> 1) & 1) + 1)
                                          for z in range(((sym >> 2) & 1) + 1)]) - 1)


def test_mirror_tables_are_involutions():
    lut = luts(SCANNER)
    for m in (1, 2, 4):
        assert np.array_equal(lut[m][lut[m]], lut[0])
        assert sorted(lut[m]) == list(range(lut.shape[1]))


def test_no_symmetry_is_the_stored_matrix():
    m = sym_matrix(0, seed=3)
    full = ob.expand_symmetries(m)
    assert full.elems.tobytes() == np.ascontiguousarray(m.elems).tobytes()
    assert np.array_equal(full.row_end, m.row_end)


def test_mirrored_workload_scanner():
    """The bench's symmetry-compressed workload reads an n^2-LOR matrix as a
    scanner of n crystals (n a multiple of 512)."""
    from mlem_b200 import mirrored

    assert mirrored.scanner_for(4194304) == (1, 32, 16, 4)
    nl, nb, bs, nr = mirrored.scanner_for(1048576)
    assert nl * nb * bs * nr == 1024
    for bad in (1000, 512 * 512 + 1, 256 * 256):
        with pytest.raises(ValueError):
            mirrored.scanner_for(bad)
