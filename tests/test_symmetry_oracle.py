"""The oracle's expansion of symmetry-compressed CSR4 matrices.

The reference regenerates the elements a symmetric scanner's matrix omits
only in its viewer (visualizematrix/dispcsr4spy.cpp:123-140, with the mirror
tables of symhandler.cpp:33-114).  These tests pin oracle_expand_symmetries
to the reference's own SymHandler: tests/golden/sym_ref.npz holds its
generateSyms order and transformLor / transformVoxel / transformDetector
results, recorded by tests/golden/make_sym_golden.py from the reference's
symhandler.cpp compiled unmodified (oracle/_ref/libref_sym.so).  They also
check a direct Python restatement of the viewer's loops and tables, and the
tables' own properties.
"""
import os

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


SYM_REF = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sym_ref.npz")


def _ref(case):
    d = np.load(SYM_REF)
    return {k[len(case) + 1:]: d[k] for k in d.files if k.startswith(case + "_")}


def _expand_with(m, ref, rows_of_interest=None):
    """The viewer's loops (dispcsr4spy.cpp:115-140: the stored rows, then for
    every generated symmetry each row's elements at transformLor(row) with
    transformVoxel(column)), with the reference's recorded transforms."""
    lor_idx = {int(r): i for i, r in enumerate(ref["lors"])}
    vox_idx = {}
    for i, v in enumerate(ref["voxels"]):
        vox_idx.setdefault(int(v), i)
    sym = m.flags
    masks = [int(x) for x in ref["gen"][sym] if x]
    begin = np.concatenate([[0], m.row_end[:-1]]).astype(np.int64)
    rows = range(m.n_rows) if rows_of_interest is None else rows_of_interest
    out = {}
    for r in rows:
        out.setdefault(r, []).extend(
            (int(c), float(v)) for c, v in m.elems[begin[r]:int(m.row_end[r])])
    for mask in masks:
        for r in rows:
            el = m.elems[begin[r]:int(m.row_end[r])]
            if not len(el):
                continue
            t = int(ref["lor_t"][mask][lor_idx[r]])
            out.setdefault(t, []).extend(
                (int(ref["vox_t"][mask][vox_idx[int(c)]]), float(v)) for c, v in el)
    return out


def _check(full, want):
    begin = np.concatenate([[0], full.row_end[:-1]]).astype(np.int64)
    nonempty = np.flatnonzero(np.diff(np.concatenate([[0], full.row_end]).astype(np.int64)))
    assert set(int(r) for r in nonempty) == {r for r, v in want.items() if v}
    for r, items in want.items():
        got = full.elems[begin[r]:int(full.row_end[r])]
        assert [int(c) for c in got["index"]] == [c for c, _ in items], r
        np.testing.assert_array_equal(got["value"], np.array([v for _, v in items], np.float32))


@pytest.mark.parametrize("case", ["a", "b"])
@pytest.mark.parametrize("sym", [1, 2, 3, 4, 5, 6, 7])
def test_oracle_expansion_equals_the_reference_symhandler(case, sym):
    ref = _ref(case)
    scanner = tuple(int(x) for x in ref["scanner"])
    grid = tuple(int(x) for x in ref["grid"])
    m = sym_matrix(sym, seed=10 * sym + ord(case), scanner=scanner, grid=grid)
    _check(ob.expand_symmetries(m), _expand_with(m, ref))


@pytest.mark.parametrize("sym", [5, 7])
def test_oracle_expansion_on_the_bench_scanner_sample(sym):
    """The 2,048-crystal scanner of the bench's mirrored workload: a sparse
    matrix whose rows and voxels are the recorded sample."""
    ref = _ref("c")
    scanner = tuple(int(x) for x in ref["scanner"])
    grid = tuple(int(x) for x in ref["grid"])
    nc = int(np.prod(scanner))
    R, C = nc * nc, int(np.prod(grid))
    rng = np.random.default_rng(sym)
    rows = np.sort(ref["lors"]).astype(np.int64)
    lens = np.zeros(R, np.int64)
    lens[rows] = rng.integers(1, 4, rows.size)
    row_end = np.cumsum(lens).astype(np.uint64)
    el = np.zeros(int(row_end[-1]), formats.ELEM_DTYPE)
    el["index"] = rng.choice(ref["voxels"], el.size)
    el["value"] = rng.uniform(0.1, 1.7, el.size).astype(np.float32)
    m = formats.Csr4(R, C, row_end, el, sym, grid, (1.0, 1.0, 1.0), scanner)
    _check(ob.expand_symmetries(m), _expand_with(m, ref, [int(r) for r in rows]))


@pytest.mark.parametrize("case", ["a", "b", "c"])
def test_restated_tables_equal_the_reference_luts(case):
    ref = _ref(case)
    scanner = tuple(int(x) for x in ref["scanner"])
    assert np.array_equal(luts(scanner), ref["det_t"].astype(np.int64))
    # generateSyms: x outermost, identity left out
    for sym in range(8):
        want = [x | (y << 1) | (z << 2) for x in range((sym & 1) + 1)
                for y in range(((sym >> 1) & 1) + 1) for z in range(((sym >> 2) & 1) + 1)
                if x or y or z]
        assert [int(v) for v in ref["gen"][sym] if v] == want


def test_recorded_tables_match_the_reference_library():
    """Where the reference's SymHandler is built (oracle/_ref/libref_sym.so),
    the committed tables are what it returns today."""
    lib = os.path.join(ob.REF_DIR, "libref_sym.so")
    if not os.path.exists(lib):
        pytest.skip("oracle/_ref/libref_sym.so is not built here")
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_sym_golden", os.path.join(os.path.dirname(SYM_REF), "make_sym_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    L = mk.load()
    for case, (scanner, grid, sample) in mk.CASES.items():
        ref = _ref(case)
        for got, key in zip(mk.tables(L, scanner, grid, sample),
                            ("gen", "lors", "lor_t", "voxels", "vox_t", "det_t")):
            assert np.array_equal(got, ref[key]), (case, key)
