"""C-ABI host logic on CPU: exports, file formats, checkpoints, partition, CLI
argument handling.  No GPU calls."""
import ctypes
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from mlem_b200 import _capi_sig, api, formats, synth
from mlem_b200._native import CLI_PATH, CORE_PATH, core_lib

import oracle_bind as ob


def test_library_exports_every_header_symbol():
    lib = core_lib()
    names = [p[0] for p in _capi_sig.prototypes()]
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n
    # and nothing the header does not declare
    out = subprocess.run(["nm", "-D", "--defined-only", CORE_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mlem_\w+)", out))
    assert exported == set(names)


def test_status_strings_and_version():
    lib = core_lib()
    assert lib.mlem_version() == 1
    assert lib.mlem_status_string(api.MLEM_ERR_FORMAT) == b"bad file format"


def test_csr4_roundtrip_python_writer_c_reader(tmp_path, golden):
    m, *_ = golden.case("edge_it7")
    p = tmp_path / "m.csr4"
    formats.write_csr4(p, m.n_rows, m.n_cols, m.row_end, m.elems, grid=(4, 4, 4))
    h, row_end, elems = api.csr4_read(str(p))
    assert (h["n_rows"], h["n_cols"], h["nnz"], h["grid"]) == (m.n_rows, m.n_cols, m.nnz, (4, 4, 4))
    assert h["scan_config_bytes"] == 60 and h["data_offset"] == 88
    assert np.array_equal(row_end, m.row_end)
    assert elems.tobytes() == np.ascontiguousarray(m.elems).tobytes()


def test_csr4_c_writer_matches_python_writer(tmp_path, golden):
    m, *_ = golden.case("tiny_it10")
    a, b = tmp_path / "a.csr4", tmp_path / "b.csr4"
    formats.write_csr4(a, m.n_rows, m.n_cols, m.row_end, m.elems, grid=(8, 8, 4))
    api.csr4_write(str(b), m.row_end, m.elems, m.n_rows, m.n_cols, grid=(8, 8, 4))
    assert a.read_bytes() == b.read_bytes()
    # and the committed golden file (read by the reference binary) parses
    h, *_ = api.csr4_read(os.path.join(golden.GOLDEN, "tiny.csr4"))
    assert h["n_rows"] == 512


def _good(tmp_path):
    p = tmp_path / "g.csr4"
    re_ = np.array([2, 3], np.uint64)
    el = np.zeros(3, api.ELEM_DTYPE)
    el["index"] = [0, 1, 1]
    el["value"] = [1, 2, 3]
    formats.write_csr4(p, 2, 2, re_, el)
    return p, p.read_bytes()


@pytest.mark.parametrize("mutate,needle", [
    (lambda b: b[:20], "File too short"),
    (lambda b: b"XCSR" + b[4:], "is not a CSR matrix"),
    (lambda b: b[:4] + b"\x03" + b[5:], "wrong CSR version"),
    (lambda b: b[:-4], "is too short"),
    (lambda b: b[:24] + struct.pack("<I", 56) + b[28:], "Cannot find scanner geometry"),
    (lambda b: b[:24] + struct.pack("<I", 64) + b[28:] + b"\0" * 4, "Error reading scanner geometry"),
])
def test_csr4_header_errors_like_reference(tmp_path, mutate, needle):
    p, raw = _good(tmp_path)
    bad = tmp_path / "bad.csr4"
    bad.write_bytes(mutate(raw))
    with pytest.raises(api.MlemError) as e:
        api.csr4_header(str(bad))
    assert needle in str(e.value)
    assert e.value.status in (api.MLEM_ERR_FORMAT, api.MLEM_ERR_IO)


def test_csr4_missing_file(tmp_path):
    with pytest.raises(api.MlemError) as e:
        api.csr4_header(str(tmp_path / "nope.csr4"))
    assert e.value.status == api.MLEM_ERR_IO and "Cannot open file" in e.value.message


def test_vector_io(tmp_path):
    a = np.arange(17, dtype=np.int32)
    p = tmp_path / "v.bin"
    api.vector_write(str(p), a, sync=True)
    assert np.array_equal(api.vector_read(str(p), np.int32), a)
    p.write_bytes(p.read_bytes() + b"\x01")  # not a multiple of 4: vector.hpp:43-44
    with pytest.raises(api.MlemError):
        api.vector_read(str(p), np.int32)
    empty = tmp_path / "e.bin"
    empty.write_bytes(b"")
    assert api.vector_read(str(empty), np.float32).size == 0


def test_checkpoint_protocol(tmp_path):
    d = str(tmp_path)
    assert api.checkpoint_read(d, 5) is None
    img = np.linspace(0, 1, 5, dtype=np.float32)
    api.checkpoint_write(d, img, 7)
    assert (tmp_path / "img.chkpt").read_bytes() == img.tobytes()
    assert struct.unpack("<i", (tmp_path / "iter.chkpt").read_bytes())[0] == 7
    got, it = api.checkpoint_read(d, 5)
    assert it == 7 and np.array_equal(got, img)
    # size mismatch is an error (vector.hpp:131-134)
    with pytest.raises(api.MlemError):
        api.checkpoint_read(d, 6)
    # exactly one file present: ignored (mpicsr4mlem.cpp:545-550)
    os.remove(tmp_path / "iter.chkpt")
    assert api.checkpoint_read(d, 5) is None
    api.checkpoint_write(d, img, 7)
    api.checkpoint_remove(d)
    assert not (tmp_path / "img.chkpt").exists() and not (tmp_path / "iter.chkpt").exists()
    # python mirror agrees
    api.checkpoint_write(d, img, 3)
    got2, it2 = formats.read_checkpoint(d, 5)
    assert it2 == 3 and np.array_equal(got2, img)


def test_partition_matches_oracle(golden):
    for name in ("tiny_it10", "plain_small_it10", "edge_it7"):
        m, *_ = golden.case(name)
        for n in (1, 2, 3, 4, 8):
            s, e = api.partition_rows(m.row_end, n)
            so, eo = ob.partition(m, n)
            assert np.array_equal(s, so) and np.array_equal(e, eo), (name, n)


def _cli(args, cwd):
    return subprocess.run([CLI_PATH] + args, cwd=cwd, capture_output=True, text=True, timeout=60)


def test_cli_rejects_wrong_argument_count(tmp_path):
    for args in ([], ["a", "b", "c"], ["a", "b", "c", "1", "2", "3"]):
        p = _cli(args, tmp_path)
        assert p.returncode != 0
        assert "wrong number of command line parameters" in p.stderr


def test_cli_reports_bad_matrix_before_touching_a_gpu(tmp_path):
    bad = tmp_path / "m.csr4"
    bad.write_bytes(b"NOPE" + b"\0" * 100)
    p = _cli([str(bad), "s", "o", "3"], tmp_path)
    assert p.returncode != 0 and "is not a CSR matrix" in p.stderr


def test_cli_rejects_bad_iterations(tmp_path):
    p = _cli(["m", "s", "o", "ten"], tmp_path)
    assert p.returncode != 0 and "invalid iterations" in p.stderr


def test_host_generator_is_deterministic_and_in_window():
    g = synth.Geometry(16, 16, 8, 4096, 10, 40, seed=5)
    a, b = synth.host_matrix(g), synth.host_matrix(g)
    assert np.array_equal(a.row_end, b.row_end) and a.elems.tobytes() == b.elems.tobytes()
    counts = np.diff(a.row_ptr()).astype(np.int64)
    assert counts.min() >= 1 and counts.max() <= 40
    assert (counts >= 10).mean() > 0.99
    assert a.vals.min() >= 1e-4 and a.vals.max() <= np.sqrt(3.0) + 1e-6
    assert a.cols.max() < g.n_cols
    # projection helper agrees with the oracle's double projection bit for bit
    x = synth.phantom(16, 16, 8, 3, 1)
    assert np.array_equal(synth.project_f64(a, x), ob.project_f64(a, x))
