"""The oracle's command-line tool (oracle/_bin/oracle_tool), which the bench
runs beside the GPU work: the threaded FP64 oracle must agree with the serial
one, and its generator and projection must write the same bytes as the
package's (so the reference arm, which uses the tool, times the same inputs)."""
import os
import subprocess

import numpy as np
import pytest

import oracle_bind as ob
from mlem_b200 import formats, synth

TOOL = os.path.join(ob.ORACLE_DIR, "_bin", "oracle_tool")


@pytest.fixture(scope="module")
def tool():
    if not os.path.exists(TOOL):
        subprocess.run(["make", "-C", ob.ORACLE_DIR, TOOL], check=True, capture_output=True)
    return TOOL


def test_threaded_f64_oracle_matches_the_serial_one(tmp_path, golden, tool):
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    mp, sp, out = tmp_path / "m.csr4", tmp_path / "s.sino", tmp_path / "x.f64"
    formats.write_csr4(mp, m.n_rows, m.n_cols, m.row_end, m.elems)
    formats.write_vector(sp, sino, "int32")
    serial = ob.mlem_f64(m, sino, iters)
    for threads in (1, 3, 8):
        subprocess.run([tool, "f64-mlem", str(mp), str(sp), str(iters), str(threads), str(out)],
                       check=True, capture_output=True)
        got = np.fromfile(out, np.float64)
        if threads == 1:
            assert got.tobytes() == serial.tobytes()  # one block: the serial order exactly
        assert ob.rel_l2(got, serial) <= 1e-13
    # the float reference binary's image is within its float error of the FP64 one
    assert ob.rel_l2(gold, got) <= 1e-4


def test_tool_generator_and_projection_write_the_package_bytes(tmp_path, tool):
    g = synth.GEOM_SMALL
    mp = tmp_path / "tool.csr4"
    subprocess.run([tool, "synth-matrix", str(g.nx), str(g.ny), str(g.nz), str(g.n_rows),
                    str(g.min_count), str(g.max_count), str(g.seed), repr(g.radius_scale),
                    repr(g.min_len), str(mp)], check=True, capture_output=True)
    m = synth.host_matrix(g)
    ref = tmp_path / "pkg.csr4"
    formats.write_csr4(ref, m.n_rows, m.n_cols, m.row_end, m.elems, grid=(g.nx, g.ny, g.nz))
    assert mp.read_bytes() == ref.read_bytes()
    x = synth.phantom(g.nx, g.ny, g.nz, 5, 17)
    xp, op = tmp_path / "x.f32", tmp_path / "p.f64"
    x.astype(np.float32).tofile(xp)
    subprocess.run([tool, "project-f64", str(mp), str(xp), str(op)], check=True,
                   capture_output=True)
    assert np.fromfile(op, np.float64).tobytes() == synth.project_f64(m, x).tobytes()


def test_tool_rejects_a_sinogram_of_the_wrong_length(tmp_path, golden, tool):
    m, sino, *_ = golden.case("tiny_it10")
    mp, sp = tmp_path / "m.csr4", tmp_path / "s.sino"
    formats.write_csr4(mp, m.n_rows, m.n_cols, m.row_end, m.elems)
    formats.write_vector(sp, sino[:-1], "int32")
    p = subprocess.run([tool, "f64-mlem", str(mp), str(sp), "1", "2", str(tmp_path / "o")],
                       capture_output=True, text=True)
    assert p.returncode != 0 and "sinogram length" in p.stderr
