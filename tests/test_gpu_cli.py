"""The command-line drop-in (bin/mlem_b200) on the GPU: same arguments and
files as seqcsr4mlem, checkpoint/restart interchange, batched inputs."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from mlem_b200 import formats
from mlem_b200._native import CLI_PATH

import oracle_bind as ob

pytestmark = pytest.mark.gpu


def run(args, cwd, env=None):
    e = dict(os.environ)
    e.update(env or {})
    p = subprocess.run([CLI_PATH] + [str(a) for a in args], cwd=cwd, capture_output=True,
                       text=True, timeout=300, env=e)
    assert p.returncode == 0, p.stderr
    return p.stdout


@pytest.fixture
def tiny(tmp_path, golden):
    src = golden.GOLDEN
    shutil.copy(os.path.join(src, "tiny.csr4"), tmp_path / "m.csr4")
    shutil.copy(os.path.join(src, "tiny.sino"), tmp_path / "s.sino")
    return tmp_path


def test_cli_matches_reference_image(tiny, golden):
    out = run(["m.csr4", "s.sino", "out.img", 10], tiny)
    assert "Finished iteration 10" in out and "image sum" in out
    img = formats.read_vector(tiny / "out.img", np.float32)
    gold = formats.read_vector(os.path.join(golden.GOLDEN, "tiny_it10.image"), np.float32)
    assert ob.rel_l2(img, gold) <= 1e-4


def test_cli_exact_mode_bit_exact(tiny, golden):
    run(["m.csr4", "s.sino", "out.img", 100], tiny, {"MLEM_B200_EXACT": "1"})
    img = formats.read_vector(tiny / "out.img", np.float32)
    gold = formats.read_vector(os.path.join(golden.GOLDEN, "tiny_it100.image"), np.float32)
    assert img.tobytes() == gold.tobytes()


def test_cli_checkpoint_restart_is_bit_identical(tiny):
    run(["m.csr4", "s.sino", "full.img", 10], tiny)
    full = formats.read_vector(tiny / "full.img", np.float32)
    # with checkpointing every 3 iterations: same result, no files left behind
    run(["m.csr4", "s.sino", "chk.img", 10, 3], tiny)
    assert formats.read_vector(tiny / "chk.img", np.float32).tobytes() == full.tobytes()
    assert not (tiny / "img.chkpt").exists() and not (tiny / "iter.chkpt").exists()
    # a run "killed" after iteration 6: its checkpoint files, then a restart
    run(["m.csr4", "s.sino", "six.img", 6], tiny)
    six = formats.read_vector(tiny / "six.img", np.float32)
    formats.write_vector(tiny / "img.chkpt", six, np.float32, sync=True)
    (tiny / "iter.chkpt").write_bytes(struct.pack("<i", 6))
    out = run(["m.csr4", "s.sino", "restart.img", 10, 5], tiny)
    assert "Checkpoint at iteration 6" in out and "Starting 4 MLEM iterations" in out
    assert formats.read_vector(tiny / "restart.img", np.float32).tobytes() == full.tobytes()
    assert not (tiny / "img.chkpt").exists()


def test_cli_ignores_incomplete_checkpoint(tiny):
    run(["m.csr4", "s.sino", "full.img", 4], tiny)
    (tiny / "iter.chkpt").write_bytes(struct.pack("<i", 3))  # image file missing
    out = run(["m.csr4", "s.sino", "x.img", 4, 2], tiny)
    assert "omitted incomplete checkpoint" in out and "Starting 4 MLEM iterations" in out
    a = formats.read_vector(tiny / "full.img", np.float32)
    assert formats.read_vector(tiny / "x.img", np.float32).tobytes() == a.tobytes()


def test_cli_rejects_wrong_sinogram_length(tiny):
    (tiny / "bad.sino").write_bytes(np.zeros(7, np.int32).tobytes())
    p = subprocess.run([CLI_PATH, "m.csr4", "bad.sino", "o", "2"], cwd=tiny, capture_output=True,
                       text=True, timeout=120)
    assert p.returncode != 0 and "rows" in p.stderr


def test_cli_batched_lists(tiny, golden):
    s = formats.read_vector(tiny / "s.sino", np.int32)
    formats.write_vector(tiny / "s2.sino", np.roll(s, 7), np.int32)
    run(["m.csr4", "s.sino,s2.sino", "a.img,b.img", 10], tiny)
    m = formats.read_csr4(tiny / "m.csr4", mmap=False)
    for name, sino in (("a.img", s), ("b.img", np.roll(s, 7))):
        want, _ = ob.mlem(m, sino, 10)
        assert ob.rel_l2(formats.read_vector(tiny / name, np.float32), want) <= 1e-4
