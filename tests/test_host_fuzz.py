"""Malformed inputs to the host-side C ABI: the CSR4 header reader (the
command-line driver's loader) and the matrix checks of mlem_create must
answer with an error status, never crash or read out of bounds.  The random
mutations run in a child process so that a crash fails this test instead of
ending the test run."""
import subprocess
import sys

FUZZ = r'''
import os, struct, sys, tempfile
import numpy as np
sys.path.insert(0, sys.argv[1])
from mlem_b200 import api, formats
rng = np.random.default_rng(12345)
d = tempfile.mkdtemp()
good = os.path.join(d, "good.csr4")
re_ = np.array([3, 5, 5, 9], np.uint64)
el = np.zeros(9, formats.ELEM_DTYPE)
el["index"] = rng.integers(0, 8, 9)
el["value"] = rng.uniform(0.1, 1.0, 9).astype(np.float32)
formats.write_csr4(good, 4, 8, re_, el, grid=(2, 2, 2), flags=7, scanner=(2, 3, 2, 2))
raw = open(good, "rb").read()
ok = err = 0
for i in range(3000):
    b = bytearray(raw)
    kind = i % 3
    if kind == 0:  # flip bytes in the header and scanner block
        for _ in range(int(rng.integers(1, 6))):
            b[int(rng.integers(0, 28 + 4 * 24))] = int(rng.integers(0, 256))
    elif kind == 1:  # truncate anywhere
        b = b[: int(rng.integers(0, len(b)))]
    else:  # overwrite one 32-bit field of the scanner block with an extreme value
        off = 28 + 4 * int(rng.integers(0, 24))
        if off + 4 <= len(b):
            b[off:off + 4] = struct.pack("<I", int(rng.choice([0, 1, 2**31 - 1, 2**32 - 1, 1 << 20])))
    p = os.path.join(d, "m.csr4")
    open(p, "wb").write(bytes(b))
    try:
        h = api.csr4_header(p)
        if h["n_rows"] <= 1000 and h["nnz"] <= 10000:
            api.csr4_read(p)
        ok += 1
    except api.MlemError as e:
        assert e.status in (api.MLEM_ERR_FORMAT, api.MLEM_ERR_IO, api.MLEM_ERR_INVALID), e.status
        err += 1
# the matrix checks of mlem_create run on the host before any device work
for i in range(500):
    R = int(rng.integers(1, 50))
    re_ = np.sort(rng.integers(0, 100, R)).astype(np.uint64)
    if i % 2:
        re_[int(rng.integers(0, R))] = rng.integers(0, 100)  # may decrease
    nnz = int(re_[-1]) if i % 3 else int(re_[-1]) + 1         # may disagree with the offsets
    el = np.zeros(max(nnz, 1), formats.ELEM_DTYPE)
    try:
        api.Context(re_, el[:nnz], R, 8).close()
        ok += 1
    except api.MlemError:
        err += 1
print(ok, err)
'''


def test_malformed_inputs_give_errors_not_crashes():
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", FUZZ, root], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    ok, err = map(int, p.stdout.split()[-2:])
    assert err > 0 and ok + err == 3500
