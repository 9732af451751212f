"""Loader of the golden fixtures made by tests/golden/make_golden.py."""
from __future__ import annotations

import functools
import hashlib
import json
import os
import tempfile

import numpy as np

from mlem_b200 import formats, synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@functools.lru_cache(None)
def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def _sha(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        h.update(f.read())
    return h.hexdigest()


@functools.lru_cache(None)
def case(name):
    """(matrix Csr4, sinogram int32, iterations, golden image float32, entry)."""
    c = manifest()["cases"][name]
    if c.get("workload"):
        w = synth.WORKLOADS[c["workload"]]
        m, frames = synth.host_workload(w)
        sino = frames.sinograms[0]
        with tempfile.TemporaryDirectory() as td:
            mp, sp = os.path.join(td, "m.csr4"), os.path.join(td, "s.sino")
            g = w.geometry
            formats.write_csr4(mp, m.n_rows, m.n_cols, m.row_end, m.elems, grid=(g.nx, g.ny, g.nz))
            formats.write_vector(sp, sino, np.int32)
            if _sha(mp) != c["matrix_sha256"] or _sha(sp) != c["sino_sha256"]:
                raise AssertionError(f"regenerated inputs of {name} differ from the golden hashes")
    else:
        mp = os.path.join(GOLDEN, c["matrix"])
        sp = os.path.join(GOLDEN, c["sino"])
        assert _sha(mp) == c["matrix_sha256"] and _sha(sp) == c["sino_sha256"]
        m = formats.read_csr4(mp, mmap=False)
        sino = formats.read_vector(sp, np.int32)
    img = formats.read_vector(os.path.join(GOLDEN, c["image"]), np.float32)
    return m, sino, c["iterations"], img, c


CASES = ("tiny_it10", "tiny_it100", "edge_it7", "plain_small_it10")
