"""Generate the golden fixtures by running the reference's own seqcsr4mlem.

Run from the repository root after `make -C oracle` (which compiles
oracle/_ref/seqcsr4mlem from the reference sources):

    python tests/golden/make_golden.py

Each case writes the reference's inputs and its output image here, plus a
manifest.json with the SHA-256 of every input, the iteration count and the
per-iteration image sums and zero/subnormal counts the binary printed.  Small
cases commit their CSR4 file; the standard small workload ("plain-small",
2.6M elements) commits only the hashes of its regenerated inputs and the
golden image, and the tests regenerate the inputs with the committed
generator and check the hashes first.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mlem_b200 import formats, synth  # noqa: E402

SEQ = os.path.join(ROOT, "oracle", "_ref", "seqcsr4mlem")


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def run_seq(matrix_path, sino_path, iters):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "image.out")
        p = subprocess.run([SEQ, matrix_path, sino_path, out, str(iters)], cwd=td,
                           capture_output=True, text=True, check=True)
        img = np.fromfile(out, dtype=np.float32)
    sums = re.findall(r"image sum: (\S+),", p.stdout)
    zeros = [int(z) for z in re.findall(r"Zeros: (\d+)", p.stdout)]
    subn = [int(z) for z in re.findall(r"subnormals: (\d+)", p.stdout)]
    init = re.findall(r"INIT: (.*)", p.stdout)
    return img, {"image_sums_printed": sums, "zeros": zeros, "subnormals": subn,
                 "init_line": init[0] if init else ""}


def edge_matrix():
    """Hand-made matrix with the edge cases the hot path must survive:
    empty rows (first, middle, last), a long row, duplicate columns inside a
    row, a column no row touches (norm == 0), rows whose counts are zero, and
    odd element offsets for every row start."""
    rng = np.random.default_rng(1234)
    R, C = 301, 64
    rows = []
    for r in range(R):
        if r in (0, 1, 2, 150, 300):
            rows.append([])
        elif r == 10:
            cols = np.concatenate([np.arange(C - 1), np.arange(0, C - 1, 3)])  # duplicates
            rows.append(list(cols))
        else:
            n = int(rng.integers(1, 12))
            rows.append(list(rng.integers(0, C - 1, size=n)))  # column C-1 never used
    counts = np.array([len(x) for x in rows], np.uint64)
    row_end = np.cumsum(counts, dtype=np.uint64)
    elems = np.zeros(int(row_end[-1]), formats.ELEM_DTYPE)
    elems["index"] = np.concatenate([np.array(x, np.uint32) for x in rows if x])
    elems["value"] = rng.uniform(0.05, 1.75, size=elems.size).astype(np.float32)
    sino = rng.poisson(20.0, size=R).astype(np.int32)
    sino[5:15] = 0
    return formats.Csr4(R, C, row_end, elems, 0, (4, 4, 4)), sino


def main():
    if not os.path.exists(SEQ):
        sys.exit("oracle/_ref/seqcsr4mlem is missing: run `make -C oracle` first")
    manifest = {"generator": "mlem_b200/gen/siddon_core.h + mlem_b200/synth.py",
                "reference_binary": "mlem_seq/seqcsr4mlem.cpp built by oracle/Makefile",
                "cases": {}}

    # 1. tiny Siddon case, committed in full, 10 and 100 iterations.
    g = synth.Geometry(8, 8, 4, 512, 1, 1000, seed=11)
    m = synth.host_matrix(g)
    x = synth.phantom(8, 8, 4, 3, 11)
    sino = synth.poisson_sinogram(synth.project_f64(m, x), 1e5, 12)
    mp, sp = os.path.join(HERE, "tiny.csr4"), os.path.join(HERE, "tiny.sino")
    formats.write_csr4(mp, m.n_rows, m.n_cols, m.row_end, m.elems, grid=(8, 8, 4))
    formats.write_vector(sp, sino, np.int32)
    for iters in (10, 100):
        img, info = run_seq(mp, sp, iters)
        name = f"tiny_it{iters}"
        formats.write_vector(os.path.join(HERE, name + ".image"), img, np.float32)
        manifest["cases"][name] = dict(matrix="tiny.csr4", sino="tiny.sino",
                                       matrix_sha256=sha256(mp), sino_sha256=sha256(sp),
                                       iterations=iters, image=name + ".image", **info)

    # 2. hand-made edge cases, committed in full.
    m, sino = edge_matrix()
    mp, sp = os.path.join(HERE, "edge.csr4"), os.path.join(HERE, "edge.sino")
    formats.write_csr4(mp, m.n_rows, m.n_cols, m.row_end, m.elems, grid=(4, 4, 4))
    formats.write_vector(sp, sino, np.int32)
    img, info = run_seq(mp, sp, 7)
    formats.write_vector(os.path.join(HERE, "edge_it7.image"), img, np.float32)
    manifest["cases"]["edge_it7"] = dict(matrix="edge.csr4", sino="edge.sino",
                                         matrix_sha256=sha256(mp), sino_sha256=sha256(sp),
                                         iterations=7, image="edge_it7.image", **info)

    # 3. the standard small workload (plain-small), inputs regenerated by the tests.
    w = synth.WORKLOADS["plain-small"]
    m, frames = synth.host_workload(w)
    with tempfile.TemporaryDirectory() as td:
        mp, sp = os.path.join(td, "m.csr4"), os.path.join(td, "s.sino")
        gg = w.geometry
        formats.write_csr4(mp, m.n_rows, m.n_cols, m.row_end, m.elems, grid=(gg.nx, gg.ny, gg.nz))
        formats.write_vector(sp, frames.sinograms[0], np.int32)
        img, info = run_seq(mp, sp, w.iterations)
        manifest["cases"]["plain_small_it10"] = dict(
            workload="plain-small", matrix=None, sino=None, matrix_sha256=sha256(mp),
            sino_sha256=sha256(sp), nnz=int(m.nnz), iterations=w.iterations,
            image="plain_small_it10.image", **info)
    formats.write_vector(os.path.join(HERE, "plain_small_it10.image"), img, np.float32)

    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(json.dumps({k: {kk: v[kk] for kk in ("iterations", "matrix_sha256")}
                      for k, v in manifest["cases"].items()}, indent=1))


if __name__ == "__main__":
    main()
