"""A symmetry-compressed matrix reconstructed two ways on one GPU: expanded at
creation (MLEM_FLAG_EXPAND_SYMMETRY's path, the full matrix on the device,
the one-pass kernels) and with the mirrors applied in the kernels
(MLEM_FLAG_MIRROR_KERNELS, only the stored elements on the device).

The stored matrix is the seeded 128x128x64 Siddon matrix of the plain-full
workload (4,194,304 LORs, about 7.8e8 elements), read as the compressed file
of a 2,048-crystal scanner (1 layer, 32 blocks of 16, 4 rings: 2048^2 LORs)
with all three mirrors (header flags x, y, z): its full matrix holds eight
times the stored elements (about 6.2e9, 50 GB).  The sinogram is the
plain-full phantom projected through the full matrix in FP64, Poisson-drawn
at 1e9 counts.

Printed (one JSON line): ms per iteration and device bytes of each context,
and the relative L2 difference between their images after the same
iterations (the same arithmetic in another summation order).

    python -m mlem_b200.mirrored [--iters 10] [--warmup 3] [--rows N] [--no-expanded]

--rows takes the first N LORs' worth of a smaller seeded matrix instead (N a
square of a multiple of 512 crystals, e.g. 1048576 for 1,024 crystals);
--no-expanded runs the mirrored kernels only, with the sinogram projected
through them in float32 (a small case for a profiler).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

def scanner_for(rows: int) -> tuple:
    """(layers, blocks, block size, rings) of a scanner with rows = crystals^2
    LORs: 1 layer, 32 blocks of 16 crystals, crystals / 512 rings."""
    n = int(round(rows ** 0.5))
    if n * n != rows or n % 512:
        raise ValueError(f"{rows} LORs are not the square of a multiple of 512 crystals")
    return (1, 32, 16, n // 512)


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))


def _timed(ctx, iters, warmup):
    ctx.init_images()
    ctx.iterate(warmup, stats=False)
    ms, _, _ = ctx.profile_phases(iters)
    return float(np.sum(ms))


def run(iters: int = 10, warmup: int = 3, device: int = 0, rows: int = 4194304,
        expanded: bool = True) -> dict:
    import dataclasses

    import torch

    from mlem_b200 import api, formats, synth

    torch.cuda.set_device(device)
    g = dataclasses.replace(synth.GEOM_FULL, n_rows=rows)
    work = dataclasses.replace(synth.WORKLOADS["plain-full"], geometry=g)
    scanner = scanner_for(rows)
    t0 = time.time()
    with api.Context.siddon(g, flags=api.FLAG_NO_CSC | api.FLAG_NO_ROW_ORDER,
                            device=device) as src:
        row_end, elems = src.csr()
    m = formats.Csr4(g.n_rows, g.n_cols, row_end, elems, 7, (g.nx, g.ny, g.nz),
                     (1.0, 1.0, 1.0), scanner)
    out = {"workload": "mirrored-plain-full" if rows == 4194304 else f"mirrored-{rows}-lors",
           "scanner": list(scanner), "symmetry": "xyz", "stored_nnz": int(m.nnz),
           "iterations": iters}
    images = {}
    sino = None
    runs = [("mirrored", api.FLAG_MIRROR_KERNELS | api.FLAG_NO_CSC)]
    if expanded:
        runs.insert(0, ("expanded", api.FLAG_NO_CSC))
    for name, flags in runs:
        with api.Context.symmetric(m, flags=flags, device=device) as ctx:
            if sino is None:  # the full matrix's projection of the phantom (FP64 when expanded)
                project = ctx.project_f64 if name == "expanded" else (
                    lambda x: ctx.fwproj(np.asarray(x, np.float32)).astype(np.float64))
                sino = synth.make_frames(work, project).sinograms
            ctx.set_sinograms(sino)
            ctx.init_images()
            if name == "expanded":
                ctx.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                               visit=api.VISIT_SORTED_CHUNKED)
                tuning = ctx.tuning()
            else:
                tuning = ctx.autotune()
            ms = _timed(ctx, iters, warmup)
            ctx.init_images()
            ctx.iterate(iters, stats=False)
            images[name] = ctx.get_images()[0]
            ctx._refresh()
            out[name] = {"nnz_on_device": int(ctx.nnz), "device_bytes": int(ctx.info.device_bytes),
                         "ms_per_iteration": round(ms, 4),
                         "tuning": {k: tuning[k] for k in ("bk_mode", "frame_tile", "blocks_per_sm", "visit")}}
    if expanded:
        out["full_nnz"] = out["expanded"]["nnz_on_device"]
        out["rel_l2_mirrored_vs_expanded"] = _rel_l2(images["mirrored"], images["expanded"])
    out["setup_s"] = round(time.time() - t0, 1)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--rows", type=int, default=4194304)
    ap.add_argument("--no-expanded", action="store_true")
    a = ap.parse_args(argv)
    print(json.dumps(run(a.iters, a.warmup, rows=a.rows, expanded=not a.no_expanded)), flush=True)


if __name__ == "__main__":
    main()
