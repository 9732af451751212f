"""Run a synthetic MLEM workload for a few iterations with a fixed kernel
configuration -- the command the committed ncu summaries were captured with.

    python -m mlem_b200.profile_case --grid 128 128 64 --rows 1048576 \\
        --count 150 250 --mode fused --frames 1 --iters 3

Prints one JSON line with the per-phase device times of the last iteration.
"""
from __future__ import annotations

import argparse
import json

from . import api, synth


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[128, 128, 64])
    ap.add_argument("--rows", type=int, default=1 << 20)
    ap.add_argument("--count", type=int, nargs=2, default=[150, 250])
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--mode", choices=["csc", "atomic", "fused", "region", "exact", "matrix-free",
                                       "adjoint"],
                    default="csc")
    ap.add_argument("--group", type=int, default=32)
    ap.add_argument("--frame-tile", type=int, default=1)
    ap.add_argument("--blocks-per-sm", type=int, default=8)
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--natural", action="store_true", help="keep the natural voxel order")
    ap.add_argument("--visit", choices=["file", "sorted", "chunked", "staged"], default="file",
                    help="row visiting order (chunked: sorted, CTAs take chunks of rows; "
                         "staged: chunked with each warp's rows pipelined through shared memory)")
    a = ap.parse_args(argv)
    nx, ny, nz = a.grid
    g = synth.Geometry(nx, ny, nz, a.rows, a.count[0], a.count[1], seed=a.seed)
    if a.mode == "matrix-free":
        return matrix_free(a, g)
    if a.mode == "adjoint":
        return adjoint(a, g)
    flags = api.FLAG_EXACT if a.mode == "exact" else 0
    if a.natural:
        flags |= api.FLAG_NATURAL_LAYOUT
    with api.Context.siddon(g, flags=flags) as ctx:
        w = synth.Workload("profile", g, a.frames, a.iters, 0, (3, 12), (1e6, 1e9), 9000)
        fr = synth.make_frames(w, ctx.project_f64)
        ctx.set_sinograms(fr.sinograms)
        if a.mode != "exact":
            mode = {"csc": api.BK_CSC, "atomic": api.BK_ATOMIC, "fused": api.BK_FUSED,
                    "region": api.BK_REGION}[a.mode]
            visit = {"file": api.VISIT_FILE, "sorted": api.VISIT_SORTED,
                     "chunked": api.VISIT_SORTED_CHUNKED, "staged": api.VISIT_SORTED_STAGED}[a.visit]
            ctx.set_tuning(bk_mode=mode, group=a.group, frame_tile=a.frame_tile,
                           blocks_per_sm=a.blocks_per_sm, visit=visit)
        ctx.init_images()
        ms, by, ln = ctx.profile_phases(a.iters)
        print(json.dumps({"nnz": int(ctx.nnz), "mode": a.mode, "frames": a.frames,
                          "layout": "natural" if a.natural else "brick",
                          "visit": a.visit, "group": a.group,
                          "frame_tile": a.frame_tile, "blocks_per_sm": a.blocks_per_sm,
                          "phase_ms": [round(float(x), 4) for x in ms],
                          "phase_GBps": [round(float(b / (t / 1e3) / 1e9), 1) if t > 0 else 0
                                         for b, t in zip(by, ms)]}))




def matrix_free(a, g):
    """The matrix-free pass (mlem_mf_*) on the same geometry and frames: the
    sinogram comes from a stored context's double projection, which is then
    freed; one frame."""
    import time

    with api.Context.siddon(g, flags=api.FLAG_NO_CSC) as ctx:
        w = synth.Workload("profile", g, 1, a.iters, 0, (3, 12), (1e6, 1e9), 9000)
        fr = synth.make_frames(w, ctx.project_f64)
    with api.MatrixFree(g) as mf:
        mf.set_sinogram(fr.sinograms[0])
        mf.init_image()
        t0 = time.time()
        mf.iterate(a.iters)
        mf.get_image()
        print(json.dumps({"mode": "matrix-free", "rays": g.n_rows, "iters": a.iters,
                          "wall_s": round(time.time() - t0, 3), **mf.info()}))


def adjoint(a, g):
    """The two one-pass kernels of the unrolled MLEM's backward pass
    (mlem_ratio_rows_d, then mlem_adjoint_update_d) on the same geometry's
    first frame, a.iters times each, with CUDA-event times."""
    import torch

    with api.Context.siddon(g, flags=api.FLAG_NO_CSC) as ctx:
        w = synth.Workload("profile", g, 1, a.iters, 0, (3, 12), (1e6, 1e9), 9000)
        fr = synth.make_frames(w, ctx.project_f64)
        dev = torch.device("cuda", 0)
        sino = torch.from_numpy(fr.sinograms[0].astype("int32")).to(dev)
        x = torch.full((ctx.n_cols,), 1.0, device=dev)
        du = torch.rand(ctx.n_cols, device=dev, generator=torch.Generator(dev).manual_seed(1))
        rows = torch.empty(ctx.n_rows, device=dev)
        u = torch.empty(ctx.n_cols, device=dev)
        out = torch.empty(ctx.n_cols, device=dev)
        st = torch.cuda.current_stream().cuda_stream
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ms = [0.0, 0.0]
        for _ in range(a.iters):
            ev[0].record()
            ctx.ratio_rows_d(x.data_ptr(), sino.data_ptr(), rows.data_ptr(), u.data_ptr(), st)
            ev[1].record()
            ctx.adjoint_update_d(du.data_ptr(), sino.data_ptr(), rows.data_ptr(), out.data_ptr(), st)
            ev[2].record()
            torch.cuda.synchronize()
            ms[0] = ev[0].elapsed_time(ev[1])
            ms[1] = ev[1].elapsed_time(ev[2])
        print(json.dumps({"mode": "adjoint", "nnz": int(ctx.nnz), "rows": g.n_rows,
                          "ratio_rows_ms": round(ms[0], 4), "adjoint_update_ms": round(ms[1], 4)}))


if __name__ == "__main__":
    main()
