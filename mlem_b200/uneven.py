"""Uneven batched MLEM across geometries, on one GPU.

Three seeded Siddon matrices of very different size (32x32x16 voxels with
65,536 LORs; 128x128x64 with 4,194,304 LORs; 256x256x96 with 16,777,216 LORs
at about 300 elements per row, ~5e9 elements, ~40 GB), with 12, 8 and 4
sinograms, reconstructed together by one `mlem_batch`: one persistent kernel
per iteration over work items cut from all three matrices.  The matrices are
generated on the device without the CSC copy (the batch needs only the CSR).

Printed (one JSON line): the batch's ms per iteration, the same three
reconstructions run one context after another (each with its fastest
one-pass tuning), reconstructions x iterations per second, algorithmic HBM
bytes per iteration and the relative L2 difference between the batch's
images and the separate runs after the same iterations (the batch is the
same arithmetic in another scatter order, so this stays far below 1e-4).

    python -m mlem_b200.uneven [--iters 60] [--warmup 3] [--scale 1.0]

--scale < 1 shrinks every LOR count (a quick run on a smaller device).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

MEMBERS = ("uneven-small", "uneven-full", "uneven-large")


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))


def _time_ms(stream, fn, reps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn(reps)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _best_solo(ctx, stream, api):
    """Fastest one-pass (MLEM_BK_FUSED) tuning of one context on its own, over
    the same choices the batch has (frame tile, row visiting order) plus the
    lanes per row and resident blocks of the single-matrix kernel."""
    saved = ctx.get_images()
    padded = next(p for p in (1, 2, 4, 8, 16, 32, 48, 64) if ctx.n_frames <= p)
    best = None
    for tile in (1, 2, 4, 8, 16):
        if padded % tile:
            continue
        for group in (16, 32):
            for bps in (4, 8):
                for visit in (api.VISIT_FILE, api.VISIT_SORTED, api.VISIT_SORTED_CHUNKED,
                              api.VISIT_SORTED_STAGED):
                    if visit in (api.VISIT_SORTED_CHUNKED, api.VISIT_SORTED_STAGED) and group != 32:
                        continue
                    ctx.set_tuning(bk_mode=api.BK_FUSED, group=group, frame_tile=tile,
                                   blocks_per_sm=bps, visit=visit)
                    ctx.iterate(1, stats=False)
                    ms = _time_ms(stream, lambda k: ctx.iterate(k, stats=False), 2)
                    if best is None or ms < best[0]:
                        best = (ms, dict(group=group, frame_tile=tile, blocks_per_sm=bps,
                                         visit=visit))
    ctx.set_tuning(bk_mode=api.BK_FUSED, **best[1])
    ctx.set_images(saved)
    return best[1]


def run(iters=60, warmup=3, scale=1.0, device=0):
    import torch

    from . import api, synth

    torch.cuda.set_device(device)
    stream = torch.cuda.current_stream()
    members = []
    t0 = time.time()
    for name in MEMBERS:
        w = synth.WORKLOADS[name]
        g = w.geometry
        if scale != 1.0:
            g = synth.Geometry(g.nx, g.ny, g.nz, max(1024, int(g.n_rows * scale)), g.min_count,
                               g.max_count, seed=g.seed)
        ctx = api.Context.siddon(g, flags=api.FLAG_NO_CSC, device=device)
        ctx.set_stream(stream.cuda_stream)
        fr = synth.make_frames(w, ctx.project_f64)
        ctx.set_sinograms(fr.sinograms)
        ctx.init_images()
        members.append((name, g, ctx))
    setup_s = time.time() - t0

    ctxs = [c for _, _, c in members]
    start = [c.get_images() for c in ctxs]

    # --- the batch ----------------------------------------------------------
    batch = api.Batch(ctxs)
    t1 = time.time()
    sched = batch.autotune()
    tune_s = time.time() - t1
    batch.iterate(warmup, stats=False)
    for c, x in zip(ctxs, start):
        c.set_images(x)
    batch_ms = _time_ms(stream, lambda k: batch.iterate(k, stats=False), iters)
    ph_ms, ph_bytes, ph_launch = batch.profile(10)
    for c, x in zip(ctxs, start):
        c.set_images(x)
    batch.iterate(iters, stats=False)
    batch_imgs = [c.get_images() for c in ctxs]
    batch.close()

    # --- the same reconstructions, one context after another ----------------
    solo = []
    solo_ms = 0.0
    diffs = []
    for (name, g, c), x, bimg in zip(members, start, batch_imgs):
        c.set_images(x)
        t = _best_solo(c, stream, api)
        c.iterate(warmup, stats=False)
        c.set_images(x)
        ms = _time_ms(stream, lambda k: c.iterate(k, stats=False), iters)
        c.set_images(x)
        c.iterate(iters, stats=False)
        simg = c.get_images()
        d = max(_rel_l2(bimg[f], simg[f]) for f in range(c.n_frames))
        diffs.append(d)
        solo_ms += ms
        solo.append({"workload": name, "grid": [g.nx, g.ny, g.nz], "n_rows": c.n_rows,
                     "nnz": int(c.nnz), "frames": c.n_frames, "ms_per_iteration": round(ms, 4),
                     "tuning": t, "rel_l2_batch_vs_solo": d})

    recon = sum(c.n_frames for c in ctxs)
    total_bytes = float(ph_bytes.sum())
    out = {
        "workload": "uneven-3geom", "reconstructions": recon, "iterations": iters,
        "batch_ms_per_iteration": round(batch_ms, 4),
        "separate_ms_per_iteration": round(solo_ms, 4),
        "speedup_vs_separate": round(solo_ms / batch_ms, 3),
        "reconstruction_iterations_per_s": round(recon * 1e3 / batch_ms, 2),
        "hbm_gbs": round(total_bytes / (batch_ms / 1e3) / 1e9, 1),
        "bytes_per_iteration": total_bytes,
        "phases_ms": [round(float(x), 4) for x in ph_ms],
        "phase_launches": [int(x) for x in ph_launch],
        "schedule": sched, "max_rel_l2_batch_vs_separate": max(diffs),
        "members": solo, "setup_s": round(setup_s, 1), "autotune_s": round(tune_s, 1),
        "scale": scale,
    }
    for c in ctxs:
        c.close()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--iters", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    print(json.dumps(run(a.iters, a.warmup, a.scale, a.device)), flush=True)


if __name__ == "__main__":
    main()
