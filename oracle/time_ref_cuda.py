"""TEST INFRASTRUCTURE: the reference's own CUDA kernels (oracle/_ref/libref_cuda.so)
against this library's iteration, on the same GPU and the same plain-full matrix.

    python oracle/time_ref_cuda.py [--iters 6]

Prints one JSON line: per-kernel device ms per iteration of the reference's
version_4 and version_6 iterations (oracle/ref_cuda/harness.cu), this
library's autotuned iteration, and the relative L2 distance of the images
after the same iterations.
"""
import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=6)
    a = ap.parse_args()
    import numpy as np
    import torch

    import oracle_bind as ob
    from mlem_b200 import api, formats, synth

    torch.cuda.set_device(0)
    w = synth.WORKLOADS["plain-full"]
    out = {"workload": "plain-full", "iterations": a.iters}
    with api.Context.siddon(w.geometry) as ctx:
        sino = synth.make_frames(w, ctx.project_f64).sinograms[0]
        re_, el = ctx.csr()  # natural voxel order, file row order: the CSR4 file's arrays
        m = formats.Csr4(ctx.n_rows, ctx.n_cols, re_, el)
        imgs = {}
        for v in (4, 6):
            img, ms = ob.ref_cuda_mlem(m, sino, a.iters, v)
            imgs[v] = img
            out[f"reference_version_{v}_ms"] = {k: round(float(t), 4) for k, t in zip(
                ("clear", "fwproj", "correl", "bkproj", "update", "iteration"), ms)}
        del m, re_, el
        ctx.set_sinograms(sino)
        ctx.init_images()
        t = ctx.autotune()
        ctx.init_images()
        ctx.iterate(1, stats=False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s = torch.cuda.current_stream()
        ctx.set_stream(s.cuda_stream)
        ctx.init_images()
        e0.record(s)
        ctx.iterate(a.iters, stats=False)
        e1.record(s)
        torch.cuda.synchronize()
        ours = e0.elapsed_time(e1) / a.iters
        mine = ctx.get_images()[0]
        out["ours_ms_per_iteration"] = round(ours, 4)
        out["ours_method"] = api.BK_NAMES[t["bk_mode"]] + "/" + api.VISIT_NAMES[t["visit"]]
        for v in (4, 6):
            out[f"speedup_vs_version_{v}"] = round(out[f"reference_version_{v}_ms"]["iteration"] / ours, 2)
            out[f"rel_l2_ours_vs_version_{v}"] = ob.rel_l2(mine, imgs[v])
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
