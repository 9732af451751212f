#!/usr/bin/env python3
"""MLEM benchmark: iterations/s and HBM GB/s on the plain-full workload.

Workload ("plain-full"): a synthetic Siddon system matrix of 4,194,304 LORs
x 1,048,576 voxels (128x128x64 grid, 150-250 elements per row, ~0.78e9
elements, 6.2 GB CSR4 plus a 6.2 GB device CSC copy), one int32 Poisson
sinogram of an 8-ellipsoid phantom at 1e9 counts, float32.  A step is one
MLEM iteration (forward projection + correlation + back projection + update,
plus the per-iteration image-sum census the reference prints).  The matrix
(6.2 GB) is larger than the 126 MB L2, so no L2 flush is needed between
steps.  The batched line ("batched-b16") runs 16 sinograms over the same
matrix in one pass per iteration; the "uneven" line batches three matrices
of different geometry (12, 8 and 4 sinograms) in one kernel per iteration
(mlem_b200.uneven); the "mirrored" line reconstructs the plain-full matrix
read as a symmetry-compressed file (three mirrors, a 50 GB full matrix) once
expanded on the device and once with the mirrors applied in the kernels
(mlem_b200.mirrored).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  --impl reference times the reference's own
OpenMP implementation (openmpcsr4mlem, compiled from its sources into
oracle/_ref) on this host's cores on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLEM iterations/s and HBM GB/s, plain vs batched B=16, at rel L2 err <=1e-4"
UNIT = "iterations/s"
REF_MESSUNG = os.path.join(ROOT, "oracle", "_ref", "openmpcsr4mlem_messung")
PHASES = ("project", "backproject", "update", "stats")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["auto", "csc", "atomic", "fused", "region"], default="auto",
                    help="back-projection method; auto = autotuned")
    ap.add_argument("--visit", choices=["file", "sorted", "chunked", "staged"], default="file",
                    help="row visit with a fixed --mode (32 lanes per row, one-frame tile)")
    ap.add_argument("--blocks-per-sm", type=int, default=8,
                    help="resident blocks (chunked/staged: CTAs) per SM with a fixed --mode")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-osem", action="store_true")
    ap.add_argument("--no-skewed", action="store_true")
    ap.add_argument("--no-differentiable", action="store_true")
    ap.add_argument("--no-uneven", action="store_true",
                    help="skip the uneven three-geometry batch (one GPU only)")
    ap.add_argument("--no-mirrored", action="store_true",
                    help="skip the symmetry-compressed matrix, expanded vs mirrored kernels (one GPU only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=3)
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(
            ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
             "-lms", "100", "-i", str(self.gpu)],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[6:10]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def two_pass_bytes(nnz, rows, cols):
    """Algorithmic bytes of one plain iteration as two passes over the matrix:
    CSR (8R offsets + 8Z + 4C image + 4R sinogram + 4R correlation) and CSC
    (8C offsets + 8Z + 4R correlation + 4C norm + 8C image read and write)."""
    return float(16 * int(nnz) + 20 * int(rows) + 24 * int(cols))


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of the dominant kernels from the committed ncu
    summary (profiles/traffic.json), keyed by kernel name; {} if absent."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's openmpcsr4mlem on this host
# ---------------------------------------------------------------------------
def write_inputs(tmpdir, row_end, elems, n_rows, n_cols, grid, sino):
    from mlem_b200 import formats
    mp = os.path.join(tmpdir, "matrix.csr4")
    sp = os.path.join(tmpdir, "sino.bin")
    formats.write_csr4(mp, n_rows, n_cols, row_end, elems, grid=grid)
    formats.write_vector(sp, sino, "int32")
    return mp, sp


def scratch_dir(need_bytes):
    for d in ("/dev/shm", tempfile.gettempdir()):
        try:
            if shutil.disk_usage(d).free > need_bytes * 1.2:
                return tempfile.mkdtemp(prefix="mlem_bench_", dir=d)
        except OSError:
            continue
    return None


def run_reference_binary(matrix_path, sino_path, iters, threads, timeout=900):
    """Per-iteration seconds printed by openmpcsr4mlem -DMESSUNG (iter,elapsed)."""
    out = os.path.join(os.path.dirname(matrix_path), "image.out")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.time()
    p = subprocess.run([REF_MESSUNG, matrix_path, sino_path, out, str(iters)], env=env,
                       capture_output=True, text=True, timeout=timeout,
                       cwd=os.path.dirname(matrix_path))
    if p.returncode != 0:
        raise RuntimeError(f"openmpcsr4mlem failed: {p.stderr[-500:]}")
    secs = [float(m.group(2)) for m in re.finditer(r"^(\d+),([0-9.eE+-]+)$", p.stdout, re.M)]
    return secs, time.time() - t0


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def run_ours(a, rank, world, local_rank):
    import numpy as np
    import torch

    from mlem_b200 import api, synth

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    w = synth.WORKLOADS["plain-full"]
    g = w.geometry
    if world > 1:  # weak scaling: every rank reconstructs its own full-size LOR set
        g = synth.Geometry(g.nx, g.ny, g.nz, g.n_rows, g.min_count, g.max_count, seed=g.seed + 100 * rank)
    t_setup = time.time()
    ctx = api.Context.siddon(g, device=local_rank)
    t_matrix = time.time() - t_setup
    frames = synth.make_frames(w, ctx.project_f64)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.set_sinograms(frames.sinograms)
    ctx._refresh()  # rows_with_counts of this sinogram
    ctx.init_images()

    mode_map = {"csc": api.BK_CSC, "atomic": api.BK_ATOMIC, "fused": api.BK_FUSED,
                "region": api.BK_REGION}
    if a.mode == "auto":
        tuning = ctx.autotune()
    else:
        visit = {"file": api.VISIT_FILE, "sorted": api.VISIT_SORTED,
                 "chunked": api.VISIT_SORTED_CHUNKED, "staged": api.VISIT_SORTED_STAGED}[a.visit]
        ctx.set_tuning(bk_mode=mode_map[a.mode], group=32, frame_tile=1,
                       blocks_per_sm=a.blocks_per_sm, visit=visit)
        tuning = ctx.tuning()
    ctx.init_images()
    ctx.iterate(a.warmup, stats=False)
    kernels_per_iter = ctx.kernels_per_iteration()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # --- timed region: K iterations, device events on the context's stream ---
    clocks = ClockSampler(local_rank) if rank == 0 else None
    barrier()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.iterate(a.steps, stats=False)
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1)
    # per-phase events (a second pass, same kernels)
    ph_ms, ph_bytes, ph_launch = ctx.profile_phases(max(10, min(a.steps, 50)))
    clk = clocks.stop() if clocks else None
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / a.steps
    value = world * a.steps / (ms / 1e3)

    # parity of this run's image against the FP64 projection of its phantom is
    # covered by the tests; report the image sum as a sanity figure
    img = ctx.get_images()[0]
    image_sum = float(img.astype(np.float64).sum())

    # --- end to end through the C ABI: pinned host sinogram + image in, image out ---
    sino_h = torch.from_numpy(frames.sinograms[0].copy()).pin_memory()
    img_h = torch.from_numpy(img.copy()).pin_memory()
    k_e2e = max(5, min(a.steps, 50))
    ctx.step_host_ptr(sino_h.data_ptr(), img_h.data_ptr(), 1)  # warm (captures the 1-step graph)
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(k_e2e):
        ctx.step_host_ptr(sino_h.data_ptr(), img_h.data_ptr(), 1)
    f1.record(stream)
    barrier()
    e2e_ms = f0.elapsed_time(f1) / k_e2e
    e2e = {"value": world * 1e3 / e2e_ms, "unit": UNIT,
           "h2d_bytes_per_step": int(4 * ctx.n_rows + 4 * ctx.n_cols),
           "d2h_bytes_per_step": int(4 * ctx.n_cols),
           "call": "mlem_step_host (pinned host sinogram + image)"}

    peak, peak_kind = measured_peak()
    total_bytes = float(ph_bytes.sum())
    dom = int(ph_ms[:3].argmax())
    kernel_names = {
        api.BK_CSC: ("k_fwproj", "k_bkproj_csc", "-", "k_stats"),
        api.BK_ATOMIC: ("k_fwproj", "k_bkproj_scatter", "k_apply_update", "k_stats"),
        api.BK_FUSED: ({api.VISIT_SORTED_CHUNKED: "k_fused_chunked",
                        api.VISIT_SORTED_STAGED: "k_fused_staged"}.get(tuning["visit"], "k_fused_row"),
                       "-", "k_apply_update", "k_stats"),
        api.BK_REGION: ("k_rb_fwproj", "k_rb_bkproj", "-", "k_stats"),  # bkproj applies the update
    }[tuning["bk_mode"]]
    traffic = committed_traffic().get(kernel_names[dom])
    achieved = ph_bytes[dom] / (ph_ms[dom] / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": kernel_names[dom], "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": ph_bytes[dom] / max(1, ph_launch[dom]),
                "ms_per_launch": ph_ms[dom] / max(1, ph_launch[dom])}
    phases = {PHASES[p]: {"ms": round(float(ph_ms[p]), 4), "GB": round(ph_bytes[p] / 1e9, 4),
                          "GB/s": round(ph_bytes[p] / (ph_ms[p] / 1e3) / 1e9, 1) if ph_ms[p] > 0 else None,
                          "kernel": kernel_names[p], "launches": int(ph_launch[p])}
              for p in range(4)}

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Siddon matrix, ellipsoid phantom, Poisson sinogram)",
        "config": {"workload": "plain-full", "grid": [g.nx, g.ny, g.nz], "n_rows": ctx.n_rows,
                   "n_cols": ctx.n_cols, "nnz": int(ctx.nnz), "frames": 1,
                   "bk_mode": api.BK_NAMES[tuning["bk_mode"]], "group": tuning["group"],
                   "frame_tile": tuning["frame_tile"], "blocks_per_sm": tuning["blocks_per_sm"],
                   "row_visit": api.VISIT_NAMES[tuning["visit"]],
                   "l2": "inputs larger than L2 (6.2 GB matrix), no flush",
                   # rows whose counts are zero add nothing to the update; the sorted
                   # one-pass walks leave them out (the roofline counts the rest)
                   "rows_with_counts": int(ctx.info.rows_with_counts),
                   "nnz_with_counts": int(ctx.info.nnz_with_counts),
                   "parallelism": "replicas" if world > 1 else "single"},
        "hbm_gbs": round(total_bytes / (ms_per_step / 1e3) / 1e9, 1),
        # the same iteration against the two-pass byte count of the reference's
        # algorithm (CSR pass for calcFwProj + CSC pass for calcBkProj):
        # 16 Z + 20 R + 24 C bytes over every row, which the one-pass kernel does
        # not move (one pass, and only the rows with counts)
        "two_pass_formula": {
            "bytes_per_iteration": two_pass_bytes(ctx.nnz, ctx.n_rows, ctx.n_cols),
            "achieved_gbs": round(two_pass_bytes(ctx.nnz, ctx.n_rows, ctx.n_cols)
                                  / (ms_per_step / 1e3) / 1e9, 1),
            "frac": round(two_pass_bytes(ctx.nnz, ctx.n_rows, ctx.n_cols)
                          / (ms_per_step / 1e3) / 1e9 / peak, 4)},
        "iteration_roofline_frac": round(total_bytes / (ms_per_step / 1e3) / 1e9 / peak, 4),
        "bytes_per_iteration": total_bytes,
        "roofline": roofline, "phases": phases, "e2e": e2e,
        "gpu_launches": int(kernels_per_iter * a.steps),
        "clocks": clk, "image_sum": image_sum, "setup_s": {"matrix": round(t_matrix, 2)},
    }

    # --- batched: 16 sinograms in one pass over the matrix per iteration ---
    if not a.no_batched:
        wb = synth.WORKLOADS["batched-b16"]
        fb = synth.make_frames(wb, ctx.project_f64)
        ctx.set_sinograms(fb.sinograms)
        ctx.init_images()
        tb = ctx.autotune()
        ctx.init_images()
        ctx.iterate(a.warmup, stats=False)
        kb = max(10, a.steps // 4)
        barrier()
        e0.record(stream)
        ctx.iterate(kb, stats=False)
        e1.record(stream)
        barrier()
        bms = e0.elapsed_time(e1) / kb
        bph_ms, bph_bytes, _ = ctx.profile_phases(10)
        line["batched"] = {
            "workload": "batched-b16", "frames": 16, "ms_per_iteration": round(bms, 4),
            "frame_iterations_per_s": round(16 * 1e3 / bms, 2),
            "per_frame_speedup_vs_plain": round((16 / bms) / (1 / ms_per_step), 3),
            "hbm_gbs": round(float(bph_bytes.sum()) / (bms / 1e3) / 1e9, 1),
            "bk_mode": api.BK_NAMES[tb["bk_mode"]], "group": tb["group"],
            "frame_tile": tb["frame_tile"], "row_visit": api.VISIT_NAMES[tb["visit"]],
            "phases_ms": [round(float(x), 4) for x in bph_ms],
            "parity": batched_parity(ctx, fb.sinograms, tb, 10),
        }

    # --- ordered subsets: 8 interleaved row subsets, the plain sinogram ---
    if not a.no_osem:
        n_sub = 8
        ctx.set_sinograms(frames.sinograms)
        ctx.init_images()
        ctx.set_subsets(n_sub)
        to = ctx.autotune()
        ctx.init_images()
        ctx.iterate(a.warmup, stats=False)
        ko = max(10, a.steps // 2)
        barrier()
        e0.record(stream)
        ctx.iterate(ko, stats=False)
        e1.record(stream)
        barrier()
        oms = e0.elapsed_time(e1) / ko
        line["osem"] = {
            "workload": "plain-full", "subsets": n_sub, "ms_per_iteration": round(oms, 4),
            "sub_iterations_per_s": round(n_sub * 1e3 / oms, 2),
            "iteration_time_vs_plain": round(oms / ms_per_step, 3),
            "frame_tile": to["frame_tile"], "group": to["group"],
            "row_visit": api.VISIT_NAMES[to["visit"]],
            "gpu_launches_per_iteration": int(ctx.kernels_per_iteration()),
        }
        ctx.set_subsets(1)

    # --- differentiable MLEM: 10 unrolled iterations, gradient of an MSE loss ---
    if not a.no_differentiable:
        line["differentiable"] = differentiable_line(ctx, a, stream, barrier)

    # --- a skewed matrix: the long rows run as segments (k_long.cu) ---
    if not a.no_skewed:
        line["skewed"] = skewed_line(a, stream, barrier)

    # --- CPU baseline: the reference's openmpcsr4mlem on this host (rank 0, N=1) ---
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_from_ctx(ctx, frames.sinograms[0], g, a.cpu_iters)

    ctx.close()

    # --- uneven batch over three geometries (12 + 8 + 4 frames), one GPU ---
    if world == 1 and not a.no_uneven:
        from mlem_b200 import uneven
        torch.cuda.synchronize()
        line["uneven"] = uneven.run(iters=max(10, min(a.steps, 20)), warmup=3, device=local_rank)

    # --- a symmetry-compressed matrix: expanded on the device vs mirrors in the kernels ---
    if world == 1 and not a.no_mirrored:
        from mlem_b200 import mirrored
        torch.cuda.synchronize()
        line["mirrored"] = mirrored.run(iters=10, warmup=3, device=local_rank)

    if dist is not None:
        dist.destroy_process_group()
    return line


def differentiable_line(ctx, a, stream, barrier):
    """The plain-full matrix: K = 10 relaxed MLEM iterations from a uniform
    start through torch_ext.unrolled_mlem, loss = mean squared error of the
    last image against the phantom, gradients with respect to the start image
    and the per-iteration exponents.  One step = forward + backward (the
    backward recomputes each iteration's projections from the saved images;
    calcUpdate's numerator comes from the one-pass kernels)."""
    import numpy as np
    import torch

    from mlem_b200 import synth, torch_ext

    w = synth.WORKLOADS["differentiable"]
    fr = synth.make_frames(w, ctx.project_f64)
    dev = torch.device("cuda", torch.cuda.current_device())
    sino = torch.from_numpy(fr.sinograms[0]).to(dev)
    x_true = torch.from_numpy(fr.phantoms[0].astype(np.float32)).to(dev)
    norm = torch_ext.norm_tensor(ctx, dev)
    init = float(sino.double().sum() / norm.double().sum())
    K = 10

    def step():
        x0 = torch.full((ctx.n_cols,), init, dtype=torch.float32, device=dev, requires_grad=True)
        omega = torch.ones(K, dtype=torch.float32, device=dev, requires_grad=True)
        loss = torch.mean((torch_ext.unrolled_mlem(x0, omega, sino, ctx, norm) - x_true) ** 2)
        loss.backward()
        return loss, x0.grad, omega.grad

    for _ in range(max(1, a.warmup)):
        step()
    n = 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(n):
        loss, gx, gw = step()
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1) / n
    # passes over the matrix per iteration: forward 1 (one-pass ratio); backward 4
    # (recomputed A x and one-pass ratio, then A du and A^T df)
    return {"workload": "differentiable", "unrolled_iterations": K, "ms_per_gradient_step": round(ms, 3),
            "matrix_passes_per_step": 5 * K, "ms_per_matrix_pass": round(ms / (5 * K), 4),
            "loss": float(loss.item()), "grad_x0_norm": float(gx.norm().item()),
            "grad_omega": [round(float(v), 6) for v in gw.tolist()]}


def skewed_line(a, stream, barrier):
    """1,048,576 rows of 100-199 random elements plus 64 rows of 500,000 over
    1,048,576 voxels (1.9e8 elements, seeded): the one-pass iteration with
    the long rows cut into segments, autotuned, device-timed."""
    import numpy as np
    import torch

    from mlem_b200 import api, formats

    rng = np.random.default_rng(3)
    R = C = 1 << 20
    lens = rng.integers(100, 200, size=R)
    lens[rng.choice(R, 64, replace=False)] = 500_000
    row_end = np.cumsum(lens).astype(np.uint64)
    Z = int(row_end[-1])
    el = np.zeros(Z, api.ELEM_DTYPE)
    el["index"] = rng.integers(0, C, size=Z, dtype=np.uint32)
    el["value"] = rng.uniform(0.1, 1.7, Z).astype(np.float32)
    sino = rng.poisson(30, R).astype(np.int32)
    with api.Context.from_matrix(formats.Csr4(R, C, row_end, el), flags=api.FLAG_NO_CSC) as ctx:
        del el
        ctx.set_stream(stream.cuda_stream)
        ctx.set_sinograms(sino)
        ctx.init_images()
        t = ctx.autotune()
        ctx.init_images()
        ctx.iterate(a.warmup, stats=False)
        k = max(10, a.steps // 2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(stream)
        ctx.iterate(k, stats=False)
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1) / k
        return {"workload": "skewed", "n_rows": R, "n_cols": C, "nnz": Z,
                "long_rows": 64, "long_row_elements": 500_000, "ms_per_iteration": round(ms, 4),
                "elements_per_s": round(Z / (ms / 1e3), 1),
                "bk_mode": api.BK_NAMES[t["bk_mode"]], "row_visit": api.VISIT_NAMES[t["visit"]],
                "gpu_launches_per_iteration": int(ctx.kernels_per_iteration())}


def rel_l2(a, b):
    import numpy as np
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def batched_parity(ctx, sinograms, tuning, iters):
    """Every frame of a batched reconstruction against its own single-frame
    run (same tuning method and visit), after `iters` iterations."""
    from mlem_b200 import api

    ctx.set_sinograms(sinograms)
    ctx.init_images()
    ctx.iterate(iters, stats=False)
    batch = ctx.get_images()
    worst = 0.0
    for b in range(sinograms.shape[0]):
        ctx.set_sinograms(sinograms[b:b + 1])
        ctx.set_tuning(bk_mode=tuning["bk_mode"], group=tuning["group"], frame_tile=1,
                       blocks_per_sm=tuning["blocks_per_sm"], visit=tuning["visit"])
        ctx.init_images()
        ctx.iterate(iters, stats=False)
        worst = max(worst, rel_l2(batch[b], ctx.get_images()[0]))
    return {"iterations": iters, "max_rel_l2_frame_vs_single_run": worst, "tolerance": 1e-4,
            "single_run_visit": api.VISIT_NAMES[tuning["visit"]]}


def cpu_baseline_from_ctx(ctx, sino, g, iters):
    if not os.path.exists(REF_MESSUNG):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/openmpcsr4mlem_messung not built"}
    need = 8 * ctx.nnz + 8 * ctx.n_rows + 4 * ctx.n_rows
    d = scratch_dir(need)
    if d is None:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: no scratch space for the CSR4 file"}
    try:
        row_end, elems = ctx.csr()
        mp, sp = write_inputs(d, row_end, elems, ctx.n_rows, ctx.n_cols, (g.nx, g.ny, g.nz), sino)
        del row_end, elems
        threads = host_threads()
        secs, wall = run_reference_binary(mp, sp, iters, threads)
        per = statistics.mean(secs[1:]) if len(secs) > 1 else secs[0]
        # the reference's image after these iterations against ours from the same inputs
        import numpy as np

        from mlem_b200 import api
        ref_img = np.fromfile(os.path.join(d, "image.out"), dtype=np.float32)
        ctx.set_sinograms(sino)
        ctx.init_images()
        ctx.iterate(iters, stats=False)
        parity = {"iterations": iters, "rel_l2_vs_reference_image": rel_l2(ctx.get_images()[0], ref_img),
                  "tolerance": 1e-4, "method": api.BK_NAMES[ctx.tuning()["bk_mode"]]}
        return {"value": round(1.0 / per, 4), "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"{iters} full iterations of openmpcsr4mlem (reference source, -O3 -fopenmp "
                          f"-DMESSUNG) on the same plain-full CSR4 file; mean of iterations 2..{iters}; "
                          f"wall {wall:.1f} s incl. load and serial column sums",
                "iteration_seconds": secs, "parity": parity}
    finally:
        shutil.rmtree(d, ignore_errors=True)


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(a, rank, world):
    if rank != 0:
        return None
    import numpy as np

    from mlem_b200 import synth

    if not os.path.exists(REF_MESSUNG):
        return {"impl": "reference", "unavailable": "oracle/_ref/openmpcsr4mlem_messung is not built"}
    w = synth.WORKLOADS["plain-full"]
    g = w.geometry
    m = synth.host_matrix(g)  # host generator (CPU); bit-identical to the GPU arm's matrix
    frames = synth.make_frames(w, lambda x: synth.project_f64(m, x))
    need = 8 * m.nnz + 8 * m.n_rows
    d = scratch_dir(need)
    if d is None:
        return {"impl": "reference", "unavailable": "no scratch space for the 6 GB CSR4 file"}
    try:
        mp, sp = write_inputs(d, m.row_end, m.elems, m.n_rows, m.n_cols, (g.nx, g.ny, g.nz),
                              frames.sinograms[0])
        del m
        threads = host_threads()
        k = max(1, min(a.steps, 20))
        wu = max(3, min(a.warmup, 5))  # at least 3 warm-up iterations, at most 5 (bounded run)
        secs, wall = run_reference_binary(mp, sp, wu + k, threads)
        timed = secs[wu:]
        per = statistics.mean(timed)
        value = 1.0 / per
        return {
            "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": world, "steps": len(timed), "warmup": wu, "ms_per_step": round(per * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Siddon matrix, ellipsoid phantom, Poisson sinogram)",
            "config": {"workload": "plain-full", "grid": [g.nx, g.ny, g.nz], "n_rows": g.n_rows,
                       "n_cols": g.n_cols, "frames": 1},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads,
                             "kind": "reference",
                             "sample": f"{len(timed)} timed iterations (of the {a.steps} requested; "
                                       f"capped at 20 to bound the run) of openmpcsr4mlem after "
                                       f"{wu} warm-up iterations; wall {wall:.1f} s"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
    finally:
        shutil.rmtree(d, ignore_errors=True)


def main():
    a = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        line = run_reference(a, rank, world)
    else:
        line = run_ours(a, rank, world, local_rank)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
