#!/usr/bin/env python3
"""MLEM benchmark: iterations/s and HBM GB/s on the plain-full workload.

Workload ("plain-full"): a synthetic Siddon system matrix of 4,194,304 LORs
x 1,048,576 voxels (128x128x64 grid, 150-250 elements per row, ~0.78e9
elements, 6.2 GB CSR4 plus a 6.2 GB device CSC copy), one int32 Poisson
sinogram of an 8-ellipsoid phantom at 1e9 counts, float32.  A step is one
MLEM iteration: forward projection + correlation + back projection + update,
plus the per-iteration image-sum / zero / subnormal census the reference
prints (seqcsr4mlem.cpp:172-185), whose sums are copied to the host.  The
matrix (6.2 GB) is larger than the 126 MB L2, so no L2 flush is needed
between steps.

Besides the headline line, at one GPU:
* batched: 16 sinograms over the same matrix in one pass per iteration;
* parity_full: the full-size images after 60 iterations (the workload's
  iteration count) against the reference's own seqcsr4mlem and against the
  FP64 oracle -- the autotuned one-pass path, the command-line drop-in with a
  checkpoint every 10 iterations (deterministic CSC method), and one frame of
  the 16-frame batch; every batched frame against its own single-frame run.
  The reference binary and the oracle run as background processes on the
  host cores while the GPU lines are measured;
* osem, differentiable, skewed, uneven (three matrices of different
  geometry batched), mirrored (a symmetry-compressed matrix), matrix_free
  (the rays traced in every pass instead of a stored matrix).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--parallelism single|shards|replicas]

With N > 1 (torchrun, one process per GPU) the default is --parallelism
shards: the rows are split into nnz-balanced blocks, one per rank, and each
iteration computes every block's partial update in one pass and all-reduces
the C floats once over NCCL (strong scaling: value = iterations/s of the one
reconstruction).  --parallelism replicas gives each rank its own full-size
LOR set instead (weak scaling, no data-path collective).

Prints ONE JSON line (rank 0).  --impl reference times the reference's own
OpenMP implementation (openmpcsr4mlem, compiled from its sources into
oracle/_ref) on this host's cores on the same workload; its inputs are made
by oracle/_bin/oracle_tool in a child process.
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
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
REF_MESSUNG = os.path.join(REF_DIR, "openmpcsr4mlem_messung")
REF_SEQ = os.path.join(REF_DIR, "seqcsr4mlem")
ORACLE_TOOL = os.path.join(ROOT, "oracle", "_bin", "oracle_tool")
CLI = os.path.join(ROOT, "mlem_b200", "bin", "mlem_b200")
PHASES = ("project", "backproject", "update", "stats")
TOL = 1e-4


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--parallelism", choices=["auto", "single", "shards", "replicas"],
                    default="auto", help="auto: single at N=1, shards at N>1")
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
    ap.add_argument("--no-matrix-free", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the host-core legs (openmpcsr4mlem timing and the full-size parity)")
    ap.add_argument("--no-parity-full", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=3)
    ap.add_argument("--parity-iters", type=int, default=60)
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


# ---------------------------------------------------------------------------
# shared helpers
# ---------------------------------------------------------------------------
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


def workload_config(g, nnz, parallelism="single", frames=1):
    """The workload's identity, the same in both arms (tuning lives elsewhere)."""
    return {"workload": "plain-full", "grid": f"{g.nx}x{g.ny}x{g.nz}", "n_rows": int(g.n_rows),
            "n_cols": int(g.n_cols), "nnz": int(nnz), "frames": frames,
            "iterations_per_step": 1,
            "l2": "inputs larger than L2 (6.2 GB matrix), no flush",
            "parallelism": parallelism}


def scratch_dir(need_bytes):
    for d in ("/dev/shm", tempfile.gettempdir()):
        try:
            if shutil.disk_usage(d).free > need_bytes * 1.2:
                return tempfile.mkdtemp(prefix="mlem_bench_", dir=d)
        except OSError:
            continue
    return None


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def rel_l2(a, b):
    import numpy as np
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def sig(x):
    return None if x is None else float(f"{x:.3g}")


def write_csr4_and_sinos(d, row_end, elems, n_rows, n_cols, grid, sinos: dict):
    """The CSR4 file and raw int32 sinograms of the run, for the reference's binaries."""
    from mlem_b200 import formats
    mp = os.path.join(d, "matrix.csr4")
    formats.write_csr4(mp, n_rows, n_cols, row_end, elems, grid=grid)
    paths = {}
    for name, s in sinos.items():
        paths[name] = os.path.join(d, f"{name}.sino")
        formats.write_vector(paths[name], s, "int32")
    return mp, paths


def run_reference_binary(matrix_path, sino_path, iters, threads, timeout=900):
    """Per-iteration seconds printed by openmpcsr4mlem -DMESSUNG (iter,elapsed)."""
    out = os.path.join(os.path.dirname(matrix_path), "image_omp.out")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.time()
    p = subprocess.run([REF_MESSUNG, matrix_path, sino_path, out, str(iters)], env=env,
                       capture_output=True, text=True, timeout=timeout,
                       cwd=os.path.dirname(matrix_path))
    if p.returncode != 0:
        raise RuntimeError(f"openmpcsr4mlem failed: {p.stderr[-500:]}")
    secs = [float(m.group(2)) for m in re.finditer(r"^(\d+),([0-9.eE+-]+)$", p.stdout, re.M)]
    return secs, time.time() - t0, out


# ---------------------------------------------------------------------------
# full-size parity: the reference's seqcsr4mlem and the FP64 oracle on the
# host cores, in the background while the GPU lines run
# ---------------------------------------------------------------------------
class ParityJobs:
    """For each named sinogram: seqcsr4mlem (single core, the reference's
    sequential float path) and oracle_tool f64-mlem (FP64 oracle, threads),
    both for `iters` iterations on the same CSR4 file."""

    def __init__(self, d, matrix, sinos: dict, iters, threads):
        self.d, self.iters = d, iters
        self.procs = {}
        self.t0 = time.time()
        self.error = None
        if not (os.path.exists(REF_SEQ) and os.path.exists(ORACLE_TOOL)):
            self.error = "oracle/_ref/seqcsr4mlem or oracle/_bin/oracle_tool is not built"
            return
        n = max(1, len(sinos))
        f64_threads = max(1, (threads - n) // n)
        self.f64_threads = f64_threads
        for name, sp in sinos.items():
            seq_out = os.path.join(d, f"{name}.seq.img")
            f64_out = os.path.join(d, f"{name}.f64.img")
            logs = [open(os.path.join(d, f"{name}.{k}.log"), "w") for k in ("seq", "f64")]
            ps = subprocess.Popen([REF_SEQ, matrix, sp, seq_out, str(iters)], cwd=d,
                                  stdout=logs[0], stderr=subprocess.STDOUT)
            pf = subprocess.Popen([ORACLE_TOOL, "f64-mlem", matrix, sp, str(iters),
                                   str(f64_threads), f64_out], cwd=d,
                                  stdout=logs[1], stderr=subprocess.STDOUT)
            self.procs[name] = (ps, pf, seq_out, f64_out, logs)

    def collect(self, timeout=1200):
        """{name: (seq image f32, f64 image f64)}; seconds until the last ended."""
        import numpy as np
        out = {}
        deadline = time.time() + timeout
        for name, (ps, pf, so, fo, logs) in self.procs.items():
            for p in (ps, pf):
                try:
                    p.wait(timeout=max(1.0, deadline - time.time()))
                except subprocess.TimeoutExpired:
                    p.kill()
                    p.wait()
            for f in logs:
                f.close()
            if ps.returncode != 0 or pf.returncode != 0:
                raise RuntimeError(f"{name}: seqcsr4mlem rc={ps.returncode}, "
                                   f"oracle_tool rc={pf.returncode}")
            out[name] = (np.fromfile(so, np.float32), np.fromfile(fo, np.float64))
        return out, time.time() - self.t0


def run_cli(d, matrix, sino, iters, chk):
    """The command-line drop-in, as the reference's drivers are called:
    matrix input output iterations checkpointing (default method: the
    deterministic CSC back projection).  Returns the image and whether the
    checkpoint pair was removed after the run, as mpicsr4mlem does, its wall
    time and its phases (MLEM_B200_TIMING: seconds since the matrix load
    began, at the end of each phase)."""
    import numpy as np
    out = os.path.join(d, "cli.img")
    t0 = time.time()
    p = subprocess.run([CLI, matrix, sino, out, str(iters), str(chk)], cwd=d,
                       capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, MLEM_B200_TIMING="1"))
    if p.returncode != 0:
        raise RuntimeError(f"mlem_b200 CLI failed: {p.stderr[-300:]}")
    wall = time.time() - t0
    clean = not (os.path.exists(os.path.join(d, "img.chkpt"))
                 or os.path.exists(os.path.join(d, "iter.chkpt")))
    phases = {m.group(1): round(float(m.group(2)), 3)
              for m in re.finditer(r"^phase,(\w+),([0-9.eE+-]+)$", p.stderr, re.M)}
    return np.fromfile(out, np.float32), clean, wall, phases


# ---------------------------------------------------------------------------
# our implementation, one context per GPU (single, or weak-scaling replicas)
# ---------------------------------------------------------------------------
def run_ours(a, rank, world, local_rank, parallelism):
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
    if world > 1:  # replicas: every rank reconstructs its own full-size LOR set
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
    ctx.iterate(a.warmup)
    kernels_per_iter = ctx.kernels_per_iteration()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # --- timed region: K iterations (census sums copied to the host), device
    # events on the context's stream ---
    clocks = ClockSampler(local_rank) if rank == 0 else None
    barrier()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sums, _, _ = ctx.iterate(a.steps)
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
    img = ctx.get_images()[0]

    # --- end to end through the C ABI: K iterations, each with its own pinned host
    # sinogram uploaded and its image downloaded (mlem_stream_host: the upload of
    # iteration k+1's sinogram and the download of iteration k's image overlap the
    # kernels); mlem_step_host, which also uploads the image and runs one call per
    # iteration without overlap, is reported beside it ---
    k_e2e = max(5, min(a.steps, 50))
    sino_h = [torch.from_numpy(frames.sinograms[0].copy()).pin_memory() for _ in range(2)]
    img_h = [torch.from_numpy(img.copy()).pin_memory() for _ in range(k_e2e)]
    sino_ptrs = [sino_h[k % 2].data_ptr() for k in range(k_e2e)]
    img_ptrs = [t.data_ptr() for t in img_h]
    ctx.stream_host_ptr(sino_ptrs[:2], img_ptrs[:2])  # warm (captures the 1-step graph)
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    ctx.stream_host_ptr(sino_ptrs, img_ptrs)
    f1.record(stream)
    barrier()
    e2e_ms = f0.elapsed_time(f1) / k_e2e
    step_h = torch.from_numpy(img.copy()).pin_memory()
    ctx.step_host_ptr(sino_h[0].data_ptr(), step_h.data_ptr(), 1)
    barrier()
    f0.record(stream)
    for _ in range(k_e2e):
        ctx.step_host_ptr(sino_h[0].data_ptr(), step_h.data_ptr(), 1)
    f1.record(stream)
    barrier()
    step_ms = f0.elapsed_time(f1) / k_e2e
    e2e = {"value": round(world * 1e3 / e2e_ms, 3), "unit": UNIT,
           "h2d_bytes_per_step": int(4 * ctx.n_rows),
           "d2h_bytes_per_step": int(4 * ctx.n_cols),
           "call": "mlem_stream_host (K iterations, each with its pinned host sinogram in and "
                   "its image out; copies overlap the kernels)",
           "step_host": {"value": round(world * 1e3 / step_ms, 3), "unit": UNIT,
                         "h2d_bytes_per_step": int(4 * ctx.n_rows + 4 * ctx.n_cols),
                         "d2h_bytes_per_step": int(4 * ctx.n_cols),
                         "call": "mlem_step_host (sinogram + image in, image out, one call per "
                                 "iteration)"}}

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
                "ms_per_launch": round(ph_ms[dom] / max(1, ph_launch[dom]), 4)}
    phases = {PHASES[p]: {"ms": round(float(ph_ms[p]), 4), "GB": round(ph_bytes[p] / 1e9, 4),
                          "GB/s": round(ph_bytes[p] / (ph_ms[p] / 1e3) / 1e9, 1) if ph_ms[p] > 0 else None,
                          "kernel": kernel_names[p], "launches": int(ph_launch[p])}
              for p in range(4)}
    tp = two_pass_bytes(ctx.nnz, ctx.n_rows, ctx.n_cols)

    head = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Siddon matrix, ellipsoid phantom, Poisson sinogram)",
        "config": workload_config(g, ctx.nnz, parallelism),
        "roofline": roofline, "e2e": e2e,
        "gpu_launches": int(kernels_per_iter * a.steps),
        "clocks": clk,
    }
    detail = {
        "tuning": {"bk_mode": api.BK_NAMES[tuning["bk_mode"]], "group": tuning["group"],
                   "frame_tile": tuning["frame_tile"], "blocks_per_sm": tuning["blocks_per_sm"],
                   "row_visit": api.VISIT_NAMES[tuning["visit"]],
                   # rows whose counts are zero add nothing to the update; the sorted
                   # one-pass walks leave them out (the roofline counts the rest)
                   "rows_with_counts": int(ctx.info.rows_with_counts),
                   "nnz_with_counts": int(ctx.info.nnz_with_counts)},
        "hbm_gbs": round(total_bytes / (ms_per_step / 1e3) / 1e9, 1),
        # the same iteration against the two-pass byte count of the reference's
        # algorithm (CSR pass for calcFwProj + CSC pass for calcBkProj):
        # 16 Z + 20 R + 24 C bytes over every row, which the one-pass kernel does
        # not move (one pass, and only the rows with counts)
        "two_pass_formula": {"bytes_per_iteration": tp,
                             "achieved_gbs": round(tp / (ms_per_step / 1e3) / 1e9, 1),
                             "frac": round(tp / (ms_per_step / 1e3) / 1e9 / peak, 4)},
        "iteration_roofline_frac": round(total_bytes / (ms_per_step / 1e3) / 1e9 / peak, 4),
        "bytes_per_iteration": total_bytes, "phases": phases,
        "last_image_sum": float(sums[-1, 0]), "setup_s": {"matrix": round(t_matrix, 2)},
    }
    tail = {}

    # --- the deterministic method (the CSC back projection, over the CSC in visiting
    # order with the sorted visit; the CLI's default), autotuned among the
    # deterministic methods and timed like the headline, then the fast tuning back ---
    if a.mode == "auto":
        td = ctx.autotune(deterministic_only=True)
        ctx.init_images()
        ctx.iterate(a.warmup, stats=False)
        kd = max(10, a.steps // 4)
        barrier()
        e0.record(stream)
        ctx.iterate(kd)
        e1.record(stream)
        barrier()
        dms = e0.elapsed_time(e1) / kd

        def set_sinograms_ms():
            # mlem_set_sinograms, host sums and upload included (best of 3)
            best = float("inf")
            for _ in range(3):
                barrier()
                e0.record(stream)
                ctx.set_sinograms(frames.sinograms)
                e1.record(stream)
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best

        # with the CSC method the call also refills its copy of the CSC in
        # visiting order cut to the rays with counts; the difference to the
        # same call under the fast method is that copy's cost per sinogram
        det_set = set_sinograms_ms()
        ctx.set_tuning(bk_mode=tuning["bk_mode"], group=tuning["group"],
                       frame_tile=tuning["frame_tile"], blocks_per_sm=tuning["blocks_per_sm"],
                       visit=tuning["visit"])
        fast_set = set_sinograms_ms()
        ctx.init_images()
        head["deterministic"] = {
            "method": f"{api.BK_NAMES[td['bk_mode']]}/{api.VISIT_NAMES[td['visit']]}",
            "ms_per_iteration": round(dms, 4), "iterations_per_s": round(world * 1e3 / dms, 3),
            "two_pass_formula_frac": round(tp / (dms / 1e3) / 1e9 / peak, 4),
            "set_sinograms_ms": round(det_set, 3), "set_sinograms_ms_fast_method": round(fast_set, 3)}

    host_legs = rank == 0 and world == 1 and not a.no_cpu_baseline
    wb = synth.WORKLOADS["batched-b16"]
    fb = synth.make_frames(wb, ctx.project_f64) if not a.no_batched else None
    # the batched frame checked against the reference binary: the one with the
    # fewest counts (the noisiest reconstruction)
    kf = int(np.argmin(fb.totals)) if fb is not None else None

    # --- host legs: the reference's openmpcsr4mlem timed on this host, then the
    # full-size parity jobs started in the background ---
    d = jobs = mpath = spaths = None
    if host_legs:
        need = 8 * ctx.nnz + 8 * ctx.n_rows + 12 * ctx.n_rows
        d = scratch_dir(need)
    try:
        if host_legs and d is None:
            head["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": "unavailable: no scratch space for the CSR4 file"}
        elif host_legs:
            row_end, elems = ctx.csr()
            sinos = {"plain": frames.sinograms[0]}
            if fb is not None:
                sinos["batched_frame"] = fb.sinograms[kf]
            mpath, spaths = write_csr4_and_sinos(d, row_end, elems, ctx.n_rows, ctx.n_cols,
                                                 (g.nx, g.ny, g.nz), sinos)
            del row_end, elems
            head["cpu_baseline"] = cpu_baseline(ctx, mpath, spaths["plain"], frames.sinograms[0],
                                                a.cpu_iters)
            if not a.no_parity_full:
                jobs = ParityJobs(d, mpath, spaths, a.parity_iters, host_threads())

        # --- what the L2 serves to random addresses (the one-pass walk's bound) ---
        l2 = api.measure_l2_rates(torch.cuda.current_device())
        head["l2_rates"] = {k: round(v / 1e9, 1) for k, v in l2.items()}
        head["l2_rates"]["unit"] = "G/s"
        # the dominant kernel against the L2's float-reduction rate: its reduction
        # sector operations per launch (committed ncu capture, scaled to this
        # workload) at the measured rate of random 4-byte reductions
        red = committed_traffic().get(roofline["kernel"] + "_red_sectors")
        if red and frames.sinograms.shape[0] == 1:
            floor = red / l2["red_4B_per_s"] * 1e3
            roofline["l2_reduction_floor_ms"] = round(floor, 4)
            roofline["frac_of_l2_reduction_floor"] = round(floor / roofline["ms_per_launch"], 4)

        # --- batched: 16 sinograms in one pass over the matrix per iteration ---
        if fb is not None:
            ctx.set_sinograms(fb.sinograms)
            ctx._refresh()
            visited16 = int(ctx.info.nnz_with_counts)
            ctx.init_images()
            tb = ctx.autotune()
            ctx.init_images()
            ctx.iterate(a.warmup, stats=False)
            kb = max(10, a.steps // 4)
            barrier()
            e0.record(stream)
            ctx.iterate(kb)
            e1.record(stream)
            barrier()
            bms = e0.elapsed_time(e1) / kb
            bph_ms, bph_bytes, _ = ctx.profile_phases(10)
            tail["batched"] = {
                "frames": 16, "ms_per_iteration": round(bms, 4),
                "per_frame_speedup_vs_plain": round((16 / bms) / (1 / ms_per_step), 3),
                "frame_iterations_per_s": round(16 * 1e3 / bms, 1),
                "hbm_gbs": round(float(bph_bytes.sum()) / (bms / 1e3) / 1e9, 1),
                "method": f"{api.BK_NAMES[tb['bk_mode']]}/{api.VISIT_NAMES[tb['visit']]}"
                          f"/tile{tb['frame_tile']}",
                # one 64-byte row reduction per visited element at 16 frames, at the
                # measured rate of random 64-byte row reductions
                "reduction_floor_ms": round(visited16 / l2["red_64B_rows_per_s"] * 1e3, 3),
            }
            detail["batched_phases_ms"] = [round(float(x), 4) for x in bph_ms]

        # --- full-size parity, GPU side (the host jobs run meanwhile) ---
        pf = None
        if jobs is not None and jobs.error is None:
            pf = parity_gpu_side(ctx, a, tuning, frames.sinograms, fb, tb if fb is not None else None,
                                 kf, d, mpath, spaths["plain"])

        # --- ordered subsets: 8 interleaved row subsets, the plain sinogram ---
        if not a.no_osem:
            detail["osem"] = osem_line(ctx, a, frames.sinograms, stream, barrier, ms_per_step)

        # --- differentiable MLEM: 10 unrolled iterations, gradient of an MSE loss ---
        if not a.no_differentiable:
            detail["differentiable"] = differentiable_line(ctx, a, stream, barrier)
        ctx.close()

        # --- a skewed matrix: the long rows run as segments (k_long.cu) ---
        if not a.no_skewed:
            detail["skewed"] = skewed_line(a, stream, barrier)

        # --- uneven batch over three geometries (12 + 8 + 4 frames), one GPU ---
        if world == 1 and not a.no_uneven:
            from mlem_b200 import uneven
            torch.cuda.synchronize()
            u = uneven.run(iters=max(10, min(a.steps, 20)), warmup=3, device=local_rank)
            detail["uneven"] = u

        # --- a symmetry-compressed matrix: expanded on the device vs mirrors in the kernels ---
        if world == 1 and not a.no_mirrored:
            from mlem_b200 import mirrored
            torch.cuda.synchronize()
            detail["mirrored"] = mirrored.run(iters=10, warmup=3, device=local_rank)

        # --- matrix-free: the rays traced in every pass instead of the stored matrix ---
        if world == 1 and not a.no_matrix_free:
            torch.cuda.synchronize()
            mfl, mf_img = matrix_free_line(a, frames.sinograms[0], stream, barrier, ms_per_step,
                                           pf["fast"] if pf else None)
            detail["matrix_free"] = mfl
            if pf is not None:
                pf["matrix_free"] = mf_img

        # --- full-size parity, host side: wait for the reference binary and the oracle ---
        if jobs is not None:
            tail["parity_full"] = parity_finish(jobs, pf, a.parity_iters)
    finally:
        if d is not None:
            shutil.rmtree(d, ignore_errors=True)

    if "uneven" in detail:
        u = detail["uneven"]
        tail["uneven_summary"] = {"ms_per_iteration": u["batch_ms_per_iteration"],
                          "speedup_vs_separate": u["speedup_vs_separate"],
                          "hbm_gbs": u["hbm_gbs"],
                          "max_rel_l2_vs_separate": sig(u["max_rel_l2_batch_vs_separate"])}
    if dist is not None:
        dist.destroy_process_group()
    return detail, head, tail


def cpu_baseline(ctx, mpath, spath, sino, iters):
    """openmpcsr4mlem on all host cores, on the bench's CSR4 file."""
    from mlem_b200 import api
    if not os.path.exists(REF_MESSUNG):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/openmpcsr4mlem_messung not built"}
    import numpy as np
    threads = host_threads()
    secs, wall, out = run_reference_binary(mpath, spath, iters, threads)
    per = statistics.mean(secs[1:]) if len(secs) > 1 else secs[0]
    ref_img = np.fromfile(out, dtype=np.float32)
    ctx.set_sinograms(sino)
    ctx.init_images()
    ctx.iterate(iters, stats=False)
    return {"value": round(1.0 / per, 4), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{iters} full iterations of openmpcsr4mlem (reference source, -O3 -fopenmp "
                      f"-DMESSUNG) on the same plain-full CSR4 file; mean of iterations 2..{iters}; "
                      f"wall {wall:.1f} s incl. load and serial column sums",
            "iteration_seconds": secs,
            "parity": {"iterations": iters,
                       "rel_l2_vs_reference_image": rel_l2(ctx.get_images()[0], ref_img),
                       "tolerance": TOL, "method": api.BK_NAMES[ctx.tuning()["bk_mode"]]}}


def parity_gpu_side(ctx, a, tuning, sinograms, fb, tb, kf, d, mpath, spath):
    """The GPU images of the full-size parity check (60 iterations):
    * fast: the autotuned one-pass path on the bench's context;
    * cli: the command-line drop-in with a checkpoint every 10 iterations
      (the deterministic CSC method, its default);
    * batch: the 16-frame batch, and every frame run on its own with the same
      method and visit (frame tile 1)."""
    import numpy as np

    from mlem_b200 import api
    n = a.parity_iters
    out = {}
    ctx.set_sinograms(sinograms)
    ctx.set_tuning(**{k: tuning[k] for k in ("bk_mode", "group", "frame_tile", "blocks_per_sm",
                                              "visit")})
    ctx.init_images()
    ctx.iterate(n, stats=False)
    out["fast"] = ctx.get_images()[0]
    out["fast_method"] = f"{api.BK_NAMES[tuning['bk_mode']]}/{api.VISIT_NAMES[tuning['visit']]}"
    try:
        out["cli"], out["cli_clean"], out["cli_wall"], out["cli_phases"] = run_cli(d, mpath, spath,
                                                                                 n, 10)
    except Exception as e:  # reported, not fatal
        out["cli_error"] = str(e)[:200]
    if fb is not None:
        ctx.set_sinograms(fb.sinograms)
        ctx.set_tuning(**{k: tb[k] for k in ("bk_mode", "group", "frame_tile", "blocks_per_sm",
                                              "visit")})
        ctx.init_images()
        ctx.iterate(n, stats=False)
        batch = ctx.get_images()
        worst = 0.0
        for b in range(fb.sinograms.shape[0]):
            ctx.set_sinograms(fb.sinograms[b:b + 1])
            ctx.set_tuning(bk_mode=tb["bk_mode"], group=tb["group"], frame_tile=1,
                           blocks_per_sm=tb["blocks_per_sm"], visit=tb["visit"])
            ctx.init_images()
            ctx.iterate(n, stats=False)
            worst = max(worst, rel_l2(batch[b], ctx.get_images()[0]))
        out["batch_frame"] = batch[kf]
        out["batch_vs_single_max"] = worst
        out["kf"] = kf
        ctx.set_sinograms(sinograms)
    return out


def parity_finish(jobs, pf, n):
    """Relative L2 errors of the 60-iteration images: ours against the
    reference's seqcsr4mlem, and ours and the reference's against the FP64
    oracle of the same iterations."""
    if jobs.error:
        return {"iterations": n, "error": jobs.error}
    if pf is None or "fast" not in pf:
        return {"iterations": n, "error": "no GPU images (the GPU side did not run)"}
    try:
        ref, wait_s = jobs.collect()
    except Exception as e:
        return {"iterations": n, "error": str(e)[:300]}
    res = {"iterations": n, "tolerance": TOL, "reference": "seqcsr4mlem (1 core)",
           "fp64_oracle_threads": jobs.f64_threads, "host_wall_s": round(wait_s, 1)}
    seq, f64 = ref["plain"]
    p = {"fast_vs_seq": sig(rel_l2(pf["fast"], seq)), "fast_vs_f64": sig(rel_l2(pf["fast"], f64)),
         "seq_vs_f64": sig(rel_l2(seq, f64)), "fast_method": pf["fast_method"]}
    if "cli" in pf:
        p.update({"cli_chk10_vs_seq": sig(rel_l2(pf["cli"], seq)),
                  "cli_chk10_vs_f64": sig(rel_l2(pf["cli"], f64)),
                  "cli_checkpoints_removed": pf["cli_clean"],
                  # the command-line run end to end (process start to exit) and its phases;
                  # the host cores run the reference's parity jobs meanwhile
                  "cli_wall_s": round(pf["cli_wall"], 2), "cli_phases_s": pf["cli_phases"]})
    else:
        p["cli_error"] = pf.get("cli_error")
    res["plain"] = p
    if "matrix_free" in pf:
        p["matrix_free_vs_seq"] = sig(rel_l2(pf["matrix_free"], seq))
        p["matrix_free_vs_f64"] = sig(rel_l2(pf["matrix_free"], f64))
    if "batched_frame" in ref and "batch_frame" in pf:
        bseq, bf64 = ref["batched_frame"]
        res["batched"] = {"frame": pf["kf"],
                          "batch_vs_seq": sig(rel_l2(pf["batch_frame"], bseq)),
                          "batch_vs_f64": sig(rel_l2(pf["batch_frame"], bf64)),
                          "seq_vs_f64": sig(rel_l2(bseq, bf64)),
                          "max_frame_vs_single_run": sig(pf["batch_vs_single_max"])}
    worst = [v for blk in (res.get("plain", {}), res.get("batched", {}))
             for k, v in blk.items() if k.endswith("_vs_seq") or k == "max_frame_vs_single_run"]
    res["ok"] = bool(worst) and all(v is not None and v <= TOL for v in worst)
    return res


def matrix_free_line(a, sino, stream, barrier, ms_stored, fast_img):
    """The matrix-free prototype (mlem_mf_*): the plain-full rays kept as
    104-byte descriptors and traced again in every pass.  Device-timed
    iterations, its device memory, and its image after the parity iteration
    count against the stored path's (the same iterations); the 256x256x96
    geometry (16.8M rays, whose stored matrix is 41 GB) timed alone."""
    import numpy as np
    import torch

    from mlem_b200 import api, synth
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {}
    img = None
    for name in ("plain-full", "uneven-large"):
        g = synth.WORKLOADS[name].geometry
        with api.MatrixFree(g) as mf:
            mf.set_stream(stream.cuda_stream)
            if name == "plain-full":
                s = sino
            else:  # a uniform-count stand-in: every ray walked, nothing skipped
                s = np.full(g.n_rows, 50, np.int32)
            mf.set_sinogram(s)
            mf.init_image()
            mf.iterate(3)
            k = max(5, min(a.steps, 20))
            barrier()
            e0.record(stream)
            mf.iterate(k)
            e1.record(stream)
            barrier()
            ms = e0.elapsed_time(e1) / k
            info = mf.info()
            entry = {"ms_per_iteration": round(ms, 4), "device_bytes": info["device_bytes"],
                     "rays": g.n_rows,
                     "sinogram": "plain-full" if name == "plain-full"
                                 else "50 counts on every ray (every ray walked)"}
            if name == "plain-full":
                entry["stored_ms_per_iteration"] = round(ms_stored, 4)
                mf.init_image()
                mf.iterate(a.parity_iters)
                img = mf.get_image()
                if fast_img is not None:
                    entry["rel_l2_vs_stored_path"] = sig(rel_l2(img, fast_img))
                    entry["iterations"] = a.parity_iters
            out[name] = entry
    return out, img


def osem_line(ctx, a, sinograms, stream, barrier, ms_per_step):
    import torch

    from mlem_b200 import api
    n_sub = 8
    ctx.set_sinograms(sinograms)
    ctx.init_images()
    ctx.set_subsets(n_sub)
    to = ctx.autotune()
    ctx.init_images()
    ctx.iterate(a.warmup, stats=False)
    ko = max(10, a.steps // 2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    ctx.iterate(ko, stats=False)
    e1.record(stream)
    barrier()
    oms = e0.elapsed_time(e1) / ko
    out = {"workload": "plain-full", "subsets": n_sub, "ms_per_iteration": round(oms, 4),
           "sub_iterations_per_s": round(n_sub * 1e3 / oms, 2),
           "iteration_time_vs_plain": round(oms / ms_per_step, 3),
           "frame_tile": to["frame_tile"], "group": to["group"],
           "row_visit": api.VISIT_NAMES[to["visit"]],
           "gpu_launches_per_iteration": int(ctx.kernels_per_iteration())}
    ctx.set_subsets(1)
    return out


def differentiable_line(ctx, a, stream, barrier):
    """The plain-full matrix: K = 10 relaxed MLEM iterations from a uniform
    start through torch_ext.unrolled_mlem, loss = mean squared error of the
    last image against the phantom, gradients with respect to the start image
    and the per-iteration exponents.  One step = forward + backward (the
    forward keeps each iteration's row sums and update factor, 0.21 GB for
    the ten iterations; the backward propagates the adjoint through calcCorrel
    and both projections in one pass per iteration)."""
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
    # passes over the matrix per iteration: forward 1 (one-pass ratio with the row
    # sums A x kept); backward 1 (the adjoint pass A^T df(A du))
    return {"workload": "differentiable", "unrolled_iterations": K, "ms_per_gradient_step": round(ms, 3),
            "matrix_passes_per_step": 2 * K, "ms_per_matrix_pass": round(ms / (2 * K), 4),
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


# ---------------------------------------------------------------------------
# our implementation, row shards over N GPUs (strong scaling)
# ---------------------------------------------------------------------------
def run_shards(a, rank, world, local_rank):
    """The plain-full matrix split into nnz-balanced row blocks (the
    reference's partition, mpicsr4mlem.cpp:202-234), one per rank; each
    iteration is the block's one-pass partial update and ONE NCCL all-reduce
    of the C floats (fusedmpimlem.cpp:195-236).  Timed: K iterations on the
    device, max over ranks.  Rank 0 checks the image against a single-context
    run of the whole matrix."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    from mlem_b200 import api, distributed, synth

    torch.cuda.set_device(local_rank)
    if "MASTER_ADDR" not in os.environ:  # one rank without torchrun
        import socket
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0",
                          WORLD_SIZE="1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                            device_id=torch.device("cuda", local_rank))
    w = synth.WORKLOADS["plain-full"]
    g = w.geometry
    stream = torch.cuda.current_stream()
    t0 = time.time()
    full = api.Context.siddon(g, flags=api.FLAG_NO_CSC, device=local_rank)
    frames = synth.make_frames(w, full.project_f64)
    row_end, elems = full.csr()
    nnz = int(full.nnz)
    starts, ends = distributed.partition(row_end, world)
    blk = distributed.row_block(row_end, elems, int(starts[rank]), int(ends[rank]))
    del row_end, elems
    if rank != 0:
        full.close()
        full = None
    shard = distributed.CudaShard(blk, g.n_cols, frames.sinograms[0][blk.start:blk.end], local_rank,
                                  grid=(g.nx, g.ny, g.nz))
    setup_s = time.time() - t0
    x = distributed.init_image(shard, dist)
    distributed.iterate(shard, x, a.warmup, dist)
    dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    distributed.iterate(shard, x, a.steps, dist)
    e1.record(stream)
    dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    # end to end: every step uploads the rank's sinogram block from pinned host
    # memory and reads the image back into pinned host memory
    sino_h = torch.from_numpy(frames.sinograms[0][blk.start:blk.end].copy()).pin_memory()
    img_h = torch.empty(g.n_cols, dtype=torch.float32).pin_memory()
    k_e2e = max(5, min(a.steps, 50))
    dist.barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(k_e2e):
        shard.set_sinogram(sino_h.numpy())
        distributed.iterate(shard, x, 1, dist)
        img_h.copy_(x, non_blocking=True)
    f1.record(stream)
    dist.barrier()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1), f0.elapsed_time(f1)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, e2e_ms = float(t[0].item()), float(t[1].item()) / k_e2e
    img = shard.to_host(x)
    n_total = a.warmup + a.steps + k_e2e
    line = None
    if rank == 0:
        full.set_stream(stream.cuda_stream)
        full.set_sinograms(frames.sinograms)
        full.set_tuning(bk_mode=api.BK_FUSED, group=32, frame_tile=1, blocks_per_sm=4,
                        visit=api.VISIT_SORTED_CHUNKED)
        full.init_images()
        full.iterate(n_total, stats=False)
        ref = full.get_images()[0]
        full.close()
        line = ({"shard_rows": [int(s) for s in (starts[0], ends[0])], "setup_s": round(setup_s, 1)},
                {"metric": METRIC, "value": round(a.steps / (ms / 1e3), 3), "unit": UNIT,
                 "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                 "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True,
                 "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                 "data": "synthetic (seeded Siddon matrix, ellipsoid phantom, Poisson sinogram)",
                 "config": workload_config(g, nnz, "shards"),
                 "e2e": {"value": round(1e3 / e2e_ms, 3), "unit": UNIT,
                         "h2d_bytes_per_step": int(4 * (blk.end - blk.start)),
                         "d2h_bytes_per_step": int(4 * g.n_cols),
                         "call": "CudaShard.set_sinogram + distributed.iterate "
                                 "(pinned sinogram block in, image out)"},
                 # per iteration and rank: the one-pass kernel and the update apply
                 "gpu_launches": int(2 * a.steps * world),
                 "clocks": clk},
                {"shards": {"ranks": world, "allreduce_floats_per_iteration": int(g.n_cols),
                            "iterations": n_total,
                            "rel_l2_vs_single_context": sig(rel_l2(img, ref)),
                            "tolerance": TOL}})
    shard.close()
    dist.destroy_process_group()
    return line


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(a, rank, world, parallelism):
    """The reference's openmpcsr4mlem on this host's cores, on the plain-full
    workload.  The inputs are written by oracle_tool in a child process (the
    seeded generator and the FP64 projection, byte-identical to the GPU
    arm's), so this process maps no library of the package under test."""
    if rank != 0:
        return None
    import numpy as np

    from mlem_b200 import synth  # numpy-only parts: phantom, Poisson draw

    if not os.path.exists(REF_MESSUNG):
        return {"impl": "reference", "unavailable": "oracle/_ref/openmpcsr4mlem_messung is not built"}
    if not os.path.exists(ORACLE_TOOL):
        return {"impl": "reference", "unavailable": "oracle/_bin/oracle_tool is not built"}
    w = synth.WORKLOADS["plain-full"]
    g = w.geometry
    d = scratch_dir(8 * 9e8)
    if d is None:
        return {"impl": "reference", "unavailable": "no scratch space for the 6 GB CSR4 file"}
    try:
        mp = os.path.join(d, "matrix.csr4")
        subprocess.run([ORACLE_TOOL, "synth-matrix", str(g.nx), str(g.ny), str(g.nz),
                        str(g.n_rows), str(g.min_count), str(g.max_count), str(g.seed),
                        repr(g.radius_scale), repr(g.min_len), mp], check=True, timeout=1200)
        with open(mp, "rb") as f:
            nnz = int(np.frombuffer(f.read(24)[16:24], np.uint64)[0])
        n_ell, counts = synth.frame_spec(w, 0)
        x = synth.phantom(g.nx, g.ny, g.nz, n_ell, w.frame_seed(0))
        xp, mp_out = os.path.join(d, "phantom.f32"), os.path.join(d, "means.f64")
        x.astype(np.float32).tofile(xp)
        subprocess.run([ORACLE_TOOL, "project-f64", mp, xp, mp_out], check=True, timeout=600)
        sino = synth.poisson_sinogram(np.fromfile(mp_out, np.float64), counts, w.frame_seed(0) + 500)
        sp = os.path.join(d, "plain.sino")
        sino.astype(np.int32).tofile(sp)
        threads = host_threads()
        k = max(1, min(a.steps, 20))
        wu = max(3, min(a.warmup, 5))  # at least 3 warm-up iterations, at most 5 (bounded run)
        secs, wall, _ = run_reference_binary(mp, sp, wu + k, threads)
        timed = secs[wu:]
        per = statistics.mean(timed)
        value = 1.0 / per
        return {
            "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": world, "steps": len(timed), "warmup": wu, "ms_per_step": round(per * 1e3, 2),
            "higher_is_better": True, "scaling": "strong" if parallelism == "shards" else "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Siddon matrix, ellipsoid phantom, Poisson sinogram)",
            "config": workload_config(g, nnz, parallelism),
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
    parallelism = a.parallelism
    if parallelism == "auto":
        parallelism = "shards" if world > 1 else "single"
    if a.impl == "reference":
        line = run_reference(a, rank, world, parallelism)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        return
    if parallelism == "shards":
        parts = run_shards(a, rank, world, local_rank)
    else:
        parts = run_ours(a, rank, world, local_rank, parallelism)
    if rank == 0 and parts is not None:
        detail, head, tail = parts
        # one line: details first, then the contract's keys, then the short
        # summaries (batched, parity_full) last, where a tail of the output keeps them
        line = dict(detail)
        line.update(head)
        line.update(tail)
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
