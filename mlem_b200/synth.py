"""Seeded synthetic MLEM workloads (the reference has no generator and no data).

A workload is a Siddon system matrix (mlem_b200/gen/siddon_core.h), one or
more ellipsoid phantoms and Poisson sinograms of their projections:

* rows are lines of response between two points drawn uniformly on a
  cylinder of radius 1.2x the grid half-width, redrawn until their element
  count lies in the workload's "about lo-hi elements per row" window;
* a phantom is a number of ellipsoids of intensity uniform in [1, 10] painted
  on a zero background (later ellipsoids overwrite earlier ones);
* a sinogram is int32 Poisson(scale * A x_true), where A x_true is summed in
  double in element order and scale sets the expected total counts.

They stand in for the MADPET-II matrix and the Derenzo sinogram the
reference's thesis measured on, which are not available.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import formats
from ._native import gen_lib


@dataclass(frozen=True)
class Geometry:
    nx: int
    ny: int
    nz: int
    n_rows: int
    min_count: int = 1
    max_count: int = 0xFFFFFFFF
    seed: int = 0
    radius_scale: float = 1.2
    min_len: float = 1.0e-4

    @property
    def n_cols(self) -> int:
        return self.nx * self.ny * self.nz


@dataclass(frozen=True)
class Workload:
    """One reconstruction job: a geometry, B frames, an iteration count."""

    name: str
    geometry: Geometry
    frames: int = 1
    iterations: int = 10
    checkpoint: int = 0
    ellipsoids: tuple = (5, 5)  # (min, max) ellipsoids per phantom
    counts: tuple = (1e7, 1e7)  # (min, max) total counts per frame, log-uniform
    phantom_seed: int = 0

    def frame_seed(self, b: int) -> int:
        return self.phantom_seed + b


# The five workloads of the benchmark configuration list.  Seeds: matrix seed =
# workload index, phantom seed = 1000 * index + frame.
GEOM_SMALL = Geometry(32, 32, 16, 65536, 20, 80, seed=0)
GEOM_FULL = Geometry(128, 128, 64, 4194304, 150, 250, seed=1)
GEOM_LARGE = Geometry(256, 256, 96, 16777216, 250, 350, seed=4)

WORKLOADS = {
    "plain-small": Workload("plain-small", GEOM_SMALL, 1, 10, 0, (5, 5), (1e7, 1e7), 0),
    "plain-full": Workload("plain-full", GEOM_FULL, 1, 60, 10, (8, 8), (1e9, 1e9), 1000),
    "batched-b16": Workload("batched-b16", GEOM_FULL, 16, 60, 0, (3, 12), (1e6, 1e9), 2000),
    "differentiable": Workload("differentiable", GEOM_FULL, 1, 10, 0, (8, 8), (1e9, 1e9), 3000),
    "uneven-small": Workload("uneven-small", GEOM_SMALL, 12, 60, 0, (3, 12), (1e6, 1e9), 4000),
    "uneven-full": Workload("uneven-full", GEOM_FULL, 8, 60, 0, (3, 12), (1e6, 1e9), 4100),
    "uneven-large": Workload("uneven-large", GEOM_LARGE, 4, 60, 0, (3, 12), (1e6, 1e9), 4200),
}


def host_matrix(g: Geometry) -> formats.Csr4:
    """Generate the matrix on the host (libmlem_gen.so, OpenMP)."""
    lib = gen_lib()
    counts = np.zeros(g.n_rows, np.uint32)
    z = lib.mlem_gen_siddon_counts(g.nx, g.ny, g.nz, g.n_rows, g.min_count, g.max_count,
                                   g.radius_scale, g.min_len, g.seed,
                                   counts.ctypes.data_as(ctypes.c_void_p))
    row_end = np.cumsum(counts, dtype=np.uint64)
    elems = np.zeros(int(z), formats.ELEM_DTYPE)
    rc = lib.mlem_gen_siddon_fill(g.nx, g.ny, g.nz, g.n_rows, g.min_count, g.max_count,
                                  g.radius_scale, g.min_len, g.seed,
                                  row_end.ctypes.data_as(ctypes.c_void_p),
                                  elems.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError("Siddon fill disagrees with the counts pass")
    return formats.Csr4(g.n_rows, g.n_cols, row_end, elems, 0, (g.nx, g.ny, g.nz))


def project_f64(m: formats.Csr4, x: np.ndarray) -> np.ndarray:
    """Sequential double projection (the sinogram means)."""
    lib = gen_lib()
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(m.n_rows, np.float64)
    row_end = np.ascontiguousarray(m.row_end, dtype=np.uint64)
    elems = np.ascontiguousarray(m.elems)
    lib.mlem_gen_project_f64(m.n_rows, row_end.ctypes.data_as(ctypes.c_void_p),
                             elems.ctypes.data_as(ctypes.c_void_p),
                             x.ctypes.data_as(ctypes.c_void_p),
                             out.ctypes.data_as(ctypes.c_void_p))
    return out


def phantom(nx: int, ny: int, nz: int, n_ellipsoids: int, seed: int) -> np.ndarray:
    """Ellipsoids of intensity U[1,10] on zero, voxel-centre inclusion test;
    returned flat in voxel-index order ix + nx*(iy + ny*iz)."""
    rng = np.random.default_rng(seed)
    img = np.zeros((nz, ny, nx), np.float32)
    zc = np.arange(nz, dtype=np.float64)[:, None, None] + 0.5
    yc = np.arange(ny, dtype=np.float64)[None, :, None] + 0.5
    xc = np.arange(nx, dtype=np.float64)[None, None, :] + 0.5
    dims = np.array([nx, ny, nz], np.float64)
    for _ in range(n_ellipsoids):
        c = rng.uniform(0.3 * dims, 0.7 * dims)
        a = rng.uniform(0.08 * dims, 0.3 * dims)
        val = np.float32(rng.uniform(1.0, 10.0))
        inside = (((xc - c[0]) / a[0]) ** 2 + ((yc - c[1]) / a[1]) ** 2
                  + ((zc - c[2]) / a[2]) ** 2) <= 1.0
        img[inside] = val
    return img.reshape(-1)


def poisson_sinogram(means: np.ndarray, total_counts: float, seed: int) -> np.ndarray:
    """int32 Poisson counts with expected total `total_counts`."""
    rng = np.random.default_rng(seed)
    s = float(means.sum())
    lam = means * (total_counts / s) if s > 0 else np.zeros_like(means)
    return rng.poisson(lam).astype(np.int32)


def frame_spec(w: Workload, b: int):
    """(n_ellipsoids, total_counts) of frame b, drawn from the workload's ranges."""
    rng = np.random.default_rng(w.frame_seed(b) + 7)
    lo, hi = w.ellipsoids
    n_ell = int(rng.integers(lo, hi + 1))
    clo, chi = w.counts
    counts = float(10.0 ** rng.uniform(np.log10(clo), np.log10(chi))) if chi > clo else float(clo)
    return n_ell, counts


@dataclass
class Frames:
    phantoms: np.ndarray  # float32 [B, C]
    sinograms: np.ndarray  # int32 [B, R]
    totals: list = field(default_factory=list)


def make_frames(w: Workload, project) -> Frames:
    """Phantoms and sinograms of every frame; `project(x) -> float64[R]` is the
    double projector (host or device)."""
    g = w.geometry
    ph, sg, tot = [], [], []
    for b in range(w.frames):
        n_ell, counts = frame_spec(w, b)
        x = phantom(g.nx, g.ny, g.nz, n_ell, w.frame_seed(b))
        sg.append(poisson_sinogram(project(x), counts, w.frame_seed(b) + 500))
        ph.append(x)
        tot.append(counts)
    return Frames(np.stack(ph), np.stack(sg), tot)


def host_workload(w: Workload, matrix: Optional[formats.Csr4] = None):
    """Matrix + frames entirely on the host (small workloads and tests)."""
    m = matrix if matrix is not None else host_matrix(w.geometry)
    return m, make_frames(w, lambda x: project_f64(m, x))
