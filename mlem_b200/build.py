"""In-tree build of the native parts of mlem_b200.

    python -m mlem_b200.build [--only gen|core|cli] [-j N]

* lib/libmlem_gen.so -- host Siddon generator (gcc, OpenMP, -ffp-contract=off)
* lib/libmlem_b200.so -- the CUDA library: sm_100a kernels + C-ABI + host IO
* bin/mlem_b200       -- the command-line drop-in for seqcsr4mlem/openmpcsr4mlem

nvcc compiles for sm_100a only (-gencode arch=compute_100a,code=sm_100a); it
cross-compiles without a GPU.  Objects are rebuilt when a source or header is
newer than the object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
GEN = os.path.join(PKG, "gen")
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")
OBJ = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# IEEE division and square root, FTZ to match the reference's flush-to-zero
# mode (mlem_seq/seqcsr4mlem.cpp:194), no fast math.
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-ftz=true", "-prec-div=true", "-prec-sqrt=true",
                     "--expt-relaxed-constexpr", "-ccbin", CXX,
                     f"-I{INCLUDE}", f"-I{CSRC}", f"-I{GEN}"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", f"-I{INCLUDE}", f"-I{CSRC}"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + p.stdout + p.stderr)
    return p.stdout + p.stderr


def _headers():
    return (glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True)
            + glob.glob(os.path.join(GEN, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def build_gen(verbose=False):
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libmlem_gen.so")
    src = os.path.join(GEN, "siddon_host.c")
    if _newer(out, [src, os.path.join(GEN, "siddon_core.h")]):
        _run([CC, "-O2", "-std=c11", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
              "-Wall", "-Wextra", "-shared", "-o", out, src, "-lm"])
        if verbose:
            print("built", out)
    return out


def _compile(src, jobs_verbose=False):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    obj = os.path.join(OBJ, rel + ".o")
    if _newer(obj, [src] + _headers()):
        if src.endswith(".cu"):
            _run([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
        else:
            _run([CXX] + CXX_FLAGS + ["-c", src, "-o", obj])
        if jobs_verbose:
            print("compiled", rel)
    return obj


def _lib_sources():
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    srcs += sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    return [s for s in srcs if not s.endswith("main.cpp")]


def build_core(verbose=False, jobs=8):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    srcs = _lib_sources()
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    out = os.path.join(LIB, "libmlem_b200.so")
    if _newer(out, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", out] + objs
             + ["-cudart", "static", "-lpthread", "-Xlinker", "-rpath,$ORIGIN", "-ccbin", CXX])
        if verbose:
            print("linked", out)
    return out


def build_cli(verbose=False):
    os.makedirs(BIN, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    main_src = os.path.join(CSRC, "host", "main.cpp")
    obj = _compile(main_src, verbose)
    out = os.path.join(BIN, "mlem_b200")
    core = os.path.join(LIB, "libmlem_b200.so")
    if _newer(out, [obj, core]):
        _run([CXX, "-o", out, obj, f"-L{LIB}", "-lmlem_b200", "-Wl,-rpath,$ORIGIN/../lib"])
        if verbose:
            print("linked", out)
    return out


def build_all(verbose=False, jobs=8):
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    outs = [build_gen(verbose)]
    if _lib_sources():
        outs.append(build_core(verbose, jobs))
    if os.path.exists(os.path.join(CSRC, "host", "main.cpp")):
        outs.append(build_cli(verbose))
    return outs


def clean():
    for d in (OBJ, LIB, BIN):
        shutil.rmtree(d, ignore_errors=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["gen", "core", "cli"])
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args(argv)
    if a.clean:
        clean()
    if a.only == "gen":
        print(build_gen(True))
    elif a.only == "core":
        print(build_core(True, a.j))
    elif a.only == "cli":
        print(build_cli(True))
    else:
        for o in build_all(True, a.j):
            print(o)


if __name__ == "__main__":
    sys.exit(main())
