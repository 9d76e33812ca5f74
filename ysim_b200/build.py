"""Build the sm_100a shared library in-tree: ysim_b200/lib/libysim_b200.so.

    python -m ysim_b200.build [--force] [-v]

nvcc cross-compiles for sm_100a without a GPU.  Each source is compiled to
its own object in parallel (ysim_b200/lib/obj/), then the objects are linked
into the library.  Arithmetic flags: -fmad=false with IEEE division and square
root, so float expressions round exactly as the reference's CPU build compiled
with -ffp-contract=off.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "libysim_b200.so")
OBJ = os.path.join(HERE, "lib", "obj")
SOURCES = ["ys_sort.cu", "ys_lbvh.cu", "ys_scan.cu", "ys_scene.cu", "ys_api.cu", "ys_shash.cu", "ys_shff.cu",
           "ys_analytic.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-diag-suppress", "549"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "ysim_b200.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool, verbose: bool):
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(SRC, src)
    if not force and not _stale(obj, [path, *_headers()]):
        return obj, ""
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-c", path, "-o", obj + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + r.stdout + r.stderr)
    os.replace(obj + ".tmp", obj)
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    if not force and not _stale(OUT, objs):
        return OUT
    cmd = [nvcc(), *ARCH, "-shared", *objs, "-o", OUT + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
