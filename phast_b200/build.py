"""Build the sm_100a shared library ``phast_b200/_lib/libphastb.so`` with nvcc.

The library is plain CUDA C++ with a C ABI (``include/phastb.h``); it links
only the CUDA runtime.  Building needs nvcc but no GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libphastb.so")
SOURCES = ["capi.cu", "q4.cu", "h8.cu", "h8_tile.cu", "engine.cu", "solvers2d.cu", "solvers3d.cu", "gmg.cu", "t3.cu",
           "batch3d.cu", "pfczm.cu", "closure.cu", "anderson.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the phast_b200 CUDA library cannot be built")


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "phastb.h")]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "phastb.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False):
    """Compile the sources whose object is missing or older than the source or any header, then link."""
    if not force and not _stale():
        return LIB
    obj_dir = os.path.join(OUT_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = nvcc_path()
    objs = [os.path.join(obj_dir, src.replace(".cu", ".o")) for src in SOURCES]
    newest_header = max(os.path.getmtime(h) for h in _headers())

    def out_of_date(src, obj):
        if force or not os.path.exists(obj):
            return True
        t = os.path.getmtime(obj)
        return t < os.path.getmtime(os.path.join(CSRC, src)) or t < newest_header

    def compile_one(src, obj):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        os.replace(obj + ".tmp", obj)

    todo = [(src, obj) for src, obj in zip(SOURCES, objs) if out_of_date(src, obj)]
    # translation units compile independently; the largest dominates the wall time
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo) or 1, os.cpu_count() or 1))) as pool:
        for f in [pool.submit(compile_one, src, obj) for src, obj in todo]:
            f.result()
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, *ARCH, "-shared", "--cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
