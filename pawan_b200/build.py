"""Builds the pawan B200 CUDA library in-tree.

    python -m pawan_b200.build [--force] [-j N]

Compiles every source under pawan_b200/csrc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) into pawan_b200/_build/*.o and links
pawan_b200/_lib/libpawan_b200.so (CUDA runtime linked statically).  Per-file
flags: the FP32 pair kernel flushes denormals (--ftz=true); the plain FP64
kernel does not contract multiply-adds (--fmad=false), like the reference's
x86-64 build.  Rebuilds only what changed (sources or any header).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIBDIR = os.path.join(ROOT, "_lib")
LIB = os.path.join(LIBDIR, "libpawan_b200.so")
INCLUDE = os.path.join(REPO, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-Wall",
                 "-I" + INCLUDE, "-I" + CSRC]
PER_FILE = {
    "pair_f32.cu": ["--ftz=true"],
    "noalloc.cu": ["--ftz=true"],
    "pair_plain.cu": ["--fmad=false"],
}
SOURCES = ["pair_f32.cu", "pair_f64.cu", "pair_plain.cu", "stage.cu", "diag.cu", "influence.cu",
           "peak.cu", "runtime.cpp", "abi.cpp", "serve.cpp", "writer.cpp", "noalloc.cu"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "pawan_b200.h"))
    return hs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc()] + COMMON + PER_FILE.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = _headers()
    todo = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, [os.path.join(CSRC, src)] + hdrs):
            todo.append(src)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
            for f in [ex.submit(_compile, s, verbose) for s in todo]:
                f.result()
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.j, a.v))


if __name__ == "__main__":
    sys.exit(main())
