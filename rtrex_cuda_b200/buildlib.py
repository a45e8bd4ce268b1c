"""Build librtr.so and the rtrex_b200 CLI in-tree for sm_100a.

``python -m rtrex_cuda_b200.buildlib`` (or ``__graft_entry__.build()``) compiles
every CUDA / C++ source under ``csrc/`` with nvcc for ``sm_100a`` and links
``rtrex_cuda_b200/librtr.so`` plus the ``rtrex_cuda_b200/rtrex_b200`` binary.
Objects go to ``rtrex_cuda_b200/_build/``.  Floating-point contraction is
disabled (``-fmad=false``) so every add / multiply rounds as the reference's
x86-64 SSE2 code does.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librtr.so")
CLI = os.path.join(HERE, "rtrex_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
           "-I" + os.path.join(ROOT, "include")]
SOURCES = ["primitives.cu", "graph.cu", "count.cu", "count_rows.cu", "clean.cu", "clean_rounds.cu", "extract.cu", "capi.cu", "io.cpp", "noalloc.cu", "components.cu", "expand.cu", "escape.cu", "serve.cpp", "gen.cu", "nucleus.cu"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "rtr.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [os.path.join(CSRC, src)] + _headers()
    if _stale(obj, deps):
        cmd = [_nvcc(), *ARCH, *NVFLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if _stale(LIB, objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    cli_obj = _compile("cli.cpp", verbose)
    if _stale(CLI, [cli_obj, LIB]):
        cmd = [_nvcc(), *ARCH, "-o", CLI, cli_obj, "-L" + HERE, "-lrtr", "-Xlinker", "-rpath=$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
