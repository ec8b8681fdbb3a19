"""Builds the CUDA library in-tree: medyan_b200/libmedyan_b200.so (sm_100a).

Each translation unit is compiled by nvcc to an object under medyan_b200/_build/
and linked into one shared library. Every file is compiled without FMA
contraction: the excluded-volume formula needs it to round as the reference
does (see excl_kernels.cu), and a force computed by two different kernels
(the fused pass, the per-potential kernels of the speculative pass and of
packed batches) must round the same way in both. Run: python -m medyan_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmedyan_b200.so")
# profiling build: the same sources with the pass timeline compiled in
# (-DMEDYAN_PASS_TRACE), a library of its own that only
# medyan_b200/pass_timeline.py loads
BUILD_TRACE = os.path.join(HERE, "_build_trace")
LIB_TRACE = os.path.join(HERE, "libmedyan_b200_trace.so")

SOURCES = ["capi.cu", "ff_kernels.cu", "chain.cu", "excl_kernels.cu", "nl.cu", "cg.cu", "batch.cu", "pbatch.cu", "diff.cu", "hessian.cu", "aux.cu", "tune.cu", "noalloc.cu", "pass.cu", "async.cu", "vectorize.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
          "-I" + CSRC, "--expt-relaxed-constexpr", "--fmad=false"]
PER_FILE: dict[str, list[str]] = {}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, jobs: int | None = None, trace: bool = False) -> str:
    """Compiles the stale translation units (in parallel, one nvcc per core)
    and links the library (trace: the pass-timeline profiling library)."""
    from concurrent.futures import ThreadPoolExecutor
    build_dir, lib = (BUILD_TRACE, LIB_TRACE) if trace else (BUILD, LIB)
    extra = ["-DMEDYAN_PASS_TRACE"] if trace else []
    os.makedirs(build_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "medyan_b200.h"))
    objs, cmds = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path, *headers, __file__]):
            cmds.append([nvcc(), *ARCH, *COMMON, *extra, *PER_FILE.get(src, []), "-c", path, "-o", obj])

    def run(cmd: list[str]) -> None:
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    if cmds:
        # the longest translation units first
        cmds.sort(key=lambda c: -os.path.getsize(c[-3]))
        with ThreadPoolExecutor(max_workers=jobs or min(len(cmds), os.cpu_count() or 1)) as pool:
            for fut in [pool.submit(run, c) for c in cmds]:
                fut.result()
    if force or _stale(lib, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, trace="--trace" in sys.argv)
