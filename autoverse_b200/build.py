"""In-tree build of the engine library ``autoverse_b200/_lib/libflowlenia_cuda.so``.

Every CUDA translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); host C++ is compiled with
``-ffp-contract=off`` so seed generation and stencil taps keep the
reference's f32 rounding.  Objects are rebuilt when a source or header is
newer than the library.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libflowlenia_cuda.so")
EXTRA = os.environ.get("FLP_NVCC_EXTRA", "").split()
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-Wno-deprecated-gpu-targets", "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
          "-I", CSRC, "-I", INCLUDE]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _newest_header() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False, lib: str = LIB,
          objdir: str = OBJDIR) -> str:
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    os.makedirs(objdir, exist_ok=True)
    hdr = _newest_header()
    objs, jobs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
            continue
        cmd = [NVCC, *ARCH, *COMMON, *EXTRA, "-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if ptxas_verbose else []
        else:
            cmd = [NVCC, *COMMON, "-x", "c++", "-c", src, "-o", obj]
        jobs.append(cmd)
    # translation units are independent: compile them concurrently
    workers = max(1, min(len(jobs), os.cpu_count() or 1))

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=workers) as ex:
        for f in [ex.submit(run, c) for c in jobs]:
            f.result()
    if force or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv))
