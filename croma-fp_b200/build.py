"""Builds the CUDA library for sm_100a, in tree.

    python croma-fp_b200/build.py            # all bin counts
    python croma-fp_b200/build.py 256        # one bin count

Produces croma-fp_b200/lib/libcroma_b200_np{128,256,512}.so.  The bin count
is a compile-time constant (as np/npe are in the reference), so one library
is built per supported value.  schedule.cu is compiled with --fmad=false so
that the sub-step estimator keeps the reference's rounding sequence.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJROOT = os.path.join(HERE, "_build")
NBS = (128, 256, 512)
SOURCES = ("api.cu", "tables.cu", "schedule.cu", "fused.cu", "dsa.cu", "serve.cu",
           "ref_abi.cu", "noalloc.cu", "output.cu", "emission.cu", "h5lite.cpp", "background.cu")
NO_FMAD = {"schedule.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _flags(nb: int, src: str):
    f = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", f"-DCROMA_NB={nb}",
         "-Xptxas", "-warn-spills"]
    if src in NO_FMAD:
        f.append("--fmad=false")
    return f


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _compile(nb: int, src: str, verbose: bool):
    objdir = os.path.join(OBJROOT, f"np{nb}")
    os.makedirs(objdir, exist_ok=True)
    obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".cuh")]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "croma_b200.h"))
    if _newer(obj, deps):
        return obj
    cmd = [nvcc(), *_flags(nb, src), "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src} (nb={nb}):\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj


def build(nbs=NBS, verbose: bool = False, jobs: int = 0) -> list:
    os.makedirs(LIBDIR, exist_ok=True)
    jobs = jobs or min(12, (os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = {(nb, s): ex.submit(_compile, nb, s, verbose) for nb in nbs for s in SOURCES}
        objs = {k: f.result() for k, f in futs.items()}
    libs = []
    for nb in nbs:
        lib = os.path.join(LIBDIR, f"libcroma_b200_np{nb}.so")
        o = [objs[(nb, s)] for s in SOURCES]
        if not _newer(lib, o):
            cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib, *o,
                   "-Xcompiler", "-fPIC"]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed (nb={nb}):\n{r.stdout}\n{r.stderr}")
        libs.append(lib)
    return libs


if __name__ == "__main__":
    sel = tuple(int(a) for a in sys.argv[1:]) or NBS
    for p in build(sel, verbose=True):
        print(p)
