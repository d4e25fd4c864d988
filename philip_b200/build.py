"""Builds the in-tree CUDA library ``philip_b200/libphilip_b200.so`` for sm_100a.

The kernels are instantiated once per polynomial order (``ph_inst.cu`` with
``-DPH_N1=<p+1>``); the orders compile in parallel and are linked with the C-ABI
(``ph_capi.cu``, ``ph_batch.cu``) into one shared library. nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libphilip_b200.so")
N1_RANGE = range(2, 8)          # p = 1 .. 6
HOST_UNITS = ("ph_capi", "ph_batch", "ph_server", "ph_snapshots")   # C-ABI units

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".hpp"))] + \
        [os.path.join(HERE, "..", "include", "philip_b200.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    """Compile (when sources are newer than the library) and return the library path."""
    deps = _sources()
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    jobs = []
    for n1 in N1_RANGE:
        obj = os.path.join(BUILD, f"ph_inst_{n1}.o")
        jobs.append([nvcc, *NVCC_FLAGS, *extra, f"-DPH_N1={n1}", "-c", os.path.join(CSRC, "ph_inst.cu"), "-o", obj])
    for unit in HOST_UNITS:
        jobs.append([nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, unit + ".cu"), "-o", os.path.join(BUILD, unit + ".o")])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        for out in ex.map(lambda c: _run(c, verbose), jobs):
            logs.append(out)
    objs = [os.path.join(BUILD, f"ph_inst_{n1}.o") for n1 in N1_RANGE] + \
        [os.path.join(BUILD, unit + ".o") for unit in HOST_UNITS]
    tmp = LIB + ".tmp"
    _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp, *objs, "-lcudart", "-lcublas", "-ldl"],
         verbose)
    os.replace(tmp, LIB)
    if ptxas_info:
        sys.stdout.write("\n".join(logs))
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
