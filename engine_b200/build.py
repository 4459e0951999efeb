"""Builds engine_b200/libparadmm_b200.so in-tree for sm_100a.

    python -m engine_b200.build [--force]

graph.c is compiled with gcc; the CUDA sources with nvcc for
``-gencode arch=compute_100a,code=sm_100a``.  generic_kernels.cu is compiled
with ``-fmad=false`` so its FP64 arithmetic rounds exactly as the reference C
does.  Objects go to engine_b200/_build/ (not committed); the shared library
sits next to this file so it travels with the repository snapshot.
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
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libparadmm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                      "-I" + INCLUDE, "-I" + CSRC, "--expt-relaxed-constexpr"]
CU_SOURCES = {
    "engine.cu": [],
    "packing_kernels.cu": [],
    "generic_kernels.cu": ["-fmad=false"],
    "noalloc.cu": [],
    "onchip_kernels.cu": [],
    "setmlp.cu": [],
    "userops.cu": [],
}
C_SOURCES = {"graph.c": ["-O2", "-std=gnu11", "-fPIC", "-ffp-contract=off"]}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    jobs = []
    objs = []
    for src, extra in CU_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([nvcc] + NVCC_COMMON + extra + ["-c", s, "-o", o])
    for src, extra in C_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["gcc"] + extra + ["-I" + INCLUDE, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(4, max(1, len(jobs)))) as ex:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd), flush=True)
        list(ex.map(_run, jobs))
    if force or jobs or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        _run([nvcc] + ARCH + ["-shared", "-Xlinker", "-Bsymbolic", "-o", tmp] + objs + ["-ldl", "-lm"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
