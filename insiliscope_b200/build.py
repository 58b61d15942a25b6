"""Builds libiscu.so in-tree: the sm_100a CUDA kernels and the C ABI (include/iscu.h).

Each translation unit is compiled on its own (in parallel) into ``insiliscope_b200/_build/`` and relinked only when
a source or header is newer than the library. Units that must round exactly as the reference's
``-ffp-contract=off`` build does are compiled without floating-point contraction (``--fmad=false`` for nvcc,
``-ffp-contract=off`` for g++).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libiscu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INC = "/usr/local/cuda/include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# unit -> extra flags
UNITS = {
    "splat_noise.cu": ["--fmad=false"],
    "render.cu": ["--fmad=false"],
    "render_contrib.cu": ["--fmad=false"],
    "collect.cu": ["--fmad=false"],
    "nll.cu": [],
    "psf.cu": [],
    "psf_tc.cu": [],
    "psf_tc16.cu": [],
    "psf_noalloc.cu": [],
    "psf_plan.cu": [],
    "widefield.cu": ["--fmad=false"],
    "backend.cu": ["--fmad=false"],
    "schedule.cu": ["--fmad=false"],
    "binned.cu": [],
    "tiff.cpp": [],
    "csv.cu": [],
    "fft_place.cu": ["--fmad=false"],
    "halo.cu": [],
    "capi.cpp": [],
    "host_models.cpp": [],
}


def _headers():
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def _compile(unit: str, extra: list[str], newest_header: float, verbose: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
        return obj
    if unit.endswith(".cu"):
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
               "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE, *extra, "-c", src, "-o", obj]
    else:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
               "-I", CSRC, "-I", INCLUDE, "-I", CUDA_INC, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(BUILD, unit + ".log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {unit} failed:\n{r.stdout}{r.stderr}")
    if verbose:
        print(f"[iscu build] {unit}", file=sys.stderr)
    return obj


def build_library(verbose: bool = False) -> str:
    """Compiles and links libiscu.so (sm_100a); returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    newest = max(os.path.getmtime(h) for h in _headers())
    units = [u for u in UNITS if os.path.exists(os.path.join(CSRC, u))]
    with ThreadPoolExecutor(max_workers=max(1, min(len(units), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda u: _compile(u, UNITS[u], newest, verbose), units))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs, "-lcudart_static", "-lpthread",
           "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"linking libiscu.so failed:\n{r.stdout}{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build_library(verbose=True))
