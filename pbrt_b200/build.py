"""Builds libpbrt_b200.so in-tree for sm_100a.

nvcc cross-compiles here without a GPU. Host C++ (the BVH builder) is compiled with
-ffp-contract=off; the traversal kernels with -fmad=false on top of their explicit
round-to-nearest intrinsics, so that no fused multiply-add changes a rounding the
reference does not make.
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
LIB = os.path.join(HERE, "libpbrt_b200.so")
CLI_SRC = os.path.join(HERE, "cli", "pbrt_main.cpp")
CLI = os.path.join(HERE, "pbrt")  # the command-line renderer (src/main.rs), linked to the library
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("PBRT_NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", "g++",
                     "-I", CSRC, "-I", INCLUDE]
# Per-file extra flags: the parity-critical kernels forbid FMA contraction outright.
NVCC_EXTRA = {
    "kernels_trace.cu": ["-fmad=false"],
    "kernels_render.cu": ["-fmad=false"],
    "api.cu": ["-fmad=false"],
}
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-I", CSRC, "-I", INCLUDE]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + NVCC_EXTRA.get(src, []) + ["-c", path, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src} failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile (when a source is newer than the library) and return the library path."""
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = _sources()
    hdr = _headers_mtime()
    stale = []
    for s in cu + cpp:
        obj = os.path.join(BUILD, s + ".o")
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(os.path.join(CSRC, s)), hdr):
            stale.append(s)
    if stale:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(stale))) as ex:
            list(ex.map(lambda s: _compile(s, verbose), stale))
    objs = [os.path.join(BUILD, s + ".o") for s in cu + cpp]
    if stale or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking libpbrt_b200.so failed:\n{r.stdout}\n{r.stderr}")
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(LIB),
                                                                       os.path.getmtime(CLI_SRC)):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, CLI_SRC, "-o", CLI, "-L", HERE, "-l:libpbrt_b200.so",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"building the pbrt command failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
