"""Builds the native library (``renderer2_b200/_lib/librenderer2.so``) and the
``r2`` command-line tool for sm_100a with nvcc, in-tree.

Device code is compiled with ``-fmad=false`` and host code with
``-ffp-contract=off``: fused multiply-adds appear only where the sources write
``fmaf`` so the GPU and the host round identically.
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
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "librenderer2.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include")]
HOST_FLAGS = "-fPIC,-ffp-contract=off,-Wall,-Wno-unused-function"
NVCC_FLAGS = ARCH + COMMON + ["-lineinfo", "-fmad=false", "--expt-relaxed-constexpr",
                              "-Xcompiler", HOST_FLAGS, "-Xptxas", "-warn-spills"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp") and f != "r2_cli.cpp")
    return cu, cpp


def _needs(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "r2.h"))
    return hs


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not _needs(obj, [src] + _headers()):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [NVCC, "-x", "c++"] + COMMON + ["-Xcompiler", HOST_FLAGS, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj


def build(verbose: bool = False) -> str:
    """Compile every CUDA/C++ source and link the shared library; returns its path."""
    if shutil.which(NVCC) is None and not os.path.exists(NVCC):
        raise RuntimeError("nvcc not found; the native library cannot be built")
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    cu, cpp = _sources()
    srcs = [os.path.join(CSRC, f) for f in cu + cpp]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _needs(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    cli_src = os.path.join(CSRC, "r2_cli.cpp")
    cli = os.path.join(LIBDIR, "r2")
    if os.path.exists(cli_src) and _needs(cli, [cli_src, LIB]):
        cmd = [NVCC, "-x", "c++"] + COMMON + [cli_src, "-o", cli, "-L", LIBDIR, "-lrenderer2",
                                             "-Xlinker", "-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"cli link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
