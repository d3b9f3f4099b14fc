"""Build libctb200.so (CUDA kernels + C ABI) in-tree for sm_100a.

Objects go to ``qtctreconstruction_b200/_build/``; the shared library lands at
``qtctreconstruction_b200/libctb200.so`` so it ships with the source tree.
Rebuilds only what changed (source or header newer than the object).

    python -m qtctreconstruction_b200.build [-v]
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libctb200.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-I" + os.path.join(ROOT, "include")] + ARCH
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-I" + os.path.join(ROOT, "include"),
            "-I/usr/local/cuda/include"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj: str, src: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src, *deps])


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC, *CUFLAGS, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", *CXXFLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    deps = _headers()
    todo = [s for s in srcs if force or verbose or _stale(os.path.join(BUILD, os.path.basename(s) + ".o"), s, deps)]
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(todo)))) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, "-shared", *ARCH, "-o", LIB, *objs, "-cudart", "static", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    build_cli(verbose)
    return LIB


CLI_SRC = os.path.join(PKG, "cli", "ctbench.cpp")
CLI = os.path.join(PKG, "bin", "ctbench")


def build_cli(verbose: bool = False) -> str:
    """The headless C++ bench CLI, linked against libctb200.so (rpath $ORIGIN/..)."""
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    if os.path.exists(CLI) and os.path.getmtime(CLI) >= max(os.path.getmtime(CLI_SRC), os.path.getmtime(LIB)):
        return CLI
    cmd = [NVCC, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-I" + os.path.join(ROOT, "include"),
           CLI_SRC, "-o", CLI,
           "-L" + PKG, "-lctb200", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/..", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"ctbench build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, file=sys.stderr)
    return CLI


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
