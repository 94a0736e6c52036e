"""Builds libnaga_b200.so in-tree with nvcc for sm_100a.

Objects go to naga_b200/_build/, the shared library to naga_b200/. Sources
are compiled in parallel and only rebuilt when a source or header changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libnaga_b200.so")
SOURCES = ["errors.cpp", "scene_gen.cpp", "knn.cu", "linalg.cu", "rbf.cu", "primitives.cu", "step.cu", "engine.cu", "server.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_compiler() -> list[str]:
    # the image may export CXX pointing at a toolchain nvcc cannot use
    for c in ("/usr/bin/g++-13", "/usr/bin/g++"):
        if os.path.exists(c):
            return ["-ccbin", c]
    return []


def _headers() -> list[str]:
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".hpp", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def _compile(src: str, extra: list[str], verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max(os.path.getmtime(p) for p in [src] + _headers())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj
    cmd = [nvcc(), *_host_compiler(), "-c", src, "-o", obj, "-O3", "-std=c++17", *ARCH, "-lineinfo",
           "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}", "--expt-relaxed-constexpr", *extra]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return obj


def build(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, verbose or ptxas_verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc(), *_host_compiler(), "-shared", *ARCH, "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    import sys

    print(build(verbose="-v" in sys.argv, ptxas_verbose="--ptxas" in sys.argv))
