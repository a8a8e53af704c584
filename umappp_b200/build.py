"""Builds libumappp_b200.so in-tree with nvcc for sm_100a.

Usage: python -m umappp_b200.build [--force] [-j N]

Per-file flags: the stages whose results must round exactly as the
reference's -ffp-contract=off build (similarities, graph, sgd) are compiled
with -fmad=false; host code is compiled with -ffp-contract=off.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libumappp_b200.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                 "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "--expt-relaxed-constexpr"]
NO_FMAD = {"similarities.cu", "graph.cu", "sgd.cu"}
SOURCES = ["capi.cu", "memory.cu", "knn.cu", "knn_tc.cu", "knn_tc16.cu", "knn_tree.cu", "similarities.cu", "graph.cu", "spectral.cu", "sgd.cu", "adjoint.cu", "probe.cu",
           "find_ab.cpp"]


def _flags(src: str) -> list[str]:
    f = list(COMMON)
    if src in NO_FMAD:
        f.append("-fmad=false")
    if src.endswith(".cpp"):
        f += ["-x", "cu"]
    return f


def _headers_mtime() -> float:
    m = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for name in os.listdir(d):
            if name.endswith((".cuh", ".h", ".hpp")):
                m = max(m, os.path.getmtime(os.path.join(d, name)))
    return m


def _compile(src: str, force: bool, hm: float, verbose: bool) -> str:
    out = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(path), hm):
        return out
    cmd = [NVCC] + _flags(src) + ["-c", path, "-o", out]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return out


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hm = _headers_mtime()
    jobs = jobs or min(len(SOURCES), os.cpu_count() or 4)
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hm, verbose), SOURCES))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xlinker", "-soname=libumappp_b200.so"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))


if __name__ == "__main__":
    main()
