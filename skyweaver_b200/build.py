"""Build libskyweaver_b200.so (all CUDA kernels, the C ABI and the C++
drop-in host classes) in-tree with nvcc for sm_100a.

    python -m skyweaver_b200.build [--force] [--verbose]

Object files go to skyweaver_b200/_build/ (git-ignored); the shared library
lands next to this file so that it ships with the source tree.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libskyweaver_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "-rdc=false", "--expt-relaxed-constexpr",
    f"-I{os.path.join(REPO, 'include')}", f"-I{CSRC}",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    srcs += sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    srcs += sorted(glob.glob(os.path.join(CSRC, "host", "*.cu")))
    return srcs


def headers():
    return (glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True)
            + glob.glob(os.path.join(REPO, "include", "*.h")))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr_mtime = max((os.path.getmtime(h) for h in headers()), default=0)
    objs = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.relpath(src, CSRC).replace(os.sep, "_") + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj)
                and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime)):
            continue
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc()] + NVCC_FLAGS + ["-x", "cu", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    if force or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(args.force, args.verbose))


if __name__ == "__main__":
    main()
