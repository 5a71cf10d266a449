"""Builds the in-tree CUDA library fenzi_b200/libfenzi_b200.so for sm_100a.

Usage: python -m fenzi_b200.build   (or fenzi_b200.build.build())
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libfenzi_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    c = os.path.join(HERE, "csrc")
    return sorted(glob.glob(os.path.join(c, "*.cu")) + glob.glob(os.path.join(c, "kernels", "*.cu"))
                  + glob.glob(os.path.join(c, "host", "*.cpp")))


def headers():
    c = os.path.join(HERE, "csrc")
    return (glob.glob(os.path.join(c, "**", "*.h"), recursive=True)
            + glob.glob(os.path.join(c, "**", "*.cuh"), recursive=True)
            + [os.path.join(ROOT, "include", "fenzi_b200.h")])


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
               "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(f"--- {os.path.relpath(src, ROOT)}\n{out}")
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    subprocess.check_call([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
