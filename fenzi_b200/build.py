"""Builds the in-tree CUDA libraries for sm_100a: fenzi_b200/libfenzi_b200.so (the
product) and fenzi_b200/libfenzi_plain.so (the plain comparator path, which links
the product library and cuFFT).

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
PLAIN_LIB = os.path.join(HERE, "libfenzi_plain.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    c = os.path.join(HERE, "csrc")
    return sorted(glob.glob(os.path.join(c, "*.cu")) + glob.glob(os.path.join(c, "kernels", "*.cu"))
                  + glob.glob(os.path.join(c, "host", "*.cpp")))


def plain_sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "plain", "*.cu")))


def headers():
    c = os.path.join(HERE, "csrc")
    return (glob.glob(os.path.join(c, "**", "*.h"), recursive=True)
            + glob.glob(os.path.join(c, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date(lib=LIB, srcs=None):
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in (srcs or sources()) + headers())


def _compile(srcs, objdir, verbose):
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in srcs:
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
    return nvcc, objs


def build(force: bool = False, verbose: bool = False) -> str:
    if force or not up_to_date():
        nvcc, objs = _compile(sources(), os.path.join(HERE, "_build"), verbose)
        subprocess.check_call([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    if force or not up_to_date(PLAIN_LIB, plain_sources()) or os.path.getmtime(PLAIN_LIB) < os.path.getmtime(LIB):
        nvcc, objs = _compile(plain_sources(), os.path.join(HERE, "_build", "plain"), verbose)
        subprocess.check_call([nvcc, *ARCH, "-shared", "-o", PLAIN_LIB, *objs, "-L", HERE, "-lfenzi_b200", "-lcufft",
                               "-lcudart", "-Xlinker", "-rpath,$ORIGIN", "-Xlinker", "-rpath,/usr/local/cuda/lib64"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
