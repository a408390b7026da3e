"""Builds libvkzg.so (the C ABI of include/vkzg.h) in-tree with nvcc for sm_100a.

    python -m vkzg_b200.build [--verbose]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvkzg.so")
SOURCES = ["proof_kernels.cu", "recover_kernels.cu", "cells_kernels.cu", "setup_kernels.cu", "prover.cu",
           "server.cu", "diagnostics.cu"]
HEADERS = ["field.cuh", "field_f64.cuh", "curve.cuh", "inverse.cuh", "device_util.cuh", "bucket_sum.cuh", "kernels.h",
           "comb_windows.h", "glv.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "vkzg.h"),
                                                         os.path.join(ROOT, "include", "vkzg_b200.h")]
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", path, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        subprocess.check_call([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-ldl"])
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
