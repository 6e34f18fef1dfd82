"""Builds the in-tree CUDA library lib/libmm_b200.so for sm_100a with nvcc.

Usage: python 2_b200/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmm_b200.so")
SOURCES = ["conv.cu", "mixed.cu", "rhs.cu", "demag_setup.cu", "plan.cu", "compat.cu", "noalloc.cu", "io.cpp", "am12.cu", "unet.cu"]
HEADERS = ["fft.cuh", "fft4.cuh", "mixed.cuh", "kernel_view.cuh", "pdl.cuh", "mm_internal.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--diag-suppress", "177"]


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    files += [os.path.join(CSRC, h) for h in HEADERS]
    files.append(os.path.join(HERE, "..", "include", "mm_b200.h"))
    files.append(os.path.join(HERE, "..", "include", "libmumax2_compat.h"))
    return [f for f in files if os.path.exists(f)]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in _inputs() + [os.path.abspath(__file__)])


def build(force=False, verbose=True):
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        if not os.path.exists(src):
            continue
        obj = os.path.join(objdir, s + ".o")
        cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        elif verbose and out:
            sys.stderr.write(out.decode())
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + objs + ["-lcudart"]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
