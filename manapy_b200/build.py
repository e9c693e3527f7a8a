"""Build ``lib/libmanapy_b200.so`` from ``csrc/*.cu`` for sm_100a with nvcc."""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "lib", "libmanapy_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


# Per-file options.  The FP32-compensated kernels are compiled without multiply-add
# contraction: every FP32 operation rounds as written (explicit fmaf calls excepted), so
# the single-mesh and batched instantiations of one block body give identical bits.  The
# Euler kernels likewise round every FP64 operation as manapy's (uncontracted) code does.
FILE_FLAGS = {"fv_advdiff_f32c.cu": ["-fmad=false"], "fv_sw_f32c.cu": ["-fmad=false"],
              "fv_euler.cu": ["-fmad=false"]}


def build(verbose=False, force=False):
    """Compile every ``csrc/*.cu`` for sm_100a (objects in parallel) and link the library."""
    from concurrent.futures import ThreadPoolExecutor
    srcs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    hdrs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [os.path.join(ROOT, "include", "manapy_b200.h")]
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(s) <= t for s in srcs + hdrs + [os.path.abspath(__file__)]):
            build_host()
            return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    objdir = os.path.join(HERE, "lib", "obj")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
    if verbose:
        common.append("-Xptxas=-v")

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        subprocess.run(common + FILE_FLAGS.get(os.path.basename(src), []) + ["-c", src, "-o", obj], check=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs], check=True)
    os.replace(OUT + ".tmp", OUT)
    build_host(force=force)
    return OUT


HOST_OUT = os.path.join(HERE, "lib", "libmanapy_b200_host.so")


def build_host(force=False):
    """The native host mesh builder (``host/*.cpp``, C++17, no GPU code)."""
    srcs = sorted(glob.glob(os.path.join(HERE, "host", "*.cpp")))
    hdrs = sorted(glob.glob(os.path.join(HERE, "host", "*.hpp")))
    if not force and os.path.exists(HOST_OUT):
        t = os.path.getmtime(HOST_OUT)
        if all(os.path.getmtime(s) <= t for s in srcs + hdrs + [os.path.abspath(__file__)]):
            return HOST_OUT
    os.makedirs(os.path.dirname(HOST_OUT), exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-ffp-contract=off", "-o",
                    HOST_OUT + ".tmp", *srcs],
                   check=True)
    os.replace(HOST_OUT + ".tmp", HOST_OUT)
    return HOST_OUT


if __name__ == "__main__":
    print(build(verbose=True, force=True))
