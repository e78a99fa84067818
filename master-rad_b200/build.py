"""Builds librtb200.so (all CUDA sources, sm_100a only) next to the Python package.

nvcc flags: ``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -fmad=false``.
``-fmad=false`` is part of the arithmetic contract: no a*b+c is contracted, and every
fused multiply-add in the kernels is an explicit fmaf() (see csrc/rtb_device.cuh).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "rtb200", "librtb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = ["rtb_abi.cu", "rtb_scene.cu", "rtb_render.cu", "rtb_build.cu", "rtb_binned.cu", "rtb_static.cu", "rtb_batch.cu", "rtb_adjoint.cu", "rtb_calibrate.cu",
           "rtb_sbvh.cu"]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false",
         "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-DRTB_BUILD"]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "rtb200.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return OUT
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT] + \
        [os.path.join(CSRC, s) for s in SOURCES]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
