"""Builds the oracle (test infrastructure; never loaded by the product path).

* ``oracle/liboracle.so``: the C++ restatements (BVH builder, FP32 closest hit and sample
  loop, FP64 CPU path tracer), compiled with ``-ffp-contract=off`` so that their IEEE
  arithmetic is not contracted.
* ``oracle/_ref/libref_fmad.so`` and ``oracle/_ref/libref_nofmad.so``: the reference's own
  CUDA source (the ``PATH_TRACER`` text block of
  ``src/xyz/marsavic/gfxlab/gpu/GpuKernelSources.java``), extracted verbatim from the
  reference tree into the git-ignored ``oracle/_ref/`` and compiled with nvcc for sm_100a
  around ``oracle/ref_harness.cu``.  The default build matches what NVRTC does for the
  reference (``-fmad=true``); the second disables contraction.  This step runs only where
  the reference tree is present; elsewhere the prebuilt libraries are used as they are.
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = "/root/reference"
KERNEL_SOURCE = os.path.join(
    REF_ROOT, "src/xyz/marsavic/gfxlab/gpu/GpuKernelSources.java")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_cpu(force=False):
    out = os.path.join(HERE, "liboracle.so")
    srcs = [os.path.join(HERE, f) for f in
            ("oracle_bvh.cpp", "oracle_trace.cpp", "oracle_cpu.cpp")]
    if force or _stale(out, srcs):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
              "-ffp-contract=off", "-fno-fast-math", "-o", out] + srcs)
    return out


def extract_reference_kernel(dst):
    """Copies the PATH_TRACER text block (two blocks joined by .concat) to ``dst``."""
    text = open(KERNEL_SOURCE, encoding="utf-8").read()
    m = re.search(r'PATH_TRACER = """\n(.*?)""".concat\("""\n(.*?)"""\);', text, re.S)
    if not m:
        raise RuntimeError("PATH_TRACER text block not found")
    body = m.group(1) + m.group(2)
    if "\\" in body:
        raise RuntimeError("unexpected escape sequence in the kernel text block")
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    with open(dst, "w", encoding="utf-8") as f:
        f.write(body)


def build_reference(force=False):
    ref_dir = os.path.join(HERE, "_ref")
    if not os.path.exists(KERNEL_SOURCE):
        return None
    src = os.path.join(ref_dir, "ref_kernel.cu")
    harness = os.path.join(HERE, "ref_harness.cu")
    if force or _stale(src, [KERNEL_SOURCE]):
        extract_reference_kernel(src)
    outs = {}
    for name, flags in (("fmad", ["-fmad=true"]), ("nofmad", ["-fmad=false"]),
                        ("metrics", ["-fmad=false", "-DGFXLAB_RENDER_METRICS=1"])):
        out = os.path.join(ref_dir, "libref_%s.so" % name)
        if force or _stale(out, [src, harness]):
            _run([NVCC] + ARCH + ["-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
                                  "-DBVH_STACK_SIZE=32", "-I", ref_dir] + flags +
                 ["-o", out, harness])
        outs[name] = out
    return outs


def build(force=False):
    build_cpu(force)
    build_reference(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
