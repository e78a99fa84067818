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
# The reference checkout: RTB_REFERENCE_ROOT, or --reference-root on the command line.
REF_ROOT = os.environ.get("RTB_REFERENCE_ROOT", "/root/reference")
KERNEL_SUBPATH = "src/xyz/marsavic/gfxlab/gpu/GpuKernelSources.java"


def kernel_source(ref_root=None):
    return os.path.join(ref_root or REF_ROOT, KERNEL_SUBPATH)
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


def extract_reference_kernel(dst, ref_root=None):
    """Copies the PATH_TRACER text block (two blocks joined by .concat) to ``dst``."""
    text = open(kernel_source(ref_root), encoding="utf-8").read()
    m = re.search(r'PATH_TRACER = """\n(.*?)""".concat\("""\n(.*?)"""\);', text, re.S)
    if not m:
        raise RuntimeError("PATH_TRACER text block not found")
    body = m.group(1) + m.group(2)
    if "\\" in body:
        raise RuntimeError("unexpected escape sequence in the kernel text block")
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    with open(dst, "w", encoding="utf-8") as f:
        f.write(body)


def build_reference(force=False, ref_root=None):
    ref_dir = os.path.join(HERE, "_ref")
    ksrc = kernel_source(ref_root)
    if not os.path.exists(ksrc):
        return None
    src = os.path.join(ref_dir, "ref_kernel.cu")
    harness = os.path.join(HERE, "ref_harness.cu")
    if force or _stale(src, [ksrc]):
        extract_reference_kernel(src, ref_root)
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


def build(force=False, ref_root=None):
    build_cpu(force)
    build_reference(force, ref_root)


if __name__ == "__main__":
    root = None
    if "--reference-root" in sys.argv:
        root = sys.argv[sys.argv.index("--reference-root") + 1]
    build(force="--force" in sys.argv, ref_root=root)
