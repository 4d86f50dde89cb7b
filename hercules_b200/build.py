"""Builds the in-tree native artefacts of hercules_b200.

  libhercules_gpu.so   the C ABI of include/hercules_gpu.h (sm_100a kernels +
                       host code), CUDA runtime linked statically
  bin/hercules         the reference-compatible command line (C), linked
                       against libhercules_gpu.so

Device code is compiled with -fmad=false and host code with
-ffp-contract=off: the float arithmetic must match the reference's
operation order exactly, so no multiply-add may be fused.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhercules_gpu.so")
CLI = os.path.join(HERE, "bin", "hercules")

SOURCES = ["hg_kernels.cu", "hg_index.cu", "hg_noalloc.cu", "hg_batch.cu", "hg_umma.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    out = []
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".h", ".c")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(ROOT, "include", "hercules_gpu.h"))
    return out


def build_lib(force=False, verbose=False):
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if not force and not _newer(LIB, _deps()):
        return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
           "-Xcompiler", "-fPIC,-O2,-ffp-contract=off,-fvisibility=hidden",
           "-Xptxas", "-v" if verbose else "-O3",
           "-I" + os.path.join(ROOT, "include"), "-shared", "-o", LIB + ".tmp", *srcs, "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_cli(force=False):
    src = os.path.join(CSRC, "hercules_cli.c")
    if not os.path.exists(src):
        return None
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    if not force and not _newer(CLI, [src, LIB]):
        return CLI
    cmd = ["gcc", "-O2", "-std=gnu11", "-Wall", "-I" + os.path.join(ROOT, "include"), "-o", CLI, src,
           "-L" + HERE, "-lhercules_gpu", "-Wl,-rpath,$ORIGIN/..", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("gcc failed for the CLI")
    return CLI


def build(force=False, verbose=False):
    build_lib(force, verbose)
    build_cli(force)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
