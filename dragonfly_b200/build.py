"""Builds the in-tree CUDA library dragonfly_b200/libdfgpu.so for sm_100a.

    python -m dragonfly_b200.build          # or dragonfly_b200.build.build()

nvcc cross-compiles without a GPU; the .so is built in the package directory
so that it travels with the source tree.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdfgpu.so")
SOURCES = ["emc_api.cu", "simulate.cu", "noalloc.cu", "proposal.cu", "probe.cu"]
PUBLIC_HEADER = os.path.join(os.path.dirname(HERE), "include", "dragonfly_b200.h")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared", "--expt-relaxed-constexpr",
]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    # every source and header under csrc/ (any of them may be included by a
    # translation unit), the public header and this recipe
    deps = glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [PUBLIC_HEADER, __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra_flags=()):
    if not force and not _stale():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + list(extra_flags) + ["-o", LIB] + \
        [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else ())
