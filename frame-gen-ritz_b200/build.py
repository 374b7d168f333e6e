"""Builds libframegen_b200.so in place: the CUDA kernels (sm_100a) and the C++ host code behind the C ABI.

python frame-gen-ritz_b200/build.py [--verbose]   (nvcc cross-compiles; no GPU needed)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libframegen_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("fg_kernels.cu", "fg_formats.cu", "fg_seednet.cu", "fg_seednet_tc.cu", "fg_seednet_bwd.cu", "fg_seednet_host.cpp",
                                                    "framegen.cpp", "fg_noalloc.cu", "fg_ui.cu", "fg_blur.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("fg_params.h", "fg_device.h", "fg_seednet.h", "fg_tc.h", "fg_blur.h")] + \
          [os.path.join(REPO, "include", "framegen.h"), os.path.join(REPO, "include", "framegen_c.h")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# -fmad=false: no contraction of a*b+c into an FMA anywhere (the kernels mirror numpy / OpenCV rounding step by step)
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-shared", "-I", os.path.join(REPO, "include"),
         "-I", os.path.join(HERE, "csrc")]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in SOURCES + HEADERS)


def build(verbose=False, force=False):
    if not force and not stale():
        return LIB
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", LIB + ".tmp"] + SOURCES
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
