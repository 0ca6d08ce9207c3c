"""Build libcm1g.so (the CUDA library) in-tree with nvcc for sm_100a."""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["cm1g_api.cu", "k_adv.cu", "k_sound.cu", "k_bc.cu", "k_misc.cu", "k_pdefq_noalloc.cu", "k_learned.cu"]
LIB = os.path.join(HERE, "libcm1g.so")

# --fmad=false: keep every binary32 product and sum rounded separately, as
# the reference's Fortran build does (no FMA contraction).
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "--fmad=false", "-Xcompiler", "-fPIC", "-Xptxas", "-O3", "-shared"]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def build(verbose=False, extra=()):
    srcs = [os.path.join(HERE, "csrc", s) for s in SRC]
    newest = max(os.path.getmtime(s) for s in srcs + [os.path.join(HERE, "csrc", "cm1g_common.cuh"),
                                                       os.path.join(HERE, "..", "include", "cm1g.h")])
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest and not extra:
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-o", LIB] + srcs
    host = "/usr/bin/g++"
    if os.path.exists(host):
        cmd[1:1] = ["-ccbin", host]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
