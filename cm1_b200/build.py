"""Build libcm1g.so (the CUDA library) in-tree with nvcc for sm_100a."""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["cm1g_api.cu", "k_adv.cu", "k_scal.cu", "k_sound.cu", "k_bc.cu", "k_misc.cu", "k_pdefq_noalloc.cu", "k_learned.cu", "k_stat.cu", "k_micro.cu", "k_io.cu", "k_diff2.cu", "k_turb.cu"]
LIB = os.path.join(HERE, "libcm1g.so")

# --fmad=false: keep every binary32 product and sum rounded separately, as
# the reference's Fortran build does (no FMA contraction).
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "--fmad=false", "-Xcompiler", "-fPIC", "-Xptxas", "-O3", "-shared"]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def build(verbose=False, extra=()):
    """Compiles each source to an object in parallel (in _build/ beside the
    sources), then links libcm1g.so."""
    srcs = [os.path.join(HERE, "csrc", s) for s in SRC]
    heads = [os.path.join(HERE, "csrc", h) for h in os.listdir(os.path.join(HERE, "csrc")) if h.endswith(".cuh")]
    newest = max(os.path.getmtime(s) for s in srcs + heads + [os.path.join(HERE, "..", "include", "cm1g.h")])
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest and not extra:
        return LIB
    host = "/usr/bin/g++"
    base = [nvcc()] + (["-ccbin", host] if os.path.exists(host) else [])
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"] + list(extra)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, procs = [], []
    for src in srcs:
        obj = os.path.join(objdir, os.path.splitext(os.path.basename(src))[0] + ".o")
        cmd = base + compile_flags + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [src for src, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc " + " ".join(os.path.basename(f) for f in failed))
    cmd = base + ["-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
