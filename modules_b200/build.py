"""Build libccgpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libccgpu.so")
SOURCES = ["csrc/cc_capi.cu", "csrc/cc_batch.cu", "csrc/cc_minimize.cu", "csrc/cc_plan.cpp", "csrc/cc_noalloc.cu", "csrc/cc_serve.cu",
           "csrc/cc_multi.cu"]
HEADERS = ["csrc/cc_internal.h", "csrc/cc_kernels.cuh", "csrc/cc_lbfgs.cuh", "csrc/cc_plan.h", "csrc/cc_error.h", "csrc/cc_nufft.cuh", "csrc/cc_multi_launch.h", "../include/cc_gpu.h"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
]
OBJDIR = os.path.join(HERE, "_build")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t for f in SOURCES + HEADERS + ["build.py"])


def build(force=False, verbose=False):
    """Compile every source to an object (in parallel, for sm_100a) and link libccgpu.so."""
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    os.makedirs(OBJDIR, exist_ok=True)
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas=-v"] if verbose else []) + ["-c", os.path.join(HERE, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        objs.append(obj)
        procs.append((cmd, subprocess.Popen(cmd, cwd=HERE)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp"] + objs + ["-lcufft"]
    subprocess.run(link, check=True, cwd=HERE)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
