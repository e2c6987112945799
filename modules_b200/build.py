"""Build libccgpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libccgpu.so")
SOURCES = ["csrc/cc_capi.cu", "csrc/cc_plan.cpp", "csrc/cc_noalloc.cu", "csrc/cc_serve.cu", "csrc/cc_multi.cu"]
HEADERS = ["csrc/cc_kernels.cuh", "csrc/cc_fused.cuh", "csrc/cc_lbfgs.cuh", "csrc/cc_plan.h", "csrc/cc_error.h", "csrc/cc_nufft.cuh", "csrc/cc_multi_launch.h", "../include/cc_gpu.h"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3", "-shared", "--expt-relaxed-constexpr", "-lcufft",
]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t for f in SOURCES + HEADERS + ["build.py"])


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB + ".tmp"] + [os.path.join(HERE, s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=HERE)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
