"""Build tests/_build/adapter_check: the GPU adapter compiled against the reference's own headers (needs the reference
tree; the binary then runs on a machine without it)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "_build", "adapter_check")


def build(reference=None):
    """Compile the check program; `reference` is the reference's source tree (default: CC_REFERENCE_TREE). Returns
    None without a tree."""
    reference = reference or os.environ.get("CC_REFERENCE_TREE")
    if not reference or not os.path.isdir(reference):
        return None
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-fopenmp", "-w",
           "-I" + os.path.join(ROOT, "oracle", "standins"), "-I" + os.path.join(reference, "core"),
           "-I" + os.path.join(reference, "potential"), "-I" + os.path.join(reference, "apps", "CCOptimization"),
           "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "adapter_check.cpp"), "-o", EXE,
           "-L" + os.path.join(ROOT, "oracle", "_ref"), "-lccref",
           "-L" + os.path.join(ROOT, "modules_b200"), "-l:libccgpu.so",
           "-Wl,-rpath,$ORIGIN/../../oracle/_ref:$ORIGIN/../../modules_b200"]
    subprocess.run(cmd, check=True)
    return EXE


if __name__ == "__main__":
    print(build())
