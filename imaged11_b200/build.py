"""Compile the CUDA sources of imaged11_b200 into one in-tree shared library.

    python -m imaged11_b200.build

nvcc cross-compiles for sm_100a without a GPU.  The library lands next to this
file (``libimaged11_b200.so``) so that it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libimaged11_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def build(verbose=False, extra=(), out=None, objdir=None):
    """Compile every .cu under csrc/ and link libimaged11_b200.so (or `out`,
    with extra nvcc flags such as -DID11B_SCORE_UBIS_PER_THREAD=8)."""
    objdir = objdir or os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, *extra, "-I", os.path.join(HERE, "..", "include"),
               "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", out or LIB, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out or LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
