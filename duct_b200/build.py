"""Build recipe of libductgpu.so (sm_100a only).

All CUDA sources under duct_b200/csrc are compiled by nvcc into one shared
library, duct_b200/lib/libductgpu.so, with the CUDA runtime linked
statically (so the library does not depend on which libcudart another
component of the process loaded) and cuSOLVER (one-time eigen setup) linked
dynamically.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libductgpu.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(SRC, "*.h")) + glob.glob(
        os.path.join(HERE, "..", "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose_ptxas=False):
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = os.path.join(CUDA, "bin", "nvcc")
    cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-cudart", "static", "--expt-relaxed-constexpr",
           "-o", LIB + ".tmp", *sources(),
           "-L" + os.path.join(CUDA, "lib64"), "-lcusolver",
           "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
