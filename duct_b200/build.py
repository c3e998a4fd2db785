"""Build recipe of libductgpu.so (sm_100a only).

All CUDA sources under duct_b200/csrc are compiled by nvcc, one object per
source in parallel (duct_b200/lib/obj), and linked into one shared library,
duct_b200/lib/libductgpu.so, with the CUDA runtime linked statically (so the
library does not depend on which libcudart another component of the process
loaded) and cuSOLVER (one-time eigen setup) linked dynamically.  An object
is rebuilt when its source or any header is newer than it.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libductgpu.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")))


def _headers():
    return (glob.glob(os.path.join(SRC, "*.h")) + glob.glob(os.path.join(SRC, "*.cuh"))
            + glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def _obj(src):
    return os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")


def _needs(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(nvcc, src, verbose_ptxas):
    cmd = [nvcc, *ARCH, *FLAGS, "-c", "-o", _obj(src) + ".tmp", src]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s" % (src, r.stderr))
    os.replace(_obj(src) + ".tmp", _obj(src))
    return r.stderr


def build(force=False, verbose_ptxas=False):
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = os.path.join(CUDA, "bin", "nvcc")
    hdrs = _headers()
    todo = [s for s in sources() if force or verbose_ptxas or _needs(_obj(s), [s] + hdrs)]
    if todo:
        with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
            for s, log in zip(todo, ex.map(lambda s: _compile(nvcc, s, verbose_ptxas), todo)):
                if verbose_ptxas and log:
                    sys.stderr.write(log)
    objs = [_obj(s) for s in sources()]
    if todo or _needs(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *objs,
               "-L" + os.path.join(CUDA, "lib64"), "-lcusolver", "-ldl",
               "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
