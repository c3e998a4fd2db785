"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/duct_oracle.c and oracle/duct_oracle_dns.c into oracle/libduct_oracle.so, linked against
the OpenBLAS build bundled with SciPy (LP64 LAPACK/BLAS exported with a
``scipy_`` prefix), with OpenMP for the mode loop of the CPU baseline.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libduct_oracle.so")


def _openblas():
    import scipy  # noqa: F401  (locates the bundled OpenBLAS)
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError("SciPy's bundled OpenBLAS was not found in %s" % libdir)
    return libdir, os.path.basename(cands[0])


def build(force=False):
    srcs = [os.path.join(HERE, f) for f in ("duct_oracle.c", "duct_oracle_dns.c")]
    hdrs = [os.path.join(HERE, f) for f in ("duct_oracle.h", "orc_fft.h")]
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(f) for f in srcs + hdrs)):
        return LIB
    libdir, name = _openblas()
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-std=c11", "-Wall",
           "-o", LIB, *srcs, "-L" + libdir, "-l:" + name, "-Wl,-rpath," + libdir, "-lm"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
