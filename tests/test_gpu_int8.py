"""The FP64-accurate solve with int8-emulated GEMM passes (DUCTGPU_PREC_INT8:
every pass as 28 products of 7-bit int8 slices on tcgen05 with exact int32
accumulation, no refinement) against the FP64 DMMA path and the oracle.

Tolerance: the same 1e-12 relative bound as the FP64 tests (the emulated
products are exact up to the dropped slice terms, ~2^-49 of the row and
column scales; measured ~1e-13 at my = 129)."""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


@pytest.mark.parametrize("m,nm", [(33, 17), (65, 8), (129, 64)])
def test_int8_matches_fp64_batched(gpu_ctx, m, nm):
    gpu_ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nm)
    specs = [("d", 4.0e6), ("d", 2.5), ("n", 0.0)]
    fl, keep = [], []
    for i, (bound, lam) in enumerate(specs):
        f = synth.chebyshev_rhs(m, m, nm, seed=20 + i, ib=0)
        r, s = gpu_ctx.device_array(f.shape), gpu_ctx.device_array(f.shape)
        r.upload(f)
        keep += [r, s]
        fl.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=bound))
    try:
        # the FP64 passes on the full operators, which the int8 passes emulate
        gpu_ctx.set_pass_kernel(D.PASS_STAGED)
        gpu_ctx.solve_fields_dev(fl, D.PREC_FP64)
        gpu_ctx.synchronize()
        gpu_ctx.set_pass_kernel(-1)
        ref = [f["sol"].download() for f in fl]
        gpu_ctx.solve_fields_dev(fl, D.PREC_INT8)
        gpu_ctx.synchronize()
        for f, r in zip(fl, ref):
            got = f["sol"].download()
            assert rel(got, r) < TOL
            assert np.all(got[:, :, 0].imag == 0)
    finally:
        for x in keep:
            x.free()


def test_int8_helm3d_against_oracle(gpu_ctx, oracle):
    m, nm = 65, 4
    f = synth.chebyshev_rhs(m, m, nm, seed=7, ib=0)
    xalp = np.array([0.0, 1.0, 2.0, 3.0])
    ops = oracle.Ops(m)
    ref, _ = oracle.helm3d(f, ops, "d", 3.0, xalp)
    got = gpu_ctx.helm3d(f.copy(order="F"), "d", 3.0, xalp, ipro=0, precision=D.PREC_INT8)
    assert rel(got, ref) < TOL


def test_int8_rejects_large_grids(gpu_ctx):
    gpu_ctx.pseudomat(193)
    f = synth.chebyshev_rhs(193, 193, 1, seed=1, ib=0)
    with pytest.raises(D.DuctGPUError):
        gpu_ctx.helm3d(f, "d", 1.0, [0.0], precision=D.PREC_INT8)
