"""The GEMM-pass kernel variants (staged operator with 32 or 16 lines per
CTA, register-streamed operator, persistent) and the autotuner that picks
between them: these variants give the same solution bit for bit (same K
order in every DMMA chain); the flip-symmetric variant (another, equally
valid, decomposition: tests/test_gpu_parity.py) is among the autotuner's
candidates, and the autotuner's choice is one of them."""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu
VARIANTS = [D.PASS_STAGED, D.PASS_STAGED16, D.PASS_REGISTER, D.PASS_PERSIST]


def fields_for(ctx, m, nm):
    xalp = 0.5 * np.arange(nm)
    out, keep = [], []
    for i, (bound, lam) in enumerate([("d", 4.0e6), ("n", 0.0)]):
        f = synth.chebyshev_rhs(m, m, nm, seed=10 + i, ib=0)
        r, s = ctx.device_array(f.shape), ctx.device_array(f.shape)
        r.upload(f)
        keep += [r, s]
        out.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=bound))
    return out, keep


@pytest.mark.parametrize("m,nm", [(33, 5), (65, 8), (129, 6), (193, 3)])
def test_variants_agree_and_autotune(gpu_ctx, m, nm):
    gpu_ctx.pseudomat(m)
    fl, keep = fields_for(gpu_ctx, m, nm)
    try:
        sols = []
        for v in VARIANTS:
            gpu_ctx.set_pass_kernel(v)
            gpu_ctx.solve_fields_dev(fl)
            gpu_ctx.synchronize()
            sols.append([f["sol"].download() for f in fl])
        for s in sols[1:]:
            for a, b in zip(s, sols[0]):
                assert np.array_equal(a, b)
        gpu_ctx.set_pass_kernel(D.PASS_PARITY)
        gpu_ctx.solve_fields_dev(fl)
        gpu_ctx.synchronize()
        par = [f["sol"].download() for f in fl]
        chosen = gpu_ctx.autotune(fl, reps=2)
        folded = (D.PASS_PARITY, D.PASS_PARITY_QUEUE)    # bit-identical to each other
        assert chosen in VARIANTS + list(folded)
        gpu_ctx.solve_fields_dev(fl)
        gpu_ctx.synchronize()
        for f, b in zip(fl, par if chosen in folded else sols[0]):
            assert np.array_equal(f["sol"].download(), b)
    finally:
        gpu_ctx.set_pass_kernel(-1)   # the library's defaults
        for x in keep:
            x.free()
