"""The four flip-symmetric passes of a solve as one persistent launch
(DUCTGPU_PASS_PARITY_QUEUE): tiles taken in pass order from a global
counter, a plane's pass starting once per-plane counters show its earlier
passes done.  The tile code and its K order are those of the per-pass
launches (DUCTGPU_PASS_PARITY), so the results must be bit-identical, for
every half-block size (n = 63, 127, 191: 32, 64, 96 rows), Dirichlet and
Neumann fields together, directly and replayed from a captured graph."""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth

pytestmark = pytest.mark.gpu


def batch(ctx, m, nm):
    xalp = 0.5 * np.arange(nm)
    fields, keep = [], []
    for k, (bound, lam) in enumerate((("d", 4.0e4), ("d", 4.0e4), ("d", 4.0e4), ("n", 0.0))):
        f = synth.chebyshev_rhs(m, m, nm, seed=50 + k, ib=0)
        r, s = ctx.device_array(f.shape), ctx.device_array(f.shape)
        r.upload(f)
        keep += [r, s]
        fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lam, ib=0, bound=bound))
    return fields, keep


@pytest.mark.parametrize("m,nm", [(65, 12), (129, 8), (193, 6)])
def test_queued_passes_equal_per_pass_launches(m, nm):
    with D.Context(0) as ctx:
        ctx.pseudomat(m)
        fields, keep = batch(ctx, m, nm)
        out = {}
        for kernel in (D.PASS_PARITY, D.PASS_PARITY_QUEUE):
            ctx.set_pass_kernel(kernel)
            ctx.profile(True)
            ctx.profile_reset()
            ctx.solve_fields_dev(fields, precision=D.PREC_FP64)
            ctx.synchronize()
            _, npass = ctx.profile_read(D.K_PASS_FP64)
            ctx.profile(False)
            assert npass == (1 if kernel == D.PASS_PARITY_QUEUE else 4)
            out[kernel] = [f["sol"].download() for f in fields]
        for a, b in zip(out[D.PASS_PARITY], out[D.PASS_PARITY_QUEUE]):
            assert np.all(np.isfinite(a)) and np.array_equal(a, b)
        # replayed from a captured graph (the counters are reset inside it)
        gid = ctx.graph_create(fields)
        for f in fields:
            f["sol"].upload(np.zeros(f["sol"].shape, dtype=complex, order="F"))
        for _ in range(2):
            ctx.graph_launch(gid)
        ctx.synchronize()
        for f, b in zip(fields, out[D.PASS_PARITY]):
            assert np.array_equal(f["sol"].download(), b)
        ctx.graph_destroy(gid)
        ctx.set_pass_kernel(-1)
        for x in keep:
            x.free()
